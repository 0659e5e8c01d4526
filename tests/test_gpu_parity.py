"""Parity of the CUDA path (through the C-ABI library) with the reference.

The golden vectors were produced by the reference binary itself
(tests/golden/make_golden.py); the CPU oracle reproduces them bit for bit
(tests/test_oracle_golden.py) and supplies the quantities the reference does
not dump (footpoint tables, moments).

Tolerances, per the specification of the path:
* integer work (footpoint indices, outside flags, chain layout) and the host
  set-up (initial grid, chain values): bit-exact;
* FP64 path: |f_gpu - f_ref| <= 1e-12 * max|f_ref| after every saved step
  (the GPU solves the same spline systems with a different operation order);
* FP32-bulk path: relative L2 error <= 2e-6 and max error <= 1e-5 * max|f_ref|
  per saved step (FP32 storage and gathers, FP64 recursions).
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle.vls_oracle import Oracle

pytestmark = pytest.mark.gpu

SMALL = golden_cases(full_only=True)
LARGE = golden_cases(full_only=False)

FP64_TOL = 1e-12
FP32_L2 = 2e-6
FP32_MAX = 1e-5


def solver(cfg, precision="fp64", **over):
    from vlasolve_b200 import VlasovSolver21Spline
    c = dict(cfg)
    c.update(over)
    return VlasovSolver21Spline(c, precision=precision)


def _saved_steps(g, prefix):
    return sorted(int(k[len(prefix):]) for k in g.files if k.startswith(prefix))


@pytest.mark.parametrize("name", SMALL)
def test_initial_state_and_chains_bitexact(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    assert s.shape == tuple(g["shape"])
    np.testing.assert_array_equal(s.f, g["f_0"])
    ch = s.chains()
    if "chain0_cell" in g.files:
        for k in ("cell", "len", "R", "U", "val"):
            np.testing.assert_array_equal(ch[k], g["chain0_" + k], err_msg=k)
    else:
        assert len(ch["cell"]) == 0


@pytest.mark.parametrize("name", SMALL)
def test_footpoints_bitexact(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    o = Oracle(cfg)
    a, b = s.footpoints(), o.footpoints()
    for k in ("rI", "uI", "out", "rF", "uF", "driftR"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("name", SMALL)
def test_fp64_steps_match_reference(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    cur = 0
    for st in _saved_steps(g, "f_"):
        s.step(st - cur)
        cur = st
        ref = g["f_%d" % st]
        err = np.abs(s.f - ref).max()
        assert err <= FP64_TOL * np.abs(ref).max(), (name, st, err)


@pytest.mark.parametrize("prec", ["fp32", "fp32all"])
@pytest.mark.parametrize("name", SMALL)
def test_fp32_steps_match_reference(name, prec):
    g, cfg = load_golden(name)
    s = solver(cfg, prec)
    cur = 0
    for st in _saved_steps(g, "f_"):
        s.step(st - cur)
        cur = st
        ref = g["f_%d" % st]
        d = s.f - ref
        l2 = np.linalg.norm(d) / np.linalg.norm(ref)
        print(f"{name} {prec} step {st}: L2 rel {l2:.3e}")
        assert l2 <= FP32_L2, (name, st, l2)
        assert np.abs(d).max() <= FP32_MAX * np.abs(ref).max(), (name, st)


@pytest.mark.parametrize("name", ["udf_tiny", "plummer_small", "udf_nolink"])
def test_moments_match_oracle(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    o = Oracle(cfg)
    for _ in range(2):
        b1, M1, t1 = s.moments()
        b2, M2, t2 = o.moments()
        np.testing.assert_allclose(b1, b2, rtol=1e-13, atol=1e-15 * abs(t2))
        np.testing.assert_allclose(M1, M2, rtol=1e-13, atol=1e-15 * abs(t2))
        assert t1 == pytest.approx(t2, rel=1e-14)
        s.step(1)
        o.step(1)
        o.f = s.f  # keep both on the same state


@pytest.mark.parametrize("name", ["udf_tiny", "hernquist_small", "pldf_small"])
def test_stats_match_reference(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    ref = g["stats"]
    for st in range(min(3, len(ref))):
        row = s.stats()
        got = [row[k] for k in ("Mass", "E", "Ek", "Ep", "S", "L1", "L2")]
        # the reference prints 10 significant digits
        np.testing.assert_allclose(got, ref[st][2:], rtol=2e-9, atol=1e-14)
        s.step(1)


@pytest.mark.parametrize("name", LARGE)
def test_full_config_fp64_sampled(name):
    g, cfg = load_golden(name)
    s = solver(cfg)
    idx = g["sample_idx"]
    cur = 0
    for st in _saved_steps(g, "fs_"):
        s.step(st - cur)
        cur = st
        f = s.f
        fs = f.ravel()[idx]
        ref = g["fs_%d" % st]
        scale = np.abs(ref).max()
        if st == 0:
            np.testing.assert_array_equal(fs, ref)
        assert np.abs(fs - ref).max() <= FP64_TOL * scale, (name, st)
        np.testing.assert_allclose(f.reshape(f.shape[0], -1).sum(axis=1),
                                   g["slicesum_%d" % st], rtol=1e-11,
                                   atol=1e-12 * np.abs(g["slicesum_%d" % st]).max())


@pytest.mark.parametrize("prec", ["fp32", "fp32all"])
@pytest.mark.parametrize("name", LARGE)
def test_full_config_fp32_sampled(name, prec):
    """Every full-size configuration (the 1025-vertex r and v_r lines of
    pldf_1025 included) in both FP32 modes, with the default kernel layouts."""
    g, cfg = load_golden(name)
    s = solver(cfg, prec)
    idx = g["sample_idx"]
    cur = 0
    for st in _saved_steps(g, "fs_"):
        s.step(st - cur)
        cur = st
        fs = s.f.ravel()[idx]
        ref = g["fs_%d" % st]
        err = np.abs(fs - ref).max() / np.abs(ref).max()
        print(f"{name} {prec} step {st}: max rel err {err:.3e}")
        assert err <= FP32_MAX, st


def test_linearity_without_gravity_full_size():
    """With G = 0 the kick shift vanishes and the step is linear in f (the
    chains carry zeros): step(f1 + 2 f2) = step(f1) + 2 step(f2), checked on
    the 513x513x256 grid where the oracle would be too slow."""
    from vlasolve_b200 import VlasovSolver21Spline
    g, cfg = load_golden("hernquist_cfg3")
    # the Hernquist distribution function needs G (with G = 0 it is NaN
    # everywhere, which the upload reports): the grid comes from a G = 1 handle
    s1 = solver(cfg, "fp32")
    f0 = s1.f
    s1.close()
    s = VlasovSolver21Spline(dict(cfg, G=0.0), precision="fp32", init=False)
    rng = np.random.default_rng(7)
    f1 = f0 * (1 + 0.1 * rng.standard_normal(f0.shape))
    f2 = f0[::-1, :, :].copy()
    outs = []
    for x in (f1, f2, f1 + 2 * f2):
        s.f = x
        s.set_chain_values(np.zeros(len(s.chains()["val"])))
        s.step(1)
        outs.append(s.f)
    lhs, rhs = outs[2], outs[0] + 2 * outs[1]
    assert np.abs(lhs - rhs).max() <= 1e-6 * np.abs(rhs).max()


def test_ndfield_roundtrip_and_layout():
    g, cfg = load_golden("udf_tiny")
    s = solver(cfg)
    s.step(2)
    f = s.f
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "snap.ND")
        s.snapshot(p)
        b = open(p, "rb").read()
        n = f.size
        assert len(b) == 688 + 8 * n + 4
        np.testing.assert_array_equal(np.frombuffer(b[688:688 + 8 * n], "<f8"), f.ravel())
        assert b[24 + 4: 24 + 4 + 11] == b"1 1 0 1 2 0"
        s2 = solver(cfg)
        s2.load_snapshot(p)
        np.testing.assert_array_equal(s2.f, f)


def test_ndfield_writer_matches_reference_file_bytes():
    """The reference's own snapshot of udf_tiny after one step
    (tests/golden/udf_tiny_snapshot_step1.ND): read into a handle, written back
    by vls_write_ndfield, the two files are identical byte for byte."""
    ref_path = os.path.join(os.path.dirname(__file__), "golden", "udf_tiny_snapshot_step1.ND")
    ref = open(ref_path, "rb").read()
    g, cfg = load_golden("udf_tiny")
    s = solver(cfg)
    s.load_snapshot(ref_path)
    np.testing.assert_array_equal(s.f, g["f_1"])
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "snap.ND")
        s.snapshot(p)
        assert open(p, "rb").read() == ref


def test_ndfield_record_marker_above_2gib():
    """1025 x 1025 x 256 cells: 2.15 GB of FP64 data, whose int record marker
    wraps exactly as the reference's (NDfield.hxx:355); the file reads back."""
    import struct
    cfg = {"type": "Hernquist", "Pmin": 0.01, "Pmax": 50.0, "Pres": 1024,
           "Pscale": "logarithmic", "Umin": (-3.0, 0.0), "Umax": (3.0, 3.0),
           "Ures": (1024, 256), "Uscale": ("linear", "quadratic"), "dt": 0.0025}
    s = solver(cfg, "fp32")
    n = 1025 * 1025 * 256
    wrapped = struct.unpack("<i", struct.pack("<I", (8 * n) % 2 ** 32))[0]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "big.ND")
        s.snapshot(p)
        assert os.path.getsize(p) == 688 + 8 * n + 4
        with open(p, "rb") as fh:
            fh.seek(684)
            assert struct.unpack("<i", fh.read(4))[0] == wrapped
            fh.seek(688 + 8 * n)
            assert struct.unpack("<i", fh.read(4))[0] == wrapped
            fh.seek(688 + 8 * (n - 3))
            tail = np.frombuffer(fh.read(24), "<f8")
        f = s.f
        np.testing.assert_array_equal(tail, f.ravel()[-3:])
        s.f = np.zeros_like(f)
        s.load_snapshot(p)
        np.testing.assert_array_equal(s.f, f)


def test_reflective_kernel_where_the_reference_halts_is_an_error():
    """kernelBufferSize > 0 with the reflective kernel reaches the branch
    where the reference terminates (vlasovSolver21.hxx:389-391); vls_create
    returns VLS_EINVAL naming it instead."""
    from vlasolve_b200 import _lib
    g, cfg = load_golden("udf_reflect")
    with pytest.raises(_lib.VlsError) as e:
        solver(cfg, kernelBufferSize=2)
    assert e.value.code == _lib.VLS_EINVAL
    assert "reflect" in str(e.value)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_nonfinite_grid_is_reported(prec):
    """A NaN placed in the host grid: vls_set_f loads it and returns VLS_ENAN;
    a step from that state is reported by the enclosed-mass scan at the next
    vls_sync; a clean grid clears the state; an infinity in the chain values
    is reported by vls_set_chain_values."""
    from vlasolve_b200 import _lib
    g, cfg = load_golden("udf_rect_kbuf")
    s = solver(cfg, prec)
    f = s.f
    bad = f.copy()
    bad[2, 5, 7] = np.nan
    with pytest.raises(_lib.VlsError) as e:
        s.f = bad
    assert e.value.code == _lib.VLS_ENAN
    s.step(1)
    with pytest.raises(_lib.VlsError) as e:
        s.sync()
    assert e.value.code == _lib.VLS_ENAN
    assert "total mass" in str(e.value)
    s.f = f  # clean again
    s.step(1)
    s.sync()
    ch = s.chains()["val"].copy()
    assert len(ch) > 0
    ch[0] = np.inf
    with pytest.raises(_lib.VlsError) as e:
        s.set_chain_values(ch)
    assert e.value.code == _lib.VLS_ENAN


def test_bad_inputs_report_errors():
    from vlasolve_b200 import _lib
    g, cfg = load_golden("udf_tiny")
    with pytest.raises(_lib.VlsError) as e:
        solver(cfg, Pres=1)
    assert e.value.code == _lib.VLS_EINVAL
    s = solver(cfg)
    with pytest.raises(_lib.VlsError):
        s.load_snapshot("/nonexistent/file.ND")


def test_queued_mass_reads_match_the_waiting_ones():
    """vls_last_mass_async: the mass of every step queued into a page-locked
    host array equals vls_last_mass after the same step of an identical
    handle."""
    import torch
    g, cfg = load_golden("udf_tiny")
    a, b = solver(cfg), solver(cfg)
    want = []
    for _ in range(5):
        a.step(1)
        want.append(a.last_mass())
    got = torch.zeros(5, dtype=torch.float64).pin_memory().numpy()
    for i in range(5):
        b.step(1)
        b.last_mass_into(got, i)
    b.sync()
    np.testing.assert_array_equal(got, np.array(want))
    assert np.all(got > 0)
    with pytest.raises(IndexError):
        b.last_mass_into(got, 5)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["udf_tiny", "udf_rect_kbuf", "udf_nolink"])
def test_slice_batches_on_streams_are_bit_identical(name, prec):
    """Splitting the J slices into batches on several streams (each with its
    own scratch slot) changes no arithmetic: the grid after several steps is
    bit-identical to the single-batch run."""
    from vlasolve_b200 import VlasovSolver21Spline
    g, cfg = load_golden(name)
    a = solver(cfg, prec)
    b = VlasovSolver21Spline(cfg, precision=prec, layout={"slices_per_batch": 3, "streams": 2})
    assert b.layout()["slices_per_batch"] == 3 and b.layout()["streams"] == 2
    a.step(4)
    b.step(4)
    np.testing.assert_array_equal(a.f, b.f)
    np.testing.assert_array_equal(a.chains()["val"], b.chains()["val"])


@pytest.mark.parametrize("prec,drift", [("fp64", "window"), ("fp32", "window"),
                                        ("fp32", "strip2"), ("fp32", "strip1")])
def test_drift_wait_timeout_reports_and_falls_back(prec, drift):
    """drift_wait_spins < 0: every bounded wait of the drift for its staged
    coefficients gives up at once (the copies still land; the block's last
    wait, before its shared memory is released, keeps the full limit).  The
    step reports it (vls_sync returns VLS_ECUDA, naming the drift) and its
    cells read C from global memory, so f still matches the reference."""
    from vlasolve_b200 import VlasovSolver21Spline, _lib
    g, cfg = load_golden("udf_rect_kbuf")
    s = VlasovSolver21Spline(cfg, precision=prec,
                             layout={"drift": drift, "drift_wait_spins": -1})
    lay = s.layout()
    assert lay["drift"] == drift and lay["drift_wait_spins"] == 0
    cur = 0
    for st in _saved_steps(g, "f_")[1:]:
        s.step(st - cur)
        cur = st
        with pytest.raises(_lib.VlsError) as e:
            s.sync()
        assert e.value.code == _lib.VLS_ECUDA and "drift" in str(e.value)
        ref = g["f_%d" % st]
        d = s.f - ref
        if prec == "fp64":
            assert np.abs(d).max() <= FP64_TOL * np.abs(ref).max()
        else:
            assert np.linalg.norm(d) / np.linalg.norm(ref) <= FP32_L2
    s.sync()  # the report cleared the flag; nothing ran since


def test_default_layouts_of_the_1025_vertex_grid():
    """The kernels the 1025 x 1025 lines take by default (the ones the
    pldf_1025 parity tests run): 23-row chunks along both directions, the
    one-block strip drift in FP32, the windowed drift in FP64."""
    g, cfg = load_golden("pldf_1025")
    a = solver(cfg, "fp32").layout()
    assert a["prefilter"] == "register" and a["u_chunk_rows"] == 23 and a["r_chunk_rows"] == 23
    assert a["drift"] == "strip1"
    b = solver(cfg, "fp64").layout()
    assert b["drift"] == "window" and b["u_chunk_rows"] == 23
    c = solver(load_golden("hernquist_cfg3")[1], "fp32").layout()
    assert c["drift"] == "strip2" and c["u_chunk_rows"] == 17 and c["r_chunk_rows"] == 19
