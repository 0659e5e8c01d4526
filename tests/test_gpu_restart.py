"""Restart files: the reference's .vls files load into the solver and
continue as the reference does; the files this solver writes are the
reference's byte for byte; FP32 round trips."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

STEP2 = os.path.join(GOLDEN, "udf_tiny_restart_step2.vls")
STEP3 = os.path.join(GOLDEN, "udf_tiny_final_step3.vls")
FP64_TOL = 1e-12


def read_vls(path):
    """Grid and chain values of a .vls file (layout of vlasovSolver::write)."""
    b = open(path, "rb").read()
    o = 4
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n + 4 * 8 + 4 + 3 * 8 + 2 * 8 + 8 + 4
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n + 4 + 12 + 24
    param = 6 * 8 + 12 * 4 + 4 + 4 + 8 + 4 * 3 + 8 + 2048 - 4 * 6 - 8
    o += param
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n + param
    dims = (8, 17, 17)
    f = np.frombuffer(b, "<f8", count=int(np.prod(dims)), offset=o).reshape(dims)
    o += f.nbytes
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n + 3 * 2048
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n + 4 + 8 + 4 + 2048
    n = struct.unpack_from("<i", b, o)[0]
    o += 4 + n
    ns = struct.unpack_from("<q", b, o)[0]
    o += 8
    vals = []
    for _ in range(ns):
        cnt = struct.unpack_from("<q", b, o)[0]
        o += 8
        for _ in range(cnt):
            key, L = struct.unpack_from("<qq", b, o)
            o += 16
            for _ in range(L):
                R, U, nv = struct.unpack_from("<ddi", b, o)
                o += 20
                vals.append(struct.unpack_from("<d", b, o)[0])
                o += 8
    return f, np.array(vals)


def solver(precision="fp64"):
    from vlasolve_b200 import VlasovSolver21Spline
    g, cfg = load_golden("udf_tiny")
    return VlasovSolver21Spline(dict(cfg, Tmax=0.0125), precision=precision), g


def test_reference_restart_loads_bit_exact():
    s, g = solver()
    s.read_restart(STEP2)
    f, ch = read_vls(STEP2)
    np.testing.assert_array_equal(s.f, f)
    np.testing.assert_array_equal(s.f, g["f_2"])
    np.testing.assert_array_equal(s.chains()["val"], ch)
    assert s.time == 0.01 and s.stepCount == 2


def test_run_continues_from_reference_restart():
    s, _ = solver()
    s.read_restart(STEP2)
    s.step(1)
    f3, ch3 = read_vls(STEP3)
    scale = np.max(np.abs(f3))
    assert np.max(np.abs(s.f - f3)) <= FP64_TOL * scale
    assert np.max(np.abs(s.chains()["val"] - ch3)) <= FP64_TOL * scale


def test_written_restart_is_the_reference_file_byte_for_byte(tmp_path):
    s, _ = solver()
    s.read_restart(STEP3)
    out = str(tmp_path / "ours.vls")
    s.write_restart(out, snapshot_every=-1, restart_every=2, stats_every=-1)
    assert open(out, "rb").read() == open(STEP3, "rb").read()


def test_fp32_round_trip(tmp_path):
    s, _ = solver("fp32")
    s.step(3)
    out = str(tmp_path / "fp32.vls")
    s.write_restart(out)
    t, _ = solver("fp32")
    t.read_restart(out)
    np.testing.assert_array_equal(t.f, s.f)
    np.testing.assert_array_equal(t.chains()["val"], s.chains()["val"])
    assert (t.time, t.stepCount) == (s.time, s.stepCount)
    s.step(2)
    t.step(2)
    np.testing.assert_array_equal(t.f, s.f)


def test_restart_into_a_different_grid_is_rejected():
    from vlasolve_b200 import VlasovSolver21Spline
    from vlasolve_b200._lib import VlsError
    _, cfg = load_golden("udf_tiny")
    s = VlasovSolver21Spline(dict(cfg, Pres=20))
    with pytest.raises(VlsError):
        s.read_restart(STEP2)
    s2 = VlasovSolver21Spline(dict(cfg, dt=0.004))
    with pytest.raises(VlsError):
        s2.read_restart(STEP2)
