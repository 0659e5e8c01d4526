"""Pins the CPU oracle (oracle/vls_oracle.c) to the reference binary's own
outputs: every golden vector under tests/golden/ was produced by the
reference (tests/golden/make_golden.py).  The oracle must reproduce them
bit for bit: f at every saved step, the delayed-kernel chains, and the
statistics rows (which the reference prints with 10 significant digits)."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from oracle.vls_oracle import Oracle

SMALL = golden_cases(full_only=True)
LARGE = [c for c in golden_cases(full_only=False) if c != "hernquist_cfg3"]


def _stats_row(o, t, step):
    s = o.stats()
    return np.array([t, step, s["Mass"], s["E"], s["Ek"], s["Ep"], s["S"], s["L1"],
                     s["L2"]])


def _check_stats(row, ref):
    # the reference prints %10.10g; the oracle's values, printed the same way,
    # must give the same digits
    for k in range(1, 9):
        assert "%.10g" % row[k] == "%.10g" % ref[k], (k, row[k], ref[k])


@pytest.mark.parametrize("name", SMALL)
def test_oracle_bitexact_small(name):
    g, cfg = load_golden(name)
    o = Oracle(cfg)
    assert o.shape == tuple(g["shape"])
    ch = o.chains()
    if "chain0_cell" in g.files:
        np.testing.assert_array_equal(ch["cell"], g["chain0_cell"])
        np.testing.assert_array_equal(ch["len"], g["chain0_len"])
        np.testing.assert_array_equal(ch["R"], g["chain0_R"])
        np.testing.assert_array_equal(ch["U"], g["chain0_U"])
        np.testing.assert_array_equal(ch["val"], g["chain0_val"])
    else:
        assert len(ch["cell"]) == 0
    steps = sorted(int(k[2:]) for k in g.files if k.startswith("f_"))
    stats = g["stats"]
    cur = 0
    for s in steps:
        # stats rows are written before each step
        while cur < s:
            _check_stats(_stats_row(o, cur * cfg["dt"], cur), stats[cur])
            o.step(1)
            cur += 1
        np.testing.assert_array_equal(o.f, g["f_%d" % s], err_msg=f"{name} step {s}")
    if "chainN_val" in g.files:
        chN = o.chains()
        # the reference writes chain values front first after its rolls; the
        # oracle rotates in place, so the logical order is the array order
        np.testing.assert_array_equal(chN["cell"], g["chainN_cell"])
        vals = []
        for k in range(len(chN["cell"])):
            s0, L = chN["start"][k], chN["len"][k]
            vals.append(chN["val"][s0:s0 + L])
        np.testing.assert_array_equal(np.concatenate(vals) if vals else np.empty(0),
                                      g["chainN_val"])


@pytest.mark.parametrize("name", LARGE)
def test_oracle_bitexact_full_config_sampled(name):
    g, cfg = load_golden(name)
    o = Oracle(cfg)
    assert o.shape == tuple(g["shape"])
    idx = g["sample_idx"]
    ch = o.chains()
    np.testing.assert_array_equal(ch["cell"], g["chain0_cell"])
    np.testing.assert_array_equal(ch["len"], g["chain0_len"])
    n = min(512, len(ch["val"]))
    np.testing.assert_array_equal(ch["val"][:n], g["chain0_val_head"][:n])
    steps = sorted(int(k[3:]) for k in g.files if k.startswith("fs_"))
    cur = 0
    for s in steps:
        o.step(s - cur)
        cur = s
        f = o.f
        np.testing.assert_array_equal(f.ravel()[idx], g["fs_%d" % s])
        np.testing.assert_allclose(f.reshape(f.shape[0], -1).sum(axis=1),
                                   g["slicesum_%d" % s], rtol=1e-13, atol=0)


@pytest.mark.slow
def test_oracle_bitexact_hernquist_cfg3():
    test_oracle_bitexact_full_config_sampled("hernquist_cfg3")


def test_planted_error_is_caught():
    """A mistake planted in the oracle's input must show up against the
    golden vector (the comparison is not vacuous)."""
    g, cfg = load_golden("udf_tiny")
    o = Oracle(cfg)
    f = o.f
    k = np.unravel_index(np.argmax(f), f.shape)
    f[k] *= 1.0 + 4e-16
    o.f = f
    o.step(1)
    assert not np.array_equal(o.f, g["f_1"])


def test_oracle_halts_where_the_reference_terminates():
    """With the reflective kernel and kernelBufferSize > 0 the cells inside the
    reflection radius reach the branch of advanceParticleDrift where the
    reference prints and exits (vlasovSolver21.hxx:389-391; its run of this
    set-up ends there).  The oracle refuses the set-up the same way."""
    from oracle.vls_oracle import ReferenceHalt
    g, cfg = load_golden("udf_reflect")
    cfg = dict(cfg, kernelBufferSize=2)
    with pytest.raises(ReferenceHalt):
        Oracle(cfg)
