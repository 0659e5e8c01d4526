"""The command-line driver (vlasolve_b200/vlasolve_b200), given the reference's
own command line for a golden case, writes statistics.txt rows equal to the
reference's and the snapshot files its run loop writes."""
import os
import subprocess

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["udf_tiny", "hernquist_small", "pldf_small"])
def test_driver_statistics_match_reference(name, tmp_path):
    from vlasolve_b200.build import DRIVER, build
    build()
    g, _ = load_golden(name)
    ref = g["stats"]
    n = len(ref)
    dt = float(g["dt"])
    args = [str(a) for a in g["args"]] + [
        "-solver.dt", repr(dt), "-solver.Tmax", repr(dt * (n - 0.5)),
        "-solver.statsEvery", "1", "-solver.snapshotEvery", "2"]
    r = subprocess.run([DRIVER] + args, cwd=tmp_path, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert "Computed %d timesteps" % n in r.stdout
    rows = np.loadtxt(tmp_path / "statistics.txt", comments="#", ndmin=2)
    assert rows.shape == (n, 9)
    np.testing.assert_array_equal(rows[:, 1], ref[:, 1])
    np.testing.assert_allclose(rows[:, 0], ref[:, 0], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(rows[:, 2:], ref[:, 2:], rtol=2e-9, atol=1e-14)
    snaps = sorted(f for f in os.listdir(tmp_path) if f.startswith("snapshot_"))
    assert snaps and snaps[0] == "snapshot_0.0000.ND"


def test_driver_reload_continues_reference_restart(tmp_path):
    """-reload of the reference's step-2 restart file runs to its Tmax and
    writes final_0.0150.vls matching the reference's final dump."""
    from conftest import GOLDEN
    from test_gpu_restart import read_vls
    from vlasolve_b200.build import DRIVER, build
    build()
    stem = os.path.join(GOLDEN, "udf_tiny_restart_step2")
    r = subprocess.run([DRIVER, "-reload", stem], cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "Reloaded" in r.stdout
    ours = tmp_path / "final_0.0150.vls"
    assert ours.exists()
    f, ch = read_vls(str(ours))
    f3, ch3 = read_vls(os.path.join(GOLDEN, "udf_tiny_final_step3.vls"))
    scale = np.max(np.abs(f3))
    assert np.max(np.abs(f - f3)) <= 1e-12 * scale
    assert np.max(np.abs(ch - ch3)) <= 1e-12 * scale
