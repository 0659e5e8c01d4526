"""The header-only C++ adapter (include/vlasolve_b200.hpp): a small program
built against it runs the UDF profile, steps, and takes the adjoint of the
steps through the adapter's methods; its grid and gradients equal those of
the Python mirror of the same C-ABI calls."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

PROGRAM = r"""
#include "vlasolve_b200.hpp"
#include <cstdio>
#include <vector>

int main(int argc, char **argv) {
  vls_grid_desc g = vls::default_grid();
  g.Pres = 32;
  g.Ures[0] = 24;
  g.Ures[1] = 8;
  vls_solver_desc s = vls::default_solver();
  s.dt = 0.02;
  vls_init_desc init = vls::default_init();
  vls::vlasovSolver21_spline solver(g, s, init);
  solver.adjointForward(6, 4);  // two segments: 4 steps and 2 steps
  std::vector<double> f = solver.data();
  std::vector<double> dbins(solver.nr()), df0, dch;
  for (size_t r = 0; r < dbins.size(); ++r) dbins[r] = 0.1 * (double)r;
  solver.adjointSetInner(2);  // second checkpoint level inside each segment
  solver.adjointBackward(dbins, df0, &dch);
  FILE *o = std::fopen(argv[1], "wb");
  size_t n[3] = {f.size(), df0.size(), dch.size()};
  std::fwrite(n, sizeof(size_t), 3, o);
  std::fwrite(f.data(), sizeof(double), f.size(), o);
  std::fwrite(df0.data(), sizeof(double), df0.size(), o);
  std::fwrite(dch.data(), sizeof(double), dch.size(), o);
  std::fclose(o);
  std::printf("device bytes %zu\n", solver.deviceBytes());
  return 0;
}
"""


def test_cxx_adapter_adjoint_matches_python(tmp_path):
    from vlasolve_b200 import VlasovSolver21Spline
    from vlasolve_b200.build import HERE, build
    build()
    src = tmp_path / "adj.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "adj"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"),
                           str(src), "-L" + HERE, "-lvlasolve_b200",
                           "-Wl,-rpath," + HERE, "-o", str(exe)])
    out = tmp_path / "adj.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert int(r.stdout.split()[-1]) > 0
    raw = out.read_bytes()
    n = np.frombuffer(raw[:24], dtype=np.uint64)
    vals = np.frombuffer(raw[24:], dtype=np.float64)
    f_c = vals[:n[0]]
    df0_c = vals[n[0]:n[0] + n[1]]
    dch_c = vals[n[0] + n[1]:]

    s = VlasovSolver21Spline({"type": "UDF", "Pmin": 0.01, "Pmax": 25.0, "Pres": 32,
                              "Pscale": "logarithmic", "Umin": (-2.0, 0.0),
                              "Umax": (2.0, 1.6), "Ures": (24, 8),
                              "Uscale": ("linear", "quadratic"), "dt": 0.02})
    s.adjoint_forward(6, 4)
    np.testing.assert_array_equal(f_c, s.f.ravel())
    df0, dch = s.adjoint_backward(0.1 * np.arange(s.nr, dtype=np.float64))
    scale = np.max(np.abs(df0))
    np.testing.assert_allclose(df0_c, df0.ravel(), rtol=1e-12, atol=1e-14 * scale)
    assert dch_c.size == dch.size
    if dch.size:
        np.testing.assert_allclose(dch_c, dch, rtol=1e-12,
                                   atol=1e-14 * max(np.max(np.abs(dch)), 1e-300))
