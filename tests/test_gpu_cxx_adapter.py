"""The header-only C++ adapter (include/vlasolve_b200.hpp): a small program
built against it runs the UDF profile, steps, and takes the adjoint of the
steps through the adapter's methods; its grid, gradients and initial-state
contraction equal those of the Python mirror of the same C-ABI calls."""
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
  vls_init_desc plus = init, minus = init;
  plus.alpha = init.alpha * (1 + 1e-6);
  minus.alpha = init.alpha * (1 - 1e-6);
  const double idot = solver.adjointInitDot(plus, minus);
  FILE *o = std::fopen(argv[1], "wb");
  size_t n[3] = {f.size(), df0.size(), dch.size()};
  std::fwrite(n, sizeof(size_t), 3, o);
  std::fwrite(&idot, sizeof(double), 1, o);
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
    idot_c = float(np.frombuffer(raw[24:32], dtype=np.float64)[0])
    vals = np.frombuffer(raw[32:], dtype=np.float64)
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
    # the initial-state contraction through the adapter and through Python
    a = s.init_desc().alpha
    dg, dc = s.adjoint_init_dot({"alpha": a * (1 + 1e-6)}, {"alpha": a * (1 - 1e-6)})
    assert idot_c != 0.0
    np.testing.assert_allclose(idot_c, dg + dc, rtol=1e-12)


SPLINE_PROGRAM = r"""
#include "vlasolve_b200.hpp"
#include <cmath>
#include <cstdio>
#include <vector>

// localSpline<2>-style use: init, assign, build, then the reference's
// one-point calls; interpolSpline-style use: createInit, create, evaluate
int main(int argc, char **argv) {
  vls::localSpline2::initT ini{};
  ini.start[0] = 0.01; ini.stop[0] = 25.0; ini.N[0] = 40;
  ini.start[1] = -2.0; ini.stop[1] = 2.0; ini.N[1] = 32;
  ini.scaleType[0] = VLS_SCALE_LOG; ini.scaleType[1] = VLS_SCALE_LINEAR;
  ini.vlType[0] = ini.vlType[1] = 1;
  for (int k = 0; k < 2; ++k) ini.bCond[k][0] = ini.bCond[k][1] = VLS_BC_NATURAL;
  vls::localSpline2 sp(ini);
  std::vector<double> data((size_t)sp.dim(0) * sp.dim(1));
  for (int u = 0; u < sp.dim(1); ++u)
    for (int r = 0; r < sp.dim(0); ++r)
      data[(size_t)u * sp.dim(0) + r] = std::exp(-0.05 * r) * std::cos(0.1 * u) + 0.3;
  sp.assign(data.data());
  sp.build();
  FILE *o = std::fopen(argv[1], "wb");
  std::pair<int, double> c = sp.pos2Coord(3.7, 0);
  double out[6] = {sp.evaluateC(5, 0.25, 7, 0.75), sp.evaluateNxPy(9, 0.33),
                   sp.evaluate(3.7, -0.4), (double)c.first, c.second, 0};
  vls::interpolSpline::initT ii = vls::interpolSpline::createInit(
      0.01, 25.0, 40, -2.0, 2.0, 32, VLS_EBC_NATURAL, VLS_EBC_NATURAL, VLS_EBC_NATURAL,
      VLS_EBC_NATURAL, VLS_SCALE_LOG, VLS_SCALE_LINEAR, 1);
  vls::interpolSpline::interpT *is = vls::interpolSpline::create(ii, data.data());
  double v, g[2], h[4];
  vls::interpolSpline::evaluate(is, 3.7, -0.4, &v, g, h);
  vls::interpolSpline::destroy(is);
  out[5] = v;
  std::fwrite(out, sizeof(double), 6, o);
  std::fwrite(g, sizeof(double), 2, o);
  std::fwrite(h, sizeof(double), 4, o);
  std::fwrite(data.data(), sizeof(double), data.size(), o);
  std::fclose(o);
  return 0;
}
"""


def test_cxx_spline_adapters_match_python(tmp_path):
    from oracle import vls_oracle as vo
    from vlasolve_b200.build import HERE, build
    from vlasolve_b200.spline import InterpolSpline, LocalSpline2
    build()
    src = tmp_path / "spl.cpp"
    src.write_text(SPLINE_PROGRAM)
    exe = tmp_path / "spl"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I" + os.path.join(REPO, "include"),
                           str(src), "-L" + HERE, "-lvlasolve_b200",
                           "-Wl,-rpath," + HERE, "-o", str(exe)])
    out = tmp_path / "spl.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    vals = np.frombuffer(out.read_bytes(), dtype=np.float64)
    res, g, h, data = vals[:6], vals[6:8], vals[8:12], vals[12:].reshape(33, 41)
    sp = LocalSpline2((0.01, -2.0), (25.0, 2.0), (40, 32), scale=("logarithmic", "linear"))
    sp.assign(data)
    sp.build()
    coef = vo.prefilter2d(data, sp.step_inv[0], sp.step_inv[1])
    assert res[0] == pytest.approx(vo.evaluate_c(coef, [5], [0.25], [7], [0.75])[0], rel=1e-12)
    Ny, fy = sp.pos2Coord([0.33], 1)
    assert res[1] == pytest.approx(vo.evaluate_nxpy(coef, [9], Ny, fy)[0], rel=1e-12)
    assert res[2] == sp.evaluate([3.7], [-0.4])[0]
    I, F = sp.pos2Coord([3.7], 0)
    assert (res[3], res[4]) == (I[0], F[0])
    ini = InterpolSpline.createInit(0.01, 25.0, 40, -2.0, 2.0, 32, xscaleType="logarithmic")
    v, gg, hh = InterpolSpline.create(ini, data).evaluate([3.7], [-0.4], hess=True)
    assert res[5] == v[0]
    np.testing.assert_array_equal(g, gg[0])
    np.testing.assert_array_equal(h, hh[0])
