// vls_setup.cpp -- host set-up of the step (see vls_setup.h).
#include "vls_setup.h"

#include <cmath>
#include <cstdio>

namespace vls {

std::vector<double> gen_scale(double start, double stop, long N, int sct,
                              bool vertex) {
  std::vector<double> s;
  if (sct == VLS_SCALE_LINEAR) {
    const double dx = (stop - start) / (N);
    s.resize(N + 1);
    for (long i = 0; i < N + 1; i++) s[i] = start + dx * (double)i;
  } else if (sct == VLS_SCALE_LOG) {
    const double sg = (start < 0) ? -1 : 1;
    s = gen_scale(std::log(std::fabs(start)), std::log(std::fabs(stop)), N,
                  VLS_SCALE_LINEAR, true);
    for (long i = 0; i < N + 1; i++) s[i] = sg * std::exp(s[i]);
  } else {
    const int pp = sct;
    s = gen_scale(std::pow(start, 1. / pp), std::pow(stop, 1. / pp), N,
                  VLS_SCALE_LINEAR, true);
    for (long i = 0; i < N + 1; i++) s[i] = std::pow(s[i], (double)pp);
  }
  if (!vertex) {
    for (size_t i = 0; i + 1 < s.size(); i++) s[i] = (s[i] + s[i + 1]) * 0.5;
    s.resize(s.size() - 1);
  } else {
    s.front() = start;
    s.back() = stop;
  }
  return s;
}

double rescale(double x, int sct) {
  if (sct == VLS_SCALE_LOG) return std::log(x);
  if (sct == VLS_SCALE_LINEAR) return x;
  return std::pow(x, 1. / sct);
}

static bool valid_scale(int s) { return s >= 0 && s <= 2; }

bool make_coords(const vls_grid_desc &g, int kernelBufferSize, Coords &c,
                 std::string &err) {
  if (!valid_scale(g.Pscale) || !valid_scale(g.Uscale[0]) ||
      !valid_scale(g.Uscale[1])) {
    err = "invalid scale type (expected linear, logarithmic or quadratic)";
    return false;
  }
  if (g.Pres < 3 || g.Ures[0] < 3 || g.Ures[1] < 1) {
    err = "grid resolution too small (Pres >= 3, Ures >= 3, J cells >= 1)";
    return false;
  }
  if (g.Pres + 1 > 16383 || g.Ures[0] + 1 > 16383) {
    err = "grid resolution too large (at most 16383 vertices per direction)";
    return false;
  }
  if (!(g.Pmax > g.Pmin) || !(g.Umax[0] > g.Umin[0]) || !(g.Umax[1] > g.Umin[1])) {
    err = "grid ranges must satisfy min < max";
    return false;
  }
  if (g.Pscale == VLS_SCALE_LOG && !(g.Pmin * g.Pmax > 0)) {
    err = "cannot generate logscale from a 0-crossing range";
    return false;
  }
  if (g.Uscale[0] != VLS_SCALE_LINEAR) {
    err = "the v_r direction must use a linear scale (it spans negative values)";
    return false;
  }
  if (!(g.Pmin > 0)) {
    err = "grid.Pmin must be > 0 (spherical radius)";
    return false;
  }
  c.R = gen_scale(g.Pmin, g.Pmax, g.Pres, g.Pscale, true);
  c.U = gen_scale(g.Umin[0], g.Umax[0], g.Ures[0], g.Uscale[0], true);
  c.J = gen_scale(g.Umin[1], g.Umax[1], g.Ures[1], g.Uscale[1], false);
  c.JV = gen_scale(g.Umin[1], g.Umax[1], g.Ures[1], g.Uscale[1], true);
  c.nr = (int)c.R.size();
  c.nu = (int)c.U.size();
  c.nj = (int)c.J.size();
  c.rscale = g.Pscale;
  c.uscale = g.Uscale[0];
  // localSpline::init (localSpline.hxx:60-93): the spline re-generates the
  // vertex scale from its end points and rescales start/stop
  for (int d = 0; d < 2; d++) {
    const std::vector<double> &v = d == 0 ? c.R : c.U;
    const int sct = d == 0 ? c.rscale : c.uscale;
    std::vector<double> scl =
        gen_scale(v.front(), v.back(), (long)v.size() - 1, sct, true);
    const double start = rescale(scl.front(), sct);
    const double stop = rescale(scl.back(), sct);
    const double step = (stop - start) / ((double)scl.size() - 1);
    c.sstart[d] = start;
    c.sstep_inv[d] = 1. / step;
  }
  if (kernelBufferSize < 0 || kernelBufferSize >= c.nr) {
    err = "solver.kernelBufferSize must be in [0, N_r)";
    return false;
  }
  c.kernelRadius = c.R[kernelBufferSize];  // vlasovSolver21.hxx:436-438
  return true;
}

HostDirTables thomas_tables(int dim, double hi) {
  // localSpline::create_1D with NATURAL rows at both ends
  // (localSpline.hxx:976-981, :1019-1024, :1045-1059, :1104-1112, :1143-1153)
  HostDirTables t;
  t.M = dim + 2;
  const int M = t.M;
  t.hi2 = hi * hi;
  const double A00 = t.hi2, A01 = -2.0 * t.hi2, A02 = t.hi2;
  t.a01 = A01 / A00;
  t.a02 = A02 / A00;
  t.rp.assign(M, 0.0);
  t.q.assign(M, 0.0);
  {
    const double p1 = 4.0 / 6.0 - (1.0 / 6.0) * t.a01;
    const double q1 = (1.0 / 6.0 - (1.0 / 6.0) * t.a02) / p1;
    t.rp[1] = 1.0 / p1;
    t.q[1] = q1;
  }
  for (int k = 2; k <= M - 2; k++) {
    const double p = 4.0 / 6.0 - (1.0 / 6.0) * t.q[k - 1];
    t.q[k] = (1.0 / 6.0) / p;
    t.rp[k] = 1.0 / p;
  }
  t.L1 = -2.0 * t.hi2 - t.hi2 * t.q[M - 3];
  t.L2 = t.hi2 - t.L1 * t.q[M - 2];
  // the forward coefficients converge (geometrically, ratio 0.268) to the
  // fixed point of p = 4/6 - q/6, q = (1/6)/p; from row kc on they are
  // constant in the given precision, so the solve can drop the table there
  t.rp_inf = t.rp[M - 2];
  t.q_inf = t.q[M - 2];
  t.kc64 = M - 1;
  while (t.kc64 > 2 && t.rp[t.kc64 - 1] == t.rp_inf && t.q[t.kc64 - 1] == t.q_inf)
    t.kc64--;
  t.kc32 = M - 1;
  while (t.kc32 > 2 && (float)t.rp[t.kc32 - 1] == (float)t.rp_inf &&
         (float)t.q[t.kc32 - 1] == (float)t.q_inf)
    t.kc32--;
  return t;
}

// ---------------------------------------------------------------- profiles
// UniformDensitySphere (initGen_UniformDensitySphere.hxx:65-74, :158-173),
// PowerLawDensitySphere (initGen_PowerLawDensitySphere.hxx:63-82, :181-189),
// Plummer (initGen_Plummer.hxx:89-92, :126-131),
// Hernquist (initGen_Hernquist.hxx:48, :97-99, :133-155)
void Profile::setup(const vls_init_desc &desc, double G_) {
  d = desc;
  G = G_;
  if (d.type == VLS_INIT_UDF) {
    rho0 = (3 * d.M) / (4 * M_PI * std::pow(d.R0, 3));
    sig0 = std::sqrt((d.alpha) / (5 * d.R0));
    C1 = rho0 * std::pow(2 * M_PI * sig0 * sig0, -1.5);
    C2 = 2 * sig0 * sig0;
  } else if (d.type == VLS_INIT_PLDF) {
    if (!d.R0_given) d.R0 = 1. / d.eta;
    rho0 = ((3.0 - d.n) * d.M) / (4 * M_PI * std::pow(d.R0, 3.0 - d.n));
    sigO2 = (3.0 - d.n) / (5.0 - 2 * d.n) * (d.M * d.eta) /
            (d.R0 * (d.alpha * 0.5 + 1));
    sigR2 = sigO2 * 0.5 * d.alpha;
    C0 = rho0 / (std::sqrt(2 * sigR2 * M_PI * M_PI * M_PI) * sigO2);
    C1 = 1.0 / (2 * sigR2);
    C2 = 1.0 / (sigO2);
  } else if (d.type == VLS_INIT_HERNQUIST) {
    Vg = std::sqrt((G * d.M) / (d.R0));
  }
}

double Profile::value(double r, double u, double j) const {
  switch (d.type) {
    case VLS_INIT_UDF: {
      const double sm = 0.5 * (1. + std::erf((d.R0 - r) / d.smoothingRadius));
      double res = sm * C1 * std::exp(-(u * u + (j * j) / (r * r)) / C2);
      if (d.gap[1] > 0) {
        const double sm0 = 0.5 * (1. + std::erf((d.gap[0] - r) / 0.15));
        const double sm1 = 0.5 * (1. + std::erf(-(d.gap[1] - r) / 0.15));
        res *= (sm0 + sm1);
      }
      if (res < 1.E-200) res = 1.E-200;
      return res;
    }
    case VLS_INIT_PLDF: {
      const double sm = 0.5 * (1. + std::erf((d.R0 - r) / d.smoothingRadius));
      double res = sm * C0 * std::exp(-u * u * C1 - ((j * j) / (r * r)) * C2) *
                   std::pow(r, -d.n);
      if (res < 1.E-200) res = 1.E-200;
      return res;
    }
    case VLS_INIT_PLUMMER: {
      const double phi = -(G * d.M) / std::sqrt(r * r + d.R0 * d.R0);
      const double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      if (eps >= 0) return 0;
      return std::pow(-2. * eps, 3.5) * (3. / (M_PI * M_PI * M_PI * 7.));
    }
    case VLS_INIT_HERNQUIST: {
      const double phi = -(G * d.M) / (d.R0 + r);
      double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      if (d.Ra > 0) eps = eps + (j * j) / (2 * d.Ra * d.Ra);
      if (eps >= 0) return 0;
      const double q = std::sqrt(-(d.R0) / (G * d.M) * eps);
      const double q2 = q * q;
      double A1 = (d.M) / (8. * std::sqrt(2.) * std::pow(M_PI * d.R0 * Vg, 3.)) *
                  std::pow(1. - q2, -2.5);
      double A2 = 3 * std::asin(q) + q * std::sqrt(1. - q2) * (1. - 2 * q2) *
                                         (8 * q2 * q2 - 8 * q2 - 3);
      double result = A1 * A2;
      if (d.Ra > 0) {
        A1 = (d.M) / (std::sqrt(2.) * std::pow(M_PI * d.R0 * Vg, 3)) *
             std::pow(d.R0 / d.Ra, 2);
        A2 = q * (1. - 2 * q2);
        result += A1 * A2;
      }
      return result;
    }
  }
  return 0;
}

// --------------------------------------------------------------- drifts
void advance_particle_drift(double R, double U, double J, double dt, double R0,
                            double *outR, double *outU, bool *halted) {
  if (halted) *halted = false;
  double H0 = 0.5 * (U * U + (J * J) / (R * R));
  double sgn = (U <= 0) ? -1 : 1;
  double deltaT = dt;
  double newR = R, newU = U, tlim, tR0;
  if (sgn < 0) {
    tlim = 10 * dt;
    tR0 = 10 * dt;
  } else {
    tlim = std::sqrt(2 * R * R * H0 - J * J) / (2 * H0);
    if (R0 > 0) {
      const double A = 2 * H0;
      const double B = -2 * sgn * std::sqrt(2 * R * R * H0 - J * J);
      const double C = (R * R - R0 * R0);
      const double D = B * B - 4 * A * C;
      if (D < 0)
        tR0 = 10 * dt;
      else
        tR0 = (-B - std::sqrt(D)) / (2 * A);
      if (tR0 < 0) {
        tR0 = (-B + std::sqrt(D)) / (2 * A);
        if (tR0 < 0) tR0 = 10 * dt;
      }
    } else {
      tR0 = 10 * dt;
    }
  }
  if ((tR0 < deltaT) && (tR0 < tlim)) {
    newR = std::sqrt(std::pow(std::fabs(newR * newU) - 2 * sgn * H0 * tR0, 2) +
                     J * J) *
           std::pow(2 * H0, -0.5);
    newU = (2 * H0 - (J * J) / (newR * newR));
    newU = -std::sqrt(newU);
    sgn = -1;
    H0 = 0.5 * (newU * newU + (J * J) / (newR * newR));
    deltaT -= tR0;
    tlim = 10 * dt;
    tR0 = 10 * dt;
  }
  if (tlim < deltaT) {
    newR = std::sqrt(std::pow(std::fabs(newR * newU) - 2 * sgn * H0 * tlim, 2) +
                     J * J) *
           std::pow(2 * H0, -0.5);
    newU = 0;
    H0 = 0.5 * (J * J) / (newR * newR);
    sgn = -1;
    deltaT -= tlim;
    tR0 -= tlim;
    tlim = 10 * dt;
    // the reference terminates the process here when tR0 < deltaT
    // (vlasovSolver21.hxx:389-391): a particle inside the reflection radius R0
    // (reflective kernel with kernelBufferSize > 0) whose backward orbit
    // reaches R0 after its pericentre.  The caller turns that into an error.
    if (tR0 < deltaT && halted) *halted = true;
  }
  newR = std::sqrt(std::pow(std::fabs(newR * newU) - 2 * sgn * H0 * deltaT, 2) +
                   J * J) *
         std::pow(2 * H0, -0.5);
  newU = (2 * H0 - (J * J) / (newR * newR));
  if (newU <= 0)
    newU = 0;
  else
    newU = sgn * std::sqrt(newU);
  *outR = newR;
  *outU = newU;
}

// localSpline::pos2Coord (localSpline.hxx:352-358)
static void pos2coord(const Coords &c, double p, int dir, int32_t *I,
                      double *F) {
  double ip;
  p = rescale(p, dir == 0 ? c.rscale : c.uscale);
  double x = (p - c.sstart[dir]) * c.sstep_inv[dir];
  x = std::modf(x, &ip);
  *I = (ip > -2.0e9 && ip < 2.0e9) ? (int32_t)ip : INT32_MIN;
  *F = x;
}

void slice_footpoints(const Coords &c, int j, double dt_disp, bool reflective,
                      SliceFootpoints &fp) {
  // generateDisplacement (vlasovSolver21.hxx:102-143) then decomposeDisplacement
  // (vlasovSolver21_spline.hxx:76-100) for the cells of slice j
  const double dth = 0.5 * dt_disp;
  const double R0 = reflective ? c.kernelRadius : -1;
  const size_t n = (size_t)c.nr * c.nu;
  fp.rI.resize(n);
  fp.uI.resize(n);
  fp.rF.resize(n);
  fp.uF.resize(n);
  fp.driftR.resize(n);
  fp.driftU.resize(n);
  fp.out.resize(n);
  fp.halted = -1;
  const double J = c.J[j];
  for (int u = 0; u < c.nu; u++)
    for (int r = 0; r < c.nr; r++) {
      const size_t i = (size_t)u * c.nr + r;
      double dR, dU;
      bool halted = false;
      advance_particle_drift(c.R[r], c.U[u], J, dth, R0, &dR, &dU, &halted);
      if (halted && fp.halted < 0) fp.halted = (int64_t)i;
      fp.driftR[i] = dR;
      fp.driftU[i] = dU;
      fp.out[i] = ((dR >= c.R.back()) || (dR <= c.R.front()) ||
                   (dU >= c.U.back()) || (dU <= c.U.front()))
                      ? 1
                      : 0;
      pos2coord(c, dR, 0, &fp.rI[i], &fp.rF[i]);
      pos2coord(c, dU, 1, &fp.uI[i], &fp.uF[i]);
    }
}

void slice_chains(const Coords &c, int j, double dt_chain,
                  const SliceFootpoints &fp, SliceChains &ch) {
  // vlasovSolver21::setupBoundaryConditions (vlasovSolver21.hxx:281-322)
  const double dth = 0.5 * dt_chain;
  const double J = c.J[j];
  ch.cell.clear();
  ch.len.clear();
  ch.R.clear();
  ch.U.clear();
  for (int u = 0; u < c.nu; u++)
    for (int r = 0; r < c.nr; r++) {
      const size_t i = (size_t)u * c.nr + r;
      if (!(fp.driftR[i] < c.kernelRadius)) continue;
      double deltaT = dth, nR, nU;
      int32_t L = 0;
      advance_particle_drift(c.R[r], c.U[u], J, deltaT, -1, &nR, &nU);
      while (nR < c.kernelRadius) {
        ch.R.push_back(nR);
        ch.U.push_back(nU);
        L++;
        deltaT += dth;
        advance_particle_drift(c.R[r], c.U[u], J, deltaT, -1, &nR, &nU);
      }
      ch.R.push_back(nR);
      ch.U.push_back(nU);
      L++;
      ch.cell.push_back(((int64_t)j * c.nu + u) * c.nr + r);
      ch.len.push_back(L);
    }
}

}  // namespace vls
