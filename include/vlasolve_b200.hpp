// vlasolve_b200.hpp -- C++ adapter over the C-ABI of vlasolve_b200.h that
// keeps the surface of the reference's solver classes for the spherical path:
// vlasovSolver (vlasovSolver.hxx:13-317), vlasovSolver21
// (vlasovSolver21.hxx:19-783) and vlasovSolver21_spline
// (vlasovSolver21_spline.hxx:16-943): construct from grid/solver/init
// parameters, makeOneStep(t), statistics(), snapshot(), moments and the
// coordinate accessors.  Header-only; link with libvlasolve_b200.so.
//
// Errors become vls::error exceptions carrying the VLS_* status (the
// reference prints and exits instead).
#ifndef VLASOLVE_B200_HPP
#define VLASOLVE_B200_HPP

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vlasolve_b200.h"

namespace vls {

class error : public std::runtime_error {
 public:
  error(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const vls_handle *h) {
  if (rc != VLS_OK) throw error(rc, vls_last_error(h));
}

// Parameter blocks with the reference's defaults for the UDF profile
// (initGen_UniformDensitySphere.hxx:82-112); fill them from the -group.param
// options as the reference's gridHandler / vlasovSolver::init do.
inline vls_grid_desc default_grid() {
  vls_grid_desc g{};
  g.Pmin = 0.01;
  g.Pmax = 25;
  g.Pres = 200;
  g.Pscale = VLS_SCALE_LOG;
  g.Umin[0] = -2.0;
  g.Umin[1] = 0.0;
  g.Umax[0] = 2.0;
  g.Umax[1] = 1.6;
  g.Ures[0] = 200;
  g.Ures[1] = 200;
  g.Uscale[0] = VLS_SCALE_LINEAR;
  g.Uscale[1] = VLS_SCALE_QUADRATIC;
  return g;
}

inline vls_solver_desc default_solver() {
  vls_solver_desc s{};
  s.G = 1;
  s.T0 = 0;
  s.Tmax = 60;
  s.dt = 0.005;
  s.noLinking = 0;
  s.kernelType = VLS_KERNEL_DELAYED;
  s.kernelBufferSize = 0;
  s.precision = VLS_FP64;
  s.device = 0;
  return s;
}

inline vls_init_desc default_init() {
  vls_init_desc i{};
  i.type = VLS_INIT_UDF;
  i.M = 1;
  i.R0 = 2;
  i.alpha = 0.5;
  i.smoothingRadius = 0.5;
  i.eta = 0.1;
  i.n = 1;
  i.Ra = -1;
  i.R0_given = 1;
  return i;
}

// The spherical split semi-Lagrangian solver on one GPU.
class vlasovSolver21_spline {
 public:
  // init == nullptr leaves the grid unset (for readRestart)
  vlasovSolver21_spline(const vls_grid_desc &g, const vls_solver_desc &s,
                        const vls_init_desc *init)
      : solver_(s) {
    check(vls_create(&g, &s, &h_), nullptr);
    try {
      if (init) check(vls_init_profile(h_, init, &mass_before_), h_);
      int64_t nr, nu, nj;
      check(vls_dims(h_, &nr, &nu, &nj), h_);
      nr_ = nr;
      nu_ = nu;
      nj_ = nj;
    } catch (...) {
      vls_destroy(h_);
      throw;
    }
  }
  ~vlasovSolver21_spline() { vls_destroy(h_); }
  vlasovSolver21_spline(const vls_grid_desc &g, const vls_solver_desc &s,
                        const vls_init_desc &init)
      : vlasovSolver21_spline(g, s, &init) {}
  vlasovSolver21_spline(const vlasovSolver21_spline &) = delete;
  vlasovSolver21_spline &operator=(const vlasovSolver21_spline &) = delete;

  // vlasovSolver21_spline::makeOneStep (vlasovSolver21_spline.hxx:680-801)
  void makeOneStep(double /*t*/) { check(vls_step(h_, 1), h_); }
  void steps(int n) { check(vls_step(h_, n), h_); }
  void sync() { check(vls_sync(h_), h_); }

  // vlasovSolver::run (vlasovSolver.hxx:134-190): restart files every
  // restartEvery steps (restart_%.4f.vls), statistics every statsEvery steps
  // (row appended to `stats`), snapshots every snapshotEvery steps
  // (snapshot_%4.4f.ND); afterRunning (:235-246): a last snapshot when the
  // step count is a multiple of snapshotEvery, and final_%.4f.vls
  void run(long statsEvery, long snapshotEvery, const char *stats = "statistics.txt",
           long restartEvery = -1, bool finalDump = false) {
    auto timer = [](long every, long n) { return every >= 0 && (n % every) == 0; };
    auto checkTime = [&]() {
      double t;
      int64_t st;
      vls_get_time(h_, &t, &st);
      return solver_.Tmax <= 0 ||
             (t < solver_.Tmax && std::abs(t - solver_.Tmax) > solver_.dt / 100);
    };
    if (!checkTime()) return;
    char buf[64];
    do {
      double t;
      int64_t n;
      vls_get_time(h_, &t, &n);
      if (timer(restartEvery, n)) {
        std::snprintf(buf, sizeof(buf), "restart_%.4f.vls", t);
        writeRestart(buf, snapshotEvery, restartEvery, statsEvery);
      }
      if (timer(snapshotEvery, n)) snapshot();
      if (timer(statsEvery, n)) statistics(n == 0, stats);
      makeOneStep(t);
    } while (checkTime());
    if (finalDump) {
      double t;
      int64_t n;
      vls_get_time(h_, &t, &n);
      if (timer(snapshotEvery, n)) snapshot();
      std::snprintf(buf, sizeof(buf), "final_%.4f.vls", t);
      writeRestart(buf, snapshotEvery, restartEvery, statsEvery);
    }
  }

  // vlasovSolver::write(fname) (vlasovSolver.hxx:248-269): the .vls file
  void writeRestart(const char *name, long snapshotEvery, long restartEvery, long statsEvery) {
    check(vls_write_restart(h_, name, snapshotEvery, restartEvery, statsEvery), h_);
  }
  // vlasovSolver::init(params, fname) (vlasovSolver.hxx:104-131): the state of
  // a .vls file, into a solver created with the file's parameters
  void readRestart(const char *name) { check(vls_read_restart(h_, name), h_); }

  // vlasovSolver21::statistics (vlasovSolver21.hxx:644-690)
  vls_stats_out statistics(bool reset = false, const char *fname = "statistics.txt") {
    vls_stats_out o;
    check(vls_stats(h_, &o), h_);
    if (fname) {
      FILE *f = std::fopen(fname, reset ? "w" : "a");
      if (!f) throw error(VLS_EIO, std::string("cannot open ") + fname);
      if (reset) std::fprintf(f, "# Time Step Mass E Ek Ep S L1 L2\n");
      std::fprintf(f, "%.10g %ld %10.10g %10.10g %10.10g %10.10g %10.10g %10.10g %10.10g\n",
                   o.time, (long)o.step, o.Mass, o.E, o.Ek, o.Ep, o.S, o.L1, o.L2);
      std::fclose(f);
    }
    return o;
  }

  // vlasovSolver21::snapshot (vlasovSolver21.hxx:585-598)
  std::string snapshot(const char *name = nullptr) {
    char buf[1024];
    double t;
    int64_t n;
    vls_get_time(h_, &t, &n);
    if (!name) {
      std::snprintf(buf, sizeof(buf), "snapshot_%4.4f.ND", t);
      name = buf;
    }
    check(vls_write_ndfield(h_, name), h_);
    return name;
  }

  // quadrature21::integrate1D_acc (vlasovSolver21_spline.hxx:736)
  double enclosedMass(std::vector<double> &bins, std::vector<double> &Mr) {
    bins.resize(nr_);
    Mr.resize(nr_);
    double tot = 0;
    check(vls_moments(h_, bins.data(), Mr.data(), &tot), h_);
    return tot;
  }

  // gridBase::getDataPtr equivalents (host copies, [j][u][r])
  std::vector<double> data() {
    std::vector<double> f(nr_ * nu_ * nj_);
    check(vls_get_f(h_, f.data(), f.size()), h_);
    return f;
  }
  void setData(const std::vector<double> &f) { check(vls_set_f(h_, f.data(), f.size()), h_); }

  // grid_21.hxx:150-158
  std::vector<double> getValCoord21_R() const { return coord(0); }
  std::vector<double> getValCoord21_U() const { return coord(1); }
  std::vector<double> getValCoord21_J() const { return coord(2); }

  // Adjoint of `nsteps` linked steps (no counterpart in the reference):
  // adjointForward runs them keeping a checkpoint every `checkpointEvery`
  // steps; adjointBackward takes dL/d(final radial bins) (N_r values) and
  // returns dL/d(initial grid) ([j][u][r]) and, if asked, dL/d(initial chain
  // values); the handle holds the final state again afterwards
  void adjointForward(int nsteps, int checkpointEvery) {
    check(vls_adjoint_forward(h_, nsteps, checkpointEvery), h_);
  }
  void adjointBackward(const std::vector<double> &dbins, std::vector<double> &df0,
                       std::vector<double> *dchain0 = nullptr) {
    df0.resize(nr_ * nu_ * nj_);
    int64_t nc = 0, ne = 0;
    check(vls_get_chains(h_, &nc, &ne, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr),
          h_);
    if (dchain0) dchain0->resize((size_t)ne);
    check(vls_adjoint_backward(h_, dbins.data(), (int64_t)dbins.size(), df0.data(), df0.size(),
                               dchain0 ? dchain0->data() : nullptr, dchain0 ? ne : 0),
          h_);
  }
  // second checkpoint level inside a segment (0: chosen from free memory)
  void adjointSetInner(int innerEvery) { check(vls_adjoint_set_inner(h_, innerEvery), h_); }
  // for d/d(init.* parameter) by central differences: <dL/df0, f(plus) -
  // f(minus)> + <dL/dc0, c(plus) - c(minus)> for the last adjointBackward,
  // the two initial states made and contracted on the device
  double adjointInitDot(const vls_init_desc &plus, const vls_init_desc &minus) {
    double dg = 0, dc = 0;
    check(vls_adjoint_init_dot(h_, &plus, &minus, &dg, &dc), h_);
    return dg + dc;
  }
  // the mass of the most recent step, copied to *pinnedDst without waiting
  // (valid after the next synchronising call)
  void lastMassAsync(double *pinnedDst) { check(vls_last_mass_async(h_, pinnedDst), h_); }
  // device memory the handle holds (also its peak)
  size_t deviceBytes() {
    size_t b = 0;
    check(vls_device_bytes(h_, &b), h_);
    return b;
  }

  double massBeforeRenormalisation() const { return mass_before_; }
  size_t nr() const { return nr_; }
  size_t nu() const { return nu_; }
  size_t nj() const { return nj_; }
  vls_handle *handle() { return h_; }

 private:
  std::vector<double> coord(int which) const {
    std::vector<double> R(nr_), U(nu_), J(nj_), JV(nj_ + 1);
    check(vls_coords(h_, R.data(), U.data(), J.data(), JV.data()), h_);
    return which == 0 ? R : which == 1 ? U : J;
  }
  vls_handle *h_ = nullptr;
  vls_solver_desc solver_;
  double mass_before_ = 0;
  size_t nr_ = 0, nu_ = 0, nj_ = 0;
};

// localSpline<2, double> (localSpline.hxx:60-503) over a vls_spline2d of
// one or more slices: init(initT), assign(data), build(), evaluateC,
// evaluateNxPy, evaluate and pos2Coord with the reference's signatures (one
// point, slice 0), plus batched forms over arrays of points.
class localSpline2 {
 public:
  // localSpline::boundaryTypeV / initT (localSpline.hxx:34-46)
  struct initT {
    double start[2], stop[2];
    int N[2];
    int scaleType[2];  // VLS_SCALE_*
    int vlType[2];     // 1 VERTEX, 0 CELL
    int bCond[2][2];   // VLS_BC_NATURAL
  };
  localSpline2() = default;
  explicit localSpline2(const initT &ini, int64_t nslices = 1, int precision = VLS_FP64,
                        int device = 0) {
    init(ini, nslices, precision, device);
  }
  localSpline2(const localSpline2 &) = delete;
  localSpline2 &operator=(const localSpline2 &) = delete;
  ~localSpline2() { vls_spline2d_destroy(s_); }

  void init(const initT &ini, int64_t nslices = 1, int precision = VLS_FP64, int device = 0) {
    vls_spline2d_destroy(s_);
    s_ = nullptr;
    vls_spline2d_desc d{};
    for (int k = 0; k < 2; ++k) {
      d.start[k] = ini.start[k];
      d.stop[k] = ini.stop[k];
      d.N[k] = ini.N[k];
      d.scaleType[k] = ini.scaleType[k];
      d.vlType[k] = ini.vlType[k];
      d.bCond[k][0] = ini.bCond[k][0];
      d.bCond[k][1] = ini.bCond[k][1];
    }
    d.precision = precision;
    d.device = device;
    const int rc = vls_spline2d_create(&d, nslices, &s_);
    if (rc != VLS_OK) throw error(rc, vls_spline2d_last_error(nullptr));
    vls_spline2d_dims(s_, &dim_[0], &dim_[1], &ns_);
  }
  // values of every slice, [slice][dim1][dim0]
  void assign(const double *data) { ck(vls_spline2d_assign(s_, data, ns_)); }
  void build() { ck(vls_spline2d_build(s_)); }
  std::pair<int, double> pos2Coord(double p, int dir) const {
    int32_t I = 0;
    double F = 0;
    ck(vls_spline2d_pos2coord(s_, dir, 1, &p, &I, &F));
    return {I, F};
  }
  double evaluateC(int Nx, double x, int Ny, double y) {
    double v = 0;
    const int32_t nx = Nx, ny = Ny;
    ck(vls_spline2d_evaluate_c(s_, 1, nullptr, &nx, &x, &ny, &y, &v));
    return v;
  }
  double evaluateNxPy(int Nx, double yy) {
    double v = 0;
    const int32_t nx = Nx;
    ck(vls_spline2d_evaluate_nxpy(s_, 1, nullptr, &nx, &yy, &v));
    return v;
  }
  double evaluate(double xx, double yy) {
    double v = 0;
    ck(vls_spline2d_evaluate(s_, 1, nullptr, &xx, &yy, &v));
    return v;
  }
  // batched: n points on the given slices (slice may be null: slice 0)
  void evaluate(int64_t n, const int64_t *slice, const double *xx, const double *yy, double *v) {
    ck(vls_spline2d_evaluate(s_, n, slice, xx, yy, v));
  }
  void evaluateC(int64_t n, const int64_t *slice, const int32_t *Nx, const double *x,
                 const int32_t *Ny, const double *y, double *v) {
    ck(vls_spline2d_evaluate_c(s_, n, slice, Nx, x, Ny, y, v));
  }
  std::vector<double> coefficients(int64_t slice = 0) {
    std::vector<double> c((size_t)(dim_[0] + 2) * (dim_[1] + 2));
    ck(vls_spline2d_coefficients(s_, slice, c.data()));
    return c;
  }
  int dim(int k) const { return dim_[k]; }

 private:
  void ck(int rc) const {
    if (rc != VLS_OK) throw error(rc, vls_spline2d_last_error(s_));
  }
  vls_spline2d *s_ = nullptr;
  int32_t dim_[2] = {0, 0};
  int64_t ns_ = 0;
};

// interpolSpline<double> (interpol_spline.hxx:9-189): static createInit,
// create, evaluate (value; value and gradient; value, gradient and
// Hessian) and destroy, as the reference's einspline wrapper declares them.
struct interpolSpline {
  typedef vls_interp_init initT;
  typedef vls_interp interpT;
  static initT createInit(double xstart, double xstop, int Nx, double ystart, double ystop,
                          int Ny, int xbctL, int xbctR, int ybctL, int ybctR, int xscaleType,
                          int yscaleType, int vltype, bool useLog = false, double xbcvL = 0,
                          double xbcvR = 0, double ybcvL = 0, double ybcvR = 0) {
    initT g{};
    const int rc = vls_interp_create_init(xstart, xstop, Nx, ystart, ystop, Ny, xbctL, xbctR,
                                          ybctL, ybctR, xscaleType, yscaleType, vltype,
                                          useLog ? 1 : 0, xbcvL, xbcvR, ybcvL, ybcvR, &g);
    if (rc != VLS_OK) throw error(rc, vls_interp_last_error(nullptr));
    return g;
  }
  static interpT *create(initT &ini, const double *data, int device = 0) {
    interpT *s = nullptr;
    const int rc = vls_interp_create(&ini, data, device, &s);
    if (rc != VLS_OK) throw error(rc, vls_interp_last_error(nullptr));
    return s;
  }
  static void evaluate(interpT *s, double x, double y, double *v) { ck(s, x, y, v, 0, 0); }
  static void evaluate(interpT *s, double x, double y, double *v, double *g) {
    ck(s, x, y, v, g, 0);
  }
  static void evaluate(interpT *s, double x, double y, double *v, double *g, double *h) {
    ck(s, x, y, v, g, h);
  }
  static void destroy(interpT *s) { vls_interp_destroy(s); }

 private:
  static void ck(interpT *s, double x, double y, double *v, double *g, double *h) {
    const int rc = vls_interp_evaluate(s, 1, &x, &y, v, g, h);
    if (rc != VLS_OK) throw error(rc, vls_interp_last_error(s));
  }
};

}  // namespace vls

#endif
