// vls_setup.h -- host-side set-up of the step: coordinate tables, spline
// constants, Thomas tables, initial-condition profiles, drift footpoints and
// delayed-kernel chains.  All FP64, evaluated with the host libm in the
// reference's operation order, so that integer footpoint indices and the
// initial grid match the reference bit for bit.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vlasolve_b200.h"

namespace vls {

// scale::genScale (scale.hxx:114-151); vertex = true -> VERTEX, else CELL
std::vector<double> gen_scale(double start, double stop, long N, int sct,
                              bool vertex);
// scale::rescale (scale.hxx:175-189)
double rescale(double x, int sct);

struct Coords {
  int nr, nu, nj;
  std::vector<double> R, U, J, JV;  // R_Val, U_Val, J_Val (cell), J_V
  double sstart[2], sstep_inv[2];   // localSpline start/step_inv (r, u)
  int rscale, uscale;
  double kernelRadius;
};

bool make_coords(const vls_grid_desc &g, int kernelBufferSize, Coords &c,
                 std::string &err);

// Thomas tables of one direction (see DirTables in vls_internal.h)
struct HostDirTables {
  std::vector<double> rp, q;
  double a01, a02, hi2, L1, L2;
  int M;
  int kc64, kc32;  // first row of the constant-coefficient interior
  double rp_inf, q_inf;
};
HostDirTables thomas_tables(int dim, double hi);

// analytic distribution functions of the four profiles
struct Profile {
  vls_init_desc d;
  double G;
  double rho0, sig0, C0, C1, C2, sigR2, sigO2, Vg;
  void setup(const vls_init_desc &desc, double G_);
  double value(double r, double u, double j) const;
};

// vlasovSolver21::advanceParticleDrift (vlasovSolver21.hxx:328-408).
// *halted (may be NULL) is set where the reference terminates the process
// (:389-391, reachable with a reflection radius R0 > 0 only).
void advance_particle_drift(double R, double U, double J, double dt, double R0,
                            double *outR, double *outU, bool *halted = nullptr);

// footpoints of one J slice: integer/fraction pairs as decomposeDisplacement
// produces them, the outside flag, and driftR
struct SliceFootpoints {
  std::vector<int32_t> rI, uI;
  std::vector<double> rF, uF, driftR, driftU;
  std::vector<uint8_t> out;
  int64_t halted = -1;  // first cell (in the slice) where the reference halts, or -1
};
void slice_footpoints(const Coords &c, int j, double dt_disp, bool reflective,
                      SliceFootpoints &fp);

// chains of one J slice in the reference's build order (cell index order)
struct SliceChains {
  std::vector<int64_t> cell;
  std::vector<int32_t> len;
  std::vector<double> R, U;  // per element; the last of each chain is the tail
};
void slice_chains(const Coords &c, int j, double dt_chain,
                  const SliceFootpoints &fp, SliceChains &ch);

}  // namespace vls
