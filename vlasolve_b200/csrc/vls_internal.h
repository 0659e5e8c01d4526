// vls_internal.h -- device buffers of a handle and the kernel launchers.
//
// Device layout (HBM), one GPU holds everything:
//   f      [N_J][N_u][N_r]          T (float or double), r fastest
//   G      [slot][B][N_u+2][Pg]     T: u-direction spline coefficients of the
//                                     kicked f (rows 0 and N_u+1 are ghosts),
//                                     for a batch of B slices per ring slot;
//                                     Pg = N_r rounded up to 16 bytes
//   C      [slot][B][N_u+3][Pc]     T: 2D coefficients, Pc >= N_r+3; row N_u+2
//                                     and columns >= N_r+2 stay zero (reads
//                                     at index N exist for footpoints that
//                                     land on the last vertex with weight 0)
//   FP64: fp_idx [cells] int32      rI | uI<<16, -1 = outside, <= -2 = chain
//         fp_x, fp_y [cells] double fractional footpoint offsets
//   FP32: fp2 [cells] uint2         per direction index<<21 | round(frac*2^21);
//                                     0xFFFFFFFF = outside, 0xFFFFFFFE = chain
//                                     (second word = chain id)
//   the footpoint tables end with FOOT_PAD_ROWS zeroed rows of N_r cells and
//   32 more zeroed cells past the last slice, so that the strip drift
//   prefetches the next rows of a slice without clamping the row index
//   chains: ch_start/int64, ch_len/int32 per chain, ch_val/T per element
//           (ring buffer; logical front at (ndrift mod len)), tail footpoint
//   partial [N_J][N_r] double       per-slice radial moment partial sums
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda.h>
#include <cuda_runtime.h>

namespace vls {

// a bounded mbarrier wait gives up after ~2^20 polls (tens of milliseconds
// at most)
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 20;

// readable rows past the end of the footpoint tables (the strip drift reads
// at most 16 warps x 2 rows ahead; 32 cells more cover the lanes past N_r)
constexpr int FOOT_PAD_ROWS = 66;

// Thomas tables of one direction of the natural-BC cubic B-spline solve
// (localSpline.hxx:953-1182).  Row k of the padded line, M = dim + 2.
struct DirTables {
  const double *rp;  // 1/p_k (k = 1..M-2), device
  const double *q;   // normalised super-diagonal q_k (k = 0..M-1), device
  double a01, a02;   // normalised first row (-2, 1)
  double hi2, L1, L2;  // last-row constants
  int M;
  // from row kc on (up to M-2) rp_k and q_k equal rp_inf, q_inf when rounded
  // to the recursion's precision: kc64 for FP64, kc32 for FP32 recursions
  int kc64, kc32;
  double rp_inf, q_inf;
};

struct Geometry {
  int nr, nu, nj;
  int pc;  // row pitch of C
  int gp;  // row pitch of G (16-byte rows)
  // slices [j0, j0 + nb) are processed by this launch (grid.y = nb); the
  // scratch arrays G and C hold only those slices (local index j - j0)
  int j0, nb;
  const double *U;      // U_Val (nu)
  double u0, umax;      // U_Val.front(), U_Val.back()
  double su, hu;        // spline start / step_inv of u (rescaled, linear)
};

struct MomentTables {
  const double *bu;  // a_u + a_{u-1}, a_u = dU_u (0 for the last vertex)
  const double *wj;  // 8 pi^2 J_j dJ_j
  const double *dR4; // dR_r / 4 (0 for the last vertex)
  const double *Rcoef;  // G/(R_r^2) * dt
  const float *bu32;    // bu rounded to FP32 (the FP32 strip drift's products)
};

// Register-resident prefilter (vls_rc.cu): L rows of a line per thread,
// chunk layouts chosen per direction by rc_config.  RcDir is passed by value
// as a kernel parameter, so its tables are read as constant-bank operands.
template <typename R>
struct RcDir {
  R rp0[32], m0[32], q0[32];  // rp_k, -rp_k/6, q_k for rows k = 0..31
  R mpow[33], qpow[33];       // (-rp_inf/6)^i and (-q_inf)^i, i = 0..32
  R qfirst[32];               // prod_{k=i}^{L-1} (-q_{1+k}), i = 0..L-1 (first chunk)
  R rp_inf, m_inf, q_inf;
  R a01, a02, hi2, L1, L2;
  R inv_L2;                   // 1 / L2 (the last row without a division)
  int N, L, S;                // data rows, rows per chunk, chunks
};

// launchers (vls_kernels.cu); all asynchronous on `st`
// T: storage type of f and the coefficients; R: arithmetic of the recursions
template <typename T, typename R>
cudaError_t launch_ucol(bool kick, const T *f, T *G, const double *shift,
                        const Geometry &g, const DirTables &tu, cudaStream_t st);
template <typename T, typename R>
cudaError_t launch_prer(const T *G, T *C, const Geometry &g, const DirTables &tr,
                        cudaStream_t st);
// drift kernels (the values of the public VLS_DRIFT_* layout choices)
constexpr int DRIFT_AUTO = 0, DRIFT_WINDOW = 1, DRIFT_STRIP2 = 2, DRIFT_STRIP1 = 3;
// footpoints: FP64 handles use idx/fx/fy, FP32 handles the packed fp2 table.
// Drift with the coefficient windows staged by TMA (tmC: 3D map of C, box
// 64 columns x 40 rows x 1 slice); err receives bit 0 when a wait for a
// window ran out after `spins` polls (the cells then read C in global
// memory), bit 1 when a copy had still not landed at the block's end
template <typename T>
cudaError_t launch_drift_tma(const CUtensorMap *tmC, const T *C, T *f, const int32_t *idx,
                             const T *fx, const T *fy, const uint2 *fp2,
                             const int64_t *ch_start, const int32_t *ch_len,
                             const T *ch_val, int64_t ndrift, const MomentTables &mt,
                             double *partial, unsigned int *err, uint32_t spins,
                             const Geometry &g, cudaStream_t st);
// drift with the block's whole coefficient strip staged by TMA (tmS: 3D map
// of C with box 48 columns x 64 rows x 1 slice).  drift_strip_width returns
// the strip kind (DRIFT_STRIP2 / DRIFT_STRIP1) the grid takes, or
// DRIFT_WINDOW when none fits; want != DRIFT_AUTO requests one kind
template <typename T>
int drift_strip_width(int nu, int want);
template <typename T>
cudaError_t launch_drift_strip(const CUtensorMap *tmS, int kind, const T *C, T *f,
                               const int32_t *idx, const T *fx, const T *fy, const uint2 *fp2,
                               const int64_t *ch_start, const int32_t *ch_len,
                               const T *ch_val, int64_t ndrift, const MomentTables &mt,
                               double *partial, unsigned int *err, uint32_t spins,
                               const Geometry &g, cudaStream_t st);
// chains [c_lo, c_hi) (all of the launch's slices) of nchains in total
template <typename T>
cudaError_t launch_chain_tails(const T *C, T *ch_val, const int64_t *ch_start,
                               const int32_t *ch_len, const int32_t *t_idx,
                               const double *t_x, const double *t_y,
                               int64_t nchains, int64_t c_lo, int64_t c_hi,
                               int64_t ndrift, const Geometry &g, cudaStream_t st);
struct HostDirTables;
// chunk layout of the register kernels for a direction (-1: none takes it,
// the shared-memory segment kernels then solve the lines; u_lines for the
// ucol kernel), its chunk length in rows, and its tables
template <typename R>
int rc_config(const HostDirTables &t, bool u_lines);
int rc_chunk_rows(int cfg);
template <typename R>
RcDir<R> rc_dir(const HostDirTables &t, int cfg);
template <typename T, typename R>
cudaError_t launch_ucol_rc(int cfg, bool kick, const T *f, T *G, const double *shift,
                           const Geometry &g, const RcDir<R> &tu, cudaStream_t st);
// err: bit 2 (4) when the bulk staging of a block's rows timed out, bit 3
// (8) when the rows still had not landed at the block's end
template <typename T, typename R>
cudaError_t launch_prer_rc(int cfg, const T *G, T *C, const Geometry &g, const RcDir<R> &tr,
                           unsigned int *err, cudaStream_t st);
// adjoint of the step (vls_adjoint.cu); all adjoint arrays FP64: Cb in C
// layout and Gb, A, B in G layout, each over all J slices
// the drift transposed as a gather over the inverse footpoint map: buckets of
// cells and chain tails by the base node of their stencil (ends: [nj][nr*nu]
// bucket ends within the slice's entries; ent: ids, ascending per bucket;
// ebase: first entry of each slice).  inv_fill counts (ent == nullptr) or
// places; inv_scan turns counts into starts and writes each slice's total.
template <typename T>
cudaError_t launch_inv_fill(const int32_t *idx, const uint2 *fp2, const int32_t *t_idx, int64_t nch, uint32_t *ends, uint32_t *ent,
                            const int64_t *ebase, const Geometry &g, cudaStream_t st);
cudaError_t launch_inv_scan(uint32_t *ends, uint32_t *totals, const Geometry &g,
                            cudaStream_t st);
cudaError_t launch_inv_sort(const uint32_t *ends, uint32_t *ent, const int64_t *ebase,
                            const Geometry &g, cudaStream_t st);
// chain fronts and tails transposed; mB: pending moment term (or null)
cudaError_t launch_chain_adj(const double *lam, const double *mB, const MomentTables &mt,
                             double *ringb, double *tv, const int64_t *ch_cell,
                             const int64_t *ch_start, const int32_t *ch_len, int64_t nch,
                             int64_t ndrift, const Geometry &g, cudaStream_t st);
// cell-ordered gather (one lane per bucket column; entries read through
// their cell index)
template <typename T>
cudaError_t launch_drift_adj_gather(const double *lam, const double *mB, const MomentTables &mt,
                                    const double *tv, double *Cb, const uint32_t *ends,
                                    const uint32_t *ent, const int64_t *ebase, const T *fx,
                                    const T *fy, const uint2 *fp2, const double *t_x,
                                    const double *t_y, const Geometry &g, cudaStream_t st);
// entry-ordered form (FP32 handles whose lam does not fit in L2): packed
// words of the entries once per map, values permuted into entry order each
// step, gather
cudaError_t launch_inv_geo(const uint32_t *ent, const int64_t *ebase, const uint2 *fp2,
                           uint2 *geo, const Geometry &g, cudaStream_t st);
cudaError_t launch_inv_perm(const uint32_t *ent, const int64_t *ebase, const double *lam,
                            const double *mB, const MomentTables &mt, const double *tv,
                            double *vperm, const Geometry &g, cudaStream_t st);
cudaError_t launch_drift_adj_gather_perm(const double *vperm, const uint2 *geo, double *Cb,
                                         const uint32_t *ends, const int64_t *ebase,
                                         const int32_t *t_idx, const double *t_x,
                                         const double *t_y, const Geometry &g, cudaStream_t st);
cudaError_t launch_prer_adj(const double *Cb, double *Gb, const Geometry &g,
                            const DirTables &tr, cudaStream_t st);
template <typename T>
cudaError_t launch_ucol_adj(const T *f, double *Gb, double *A, double *B, double *lam,
                            double *sbar, const double *shift, const Geometry &g,
                            const DirTables &tu, cudaStream_t st);
// beta: 2 N_r values (beta, then the moment's transpose per radius)
cudaError_t launch_shift_adj(const double *sbar, double *beta, unsigned int *count,
                             const MomentTables &mt, const Geometry &g, cudaStream_t st);
cudaError_t launch_moment_adj(double *lam, const double *beta, const MomentTables &mt,
                              const Geometry &g, cudaStream_t st);
// chunked adjoint line kernels (vls_rc.cu), used when rc_adj_supported
bool rc_adj_supported(const HostDirTables &tu, const HostDirTables &tr);
template <typename T>
cudaError_t launch_ucol_adj_rc(const T *f, const double *Gb, double *lam, double *sbar,
                               const double *shift, const Geometry &g, const RcDir<double> &tu,
                               cudaStream_t st);
cudaError_t launch_prer_adj_rc(const double *Cb, double *Gb, const Geometry &g,
                               const RcDir<double> &tr, cudaStream_t st);
template <typename T>
cudaError_t launch_moment(const T *f, const MomentTables &mt, double *partial,
                          const Geometry &g, cudaStream_t st);
// status |= 2 when the total mass is not finite (a NaN or an infinity in f)
cudaError_t launch_scan(const double *partial, const MomentTables &mt,
                        double *T2, double *bins, double *Mr, double *shift,
                        double *mtot, unsigned int *count, unsigned int *status,
                        const Geometry &g, cudaStream_t st);
template <typename T>
cudaError_t launch_stats(const T *f, const double *R, const double *U,
                         const double *J, const double *dR, const double *dU,
                         const double *Ct1, double *part, double *out4,
                         const Geometry &g, cudaStream_t st);
template <typename T>
cudaError_t launch_convert_in(const double *src, T *dst, size_t n,
                              cudaStream_t st);
template <typename T>
cudaError_t launch_convert_out(const T *src, double *dst, size_t n,
                               cudaStream_t st);
template <typename T>
cudaError_t launch_nonfinite(const T *f, size_t n, unsigned int *flag,
                             cudaStream_t st);

// analytic initial profiles on the device (vls_profile.cu): the constants
// Profile::setup derives (vls_setup.cpp), the type a VLS_INIT_* value
struct ProfileConsts {
  int type;
  double R0, smoothingRadius, gap0, gap1, n, M, Ra, G, C0, C1, C2, Vg;
};
// f of every cell from the coordinates xyz = R (nr), U (nu), J (nj), JV (nj + 1)
cudaError_t launch_profile_grid(const ProfileConsts &p, const double *xyz, double *f, int nr,
                                int nu, int nj, cudaStream_t st);
// the mass quadrature of each (j, u) row of f (rows: nu * nj)
cudaError_t launch_profile_rows(const double *f, const double *xyz, double *rows, int nr,
                                int nu, int nj, cudaStream_t st);
// partial sums (profile_dot_blocks() of them) of w (a fp - b fm) over n cells
int profile_dot_blocks();
cudaError_t launch_profile_dot(const double *w, const double *fp, const double *fm, double a,
                               double b, size_t n, double *partial, cudaStream_t st);

}  // namespace vls
