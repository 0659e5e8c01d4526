// vls_adjoint.cu -- kernels of the adjoint (reverse-mode derivative) of the
// linked step f_{n+1} = D P_r P_u Kick(P_u f_n; s(f_n)) + chains.
//
// The reference has no derivative code; this is the transpose of the step as
// the forward kernels compute it (vls_kernels.cu, vls_rc.cu):
//   drift D       f(cell) = sum_ab wy_a wx_b C[uI+a][rI+b] / 36   -> gather over
//                 the inverse footpoint map
//   tails E       ring[tail] = same gather at the chain's end    -> the same
//   prefilter P   natural-BC Thomas solve of each line           -> transposed
//                 recurrences (localSpline.hxx:953-1182 read backwards)
//   kick          per column: gather at y = u + s_r hu           -> transposed
//                 gather, plus d/ds_r of the interpolant
//   shift s       s_r = Rcoef_r sum_{r' < r} bins_r'             -> reverse scan
//   moment        bins_r = dR_r/4 (T_r + T_{r+1}), T_r = sum_j w_j sum_u b_u f
// Adjoint values are FP64 in every precision mode; the forward state they
// linearise around is read in the handle's storage type.  The drift's
// transpose is a gather with a fixed summation order, so the gradient is
// bitwise reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "vls_dd.cuh"
#include "vls_internal.h"

namespace vls {


namespace {

__device__ __forceinline__ double bv2d(double x) { return x * x * x; }
__device__ __forceinline__ double bv1d(double x) {
  return 1.0 + 3.0 * x + 3.0 * x * x - 3.0 * x * x * x;
}
// derivatives of the kick weights w_m(fr)/6 with respect to fr
__device__ __forceinline__ void kick_weights(double fr, double w[4], double dw[4]) {
  const double a = 1.0 - fr;
  w[0] = bv2d(a) / 6.0;
  w[1] = bv1d(a) / 6.0;
  w[2] = bv1d(fr) / 6.0;
  w[3] = bv2d(fr) / 6.0;
  dw[0] = -3.0 * a * a / 6.0;
  dw[1] = -(3.0 + 6.0 * a - 9.0 * a * a) / 6.0;
  dw[2] = (3.0 + 6.0 * fr - 9.0 * fr * fr) / 6.0;
  dw[3] = 3.0 * fr * fr / 6.0;
}

// forward natural-BC solve of a line (FP64): x at xs[(k-1)*xst], k = 1..N;
// coefficients c_0..c_{M-1} to cs[k*cst] (may not alias xs)
__device__ void solve_line_fwd(const double *__restrict__ x, int xst, double *__restrict__ c,
                               int cst, const DirTables &t) {
  const int M = t.M, N = M - 2;
  double d = 0.0, dprev = 0.0;
#pragma unroll 8
  for (int k = 1; k <= N; ++k) {
    dprev = d;
    d = (x[(size_t)(k - 1) * xst] - d * (1.0 / 6.0)) * t.rp[k];
    c[(size_t)k * cst] = d;
  }
  double cc = ((0.0 - t.hi2 * dprev) - t.L1 * d) / t.L2;
  c[(size_t)(M - 1) * cst] = cc;
  double cn = cc;
#pragma unroll 8
  for (int k = N; k >= 1; --k) {
    const double v = c[(size_t)k * cst] - t.q[k] * cn;
    c[(size_t)k * cst] = v;
    cc = cn;
    cn = v;
  }
  // cn = c_1, cc = c_2
  c[0] = (0.0 - t.a01 * cn) - t.a02 * cc;
}

// transposed solve: cbar[k*cst] (k = 0..M-1) -> xbar[(k-1)*xst] (k = 1..N);
// xbar may alias neither cbar's storage nor overlap it
__device__ void solve_line_adj(const double *__restrict__ cb, int cst, double *__restrict__ xb,
                               int xst, const DirTables &t) {
  const int M = t.M, N = M - 2;
  const double c0b = cb[0];
  // back-substitution and first row, transposed (ascending): e_k = cbar_k
  // complete, dbar_k = e_k
  double e = cb[(size_t)1 * cst] - t.a01 * c0b;
  xb[0] = e;
#pragma unroll 8
  for (int k = 2; k <= N; ++k) {
    double ck = cb[(size_t)k * cst];
    if (k == 2) ck -= t.a02 * c0b;
    e = ck - t.q[k - 1] * e;
    xb[(size_t)(k - 1) * xst] = e;
  }
  double cMb = cb[(size_t)(M - 1) * cst] - t.q[N] * e;
  if (N == 1) cMb -= t.a02 * c0b;  // c_2 is then the last coefficient
  // last row, transposed
  if (N >= 2) xb[(size_t)(N - 2) * xst] += -(t.hi2 / t.L2) * cMb;
  xb[(size_t)(N - 1) * xst] += -(t.L1 / t.L2) * cMb;
  // forward elimination, transposed (descending)
  double fk = xb[(size_t)(N - 1) * xst];
  xb[(size_t)(N - 1) * xst] = t.rp[N] * fk;
#pragma unroll 8
  for (int k = N - 1; k >= 1; --k) {
    fk = xb[(size_t)(k - 1) * xst] - (1.0 / 6.0) * t.rp[k + 1] * fk;
    xb[(size_t)(k - 1) * xst] = t.rp[k] * fk;
  }
}

constexpr uint32_t AFP_CHAIN = 0xFFFFFFFEu;
constexpr int AFP_FBITS = 21;

// r-solve, transposed: each row k of every slice, Cb[j][k][0..M_r-1] ->
// Gb[j][k][0..N_r-1]
__global__ void prer_adj_kernel(const double *__restrict__ Cb, double *__restrict__ Gb,
                                Geometry g, DirTables tr) {
  const int rows = g.nu + 2;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)rows * g.nj) return;
  const int j = (int)(i / rows), k = (int)(i % rows);
  const double *cb = Cb + ((size_t)j * (g.nu + 3) + k) * g.pc;
  double *gb = Gb + ((size_t)j * rows + k) * g.nr;
  solve_line_adj(cb, 1, gb, 1, tr);
}

// u-solves and kick, transposed, one thread per (slice, column):
//   g    = P_u f_n                      (scratch A, G layout)
//   fbar = P_u^T Gb                     (in place in Gb rows 1..N_u)
//   gbar = Kick^T fbar, sbar partial    (scratch B, G layout)
//   lam  = P_u^T gbar                   (cells)
template <typename T>
__global__ void ucol_adj_kernel(const T *__restrict__ f, double *__restrict__ Gb,
                                double *__restrict__ A, double *__restrict__ B,
                                double *__restrict__ lam, double *__restrict__ sbar,
                                const double *__restrict__ shift, Geometry g, DirTables tu) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)g.nr * g.nj) return;
  const int j = (int)(i / g.nr), r = (int)(i % g.nr);
  const int N = g.nu, M = N + 2;
  const size_t gofs = (size_t)j * M * g.nr + r;
  double *gcol = A + gofs;     // g = P_u f_n, rows 0..M-1
  double *bcol = B + gofs;     // gbar
  double *Gcol = Gb + gofs;    // Gbar -> fbar (rows 1..N hold fbar_u at row u+1)
  const size_t fofs = (size_t)j * N * g.nr + r;
  // g = P_u f_n (f read as FP64)
  {
    // solve_line_fwd reads x from a double array: stage f into bcol rows 1..N
    for (int u = 0; u < N; ++u) bcol[(size_t)(u + 1) * g.nr] = (double)f[fofs + (size_t)u * g.nr];
    solve_line_fwd(bcol + g.nr, g.nr, gcol, g.nr, tu);
  }
  // fbar = P_u^T Gbar, written to bcol rows 1..N (then moved back to Gcol)
  solve_line_adj(Gcol, g.nr, bcol + g.nr, g.nr, tu);
  for (int u = 0; u < N; ++u) Gcol[(size_t)(u + 1) * g.nr] = bcol[(size_t)(u + 1) * g.nr];
  for (int k = 0; k < M; ++k) bcol[(size_t)k * g.nr] = 0.0;
  // kick, transposed (vlasovSolver21_spline.hxx:752-770 as the forward
  // kernels compute it: fast path with one fraction per column, or the exact
  // per-cell path when the fraction is within 1e-9 of a node)
  const double sft = shift[r];
  const double qf = sft * g.hu;
  const double fl = floor(qf);
  const double frd = qf - fl;
  const bool fast = frd > 1e-9 && frd < 1.0 - 1e-9 && fabs(qf) < 1e6;
  double sb = 0.0;
  double w[4], dw[4];
  if (fast) kick_weights(frd, w, dw);
  const int o = fast ? (int)fl : 0;
  const int ulo = fast ? (int)floor(-qf) + 1 : 0;
  const int uhi = fast ? (int)ceil((double)(N - 1) - qf) - 1 : -1;
  for (int u = 0; u < N; ++u) {
    const double fb = Gcol[(size_t)(u + 1) * g.nr];
    int Ny;
    if (fast) {
      if (u < ulo || u > uhi) continue;
      Ny = 1 + u + o;
    } else {
      const double newU = g.U[u] + sft;
      if (!(newU > g.u0 && newU < g.umax)) continue;
      const double y = (newU - g.su) * g.hu;
      const double yf = floor(y);
      kick_weights(y - yf, w, dw);
      Ny = 1 + (int)yf;
    }
    double dv = 0.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      // a tap on row M is the forward's always-zero guard row
      if (Ny - 1 + m >= M) continue;
      const size_t row = (size_t)(Ny - 1 + m) * g.nr;
      bcol[row] += w[m] * fb;
      dv += dw[m] * gcol[row];
    }
    sb += fb * dv * g.hu;
  }
  sbar[(size_t)j * g.nr + r] = sb;
  // lam = P_u^T gbar
  solve_line_adj(bcol, g.nr, lam + fofs, g.nr, tu);
}

// shift, transposed: sbar (per slice) -> beta_r' = sum_{r > r'} Rcoef_r sum_j sbar[j][r]
// (beta[0..N_r)), and the moment's transpose per radius to beta[N_r..2 N_r).
// Each block sums 32 radii over the slices (32 slice groups j = w, w + 32,
// ... in parallel, then the groups in order) into beta[N_r + r] as scratch;
// the last block to finish (count, left at zero again) runs the reverse
// exclusive scan over the radii, compensated as the forward's enclosed-mass
// scan, and writes the moment term over the scratch.  The summation order is
// fixed.
__global__ void __launch_bounds__(1024) shift_adj_kernel(const double *__restrict__ sbar,
                                                         double *beta, unsigned int *count,
                                                         MomentTables mt, Geometry g) {
  __shared__ double part[32][33];
  __shared__ dd wsum[32];
  __shared__ bool last;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  {
    const int r = blockIdx.x * 32 + lane;
    double s = 0.0;
    if (r < g.nr) {
#pragma unroll 8
      for (int j = w; j < g.nj; j += 32) s += __ldg(sbar + (size_t)j * g.nr + r);
    }
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && r < g.nr) {
      double t = 0.0;
      for (int k = 0; k < 32; ++k) t += part[k][lane];
      beta[g.nr + r] = t * mt.Rcoef[r];
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // q = N_r - 1 - r ascending: thread t holds q = t per .. t per + per - 1
  const int per = (g.nr + 1023) / 1024;  // 1 or 2
  double x[2] = {0.0, 0.0};
  dd loc{0.0, 0.0};
  for (int k = 0; k < per; ++k) {
    const int q = tid * per + k;
    if (q < g.nr) {
      x[k] = *((volatile double *)beta + g.nr + (g.nr - 1 - q));
      loc = dd_add(loc, dd{x[k], 0.0});
    }
  }
  dd inc = loc;
  for (int d = 1; d < 32; d <<= 1) {
    const dd o = dd_shfl_up(inc, d);
    if (lane >= d) inc = dd_add(inc, o);
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    const dd xw = wsum[lane];
    dd xi = xw;
    for (int d = 1; d < 32; d <<= 1) {
      const dd o = dd_shfl_up(xi, d);
      if (lane >= d) xi = dd_add(xi, o);
    }
    wsum[lane] = dd_add(xi, dd{-xw.hi, -xw.lo});  // exclusive over warps
  }
  __syncthreads();
  dd ex = dd_add(wsum[w], dd_add(inc, dd{-loc.hi, -loc.lo}));
  for (int k = 0; k < per; ++k) {
    const int q = tid * per + k;
    if (q < g.nr) {
      beta[g.nr - 1 - q] = ex.hi + ex.lo;  // exclusive: bins_r' enters s_r for r > r'
      ex = dd_add(ex, dd{x[k], 0.0});
    }
  }
  // the moment's transpose per radius: mB_r = beta_r dR4_r + beta_{r-1} dR4_{r-1}
  __syncthreads();
  for (int r = tid; r < g.nr; r += blockDim.x) {
    double b = beta[r] * mt.dR4[r];
    if (r > 0) b += beta[r - 1] * mt.dR4[r - 1];
    beta[g.nr + r] = b;
  }
  if (tid == 0) *count = 0u;
}

// moment, transposed: lam += w_j b_u (beta_r dR_r/4 + beta_{r-1} dR_{r-1}/4)
__global__ void moment_adj_kernel(double *__restrict__ lam, const double *__restrict__ beta,
                                  MomentTables mt, Geometry g) {
  const size_t n = (size_t)g.nr * g.nu * g.nj;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % g.nr);
    const size_t ju = i / g.nr;
    const int u = (int)(ju % g.nu), j = (int)(ju / g.nu);
    double b = beta[r] * mt.dR4[r];
    if (r > 0) b += beta[r - 1] * mt.dR4[r - 1];
    lam[i] += mt.wj[j] * mt.bu[u] * b;
  }
}

unsigned grid_for(size_t n, int threads) {
  size_t b = (n + threads - 1) / threads;
  if (b > 148 * 64) b = 148 * 64;
  return (unsigned)(b ? b : 1);
}

// ---------------------------------------------------------------------------
// The drift transposed as a gather over the inverse footpoint map.  The
// footpoints are fixed for the run, so the cells (and chain tails) whose 4 x 4
// stencil starts at base node (uI, rI) of slice j are listed once: bucket key
// uI * N_r + rI, per slice, entries ascending by id within a bucket (u << 16
// | r of the cell, N_u < 2^15, or INV_TAIL | chain id).  Every C node then
// sums the contributions of the 16 buckets that reach it, in a fixed order:
// the result does not depend on scheduling, and no FP64 atomics are issued.
//
// The moment's transpose (lam += w_j b_u B_r, B_r = beta_r dR_r/4 +
// beta_{r-1} dR_{r-1}/4) is not applied to lam as a pass of its own: the
// readers of lam in the next transposed step (this gather and the chain
// fronts) add it to the values they read (mB = B, or null for none).

constexpr uint32_t INV_TAIL = 0x80000000u;

// base node of cell i's stencil; false for cells outside the box and chain
// fronts (the forward drift's decode, vls_kernels.cu)
template <typename T>
__device__ __forceinline__ bool cell_base(size_t i, const int32_t *__restrict__ idx,
                                          const uint2 *__restrict__ fp2, int &rI, int &uI,
                                          uint2 &w) {
  if (sizeof(T) == 8) {
    const int code = idx[i];
    if (code < 0) return false;
    rI = code & 0xffff;
    uI = code >> 16;
    return true;
  }
  w = fp2[i];
  if (w.x >= AFP_CHAIN) return false;
  rI = (int)(w.x >> AFP_FBITS);
  uI = (int)(w.y >> AFP_FBITS);
  return true;
}

// one pass over the cells and chain tails: count (ent == nullptr) or place
// each into its bucket (ends then hold the bucket starts and end as the
// bucket ends)
template <typename T>
__global__ void inv_fill_kernel(const int32_t *__restrict__ idx, const uint2 *__restrict__ fp2,
                                const int32_t *__restrict__ t_idx,
                                int64_t nch, uint32_t *__restrict__ ends,
                                uint32_t *__restrict__ ent, const int64_t *__restrict__ ebase,
                                Geometry g) {
  const size_t S = (size_t)g.nr * g.nu, n = S * g.nj;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n + (size_t)nch;
       i += (size_t)gridDim.x * blockDim.x) {
    int rI, uI, j;
    uint32_t id;
    if (i < n) {
      uint2 w;
      if (!cell_base<T>(i, idx, fp2, rI, uI, w)) continue;
      j = (int)(i / S);
      const uint32_t within = (uint32_t)(i - (size_t)j * S);
      id = (within / (uint32_t)g.nr) << 16 | (within % (uint32_t)g.nr);
    } else {
      const int64_t c = (int64_t)(i - n);
      const int code = t_idx[c];
      if (code < 0) continue;
      rI = code & 0xffff;
      uI = code >> 16;
      j = t_idx[nch + c];
      id = INV_TAIL | (uint32_t)c;
    }
    uint32_t *b = ends + (size_t)j * S + (size_t)uI * g.nr + rI;
    if (!ent) {
      atomicAdd(b, 1u);
    } else {
      const uint32_t pos = atomicAdd(b, 1u);
      ent[ebase[j] + pos] = id;
    }
  }
}

// exclusive scan of each slice's bucket counts in place (one block of 1024
// threads per slice); the slice's entry count to totals[j]
__global__ void __launch_bounds__(1024) inv_scan_kernel(uint32_t *__restrict__ ends,
                                                        uint32_t *__restrict__ totals,
                                                        int64_t S) {
  __shared__ uint32_t wsum[32];
  uint32_t *e = ends + (size_t)blockIdx.x * S;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (int64_t t0 = 0; t0 < S; t0 += 1024) {
    const int64_t i = t0 + threadIdx.x;
    const uint32_t v = i < S ? e[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      uint32_t s = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    if (i < S) e[i] = carry + (w ? wsum[w - 1] : 0u) + x - v;
    carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// order each bucket's entries by id (the placement's atomics leave them in
// any order)
__global__ void inv_sort_kernel(const uint32_t *__restrict__ ends, uint32_t *__restrict__ ent,
                                const int64_t *__restrict__ ebase, int64_t S, int64_t nkeys) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nkeys;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = k / S;
    const uint32_t s = k - j * S ? ends[k - 1] : 0u, e = ends[k];
    uint32_t *p = ent + ebase[j];
    for (uint32_t a = s + 1; a < e; ++a) {
      const uint32_t v = p[a];
      uint32_t b = a;
      while (b > s && p[b - 1] > v) {
        p[b] = p[b - 1];
        --b;
      }
      p[b] = v;
    }
  }
}

// chain fronts and tails, transposed, one thread per chain: the front slot
// takes the adjoint of the cell that read it; the tail slot's adjoint (the
// value this step's tails wrote) moves to tv for the gather and is cleared.
// In the forward the tails write before the drift reads, so with L = 1 the
// front add comes first here.
__global__ void chain_adj_kernel(const double *__restrict__ lam, const double *__restrict__ mB,
                                 MomentTables mt, double *__restrict__ ringb,
                                 double *__restrict__ tv, const int64_t *__restrict__ ch_cell,
                                 const int64_t *__restrict__ ch_start,
                                 const int32_t *__restrict__ ch_len, int64_t nch,
                                 int64_t ndrift, Geometry g) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const int L = ch_len[c];
  double *ring = ringb + ch_start[c];
  const int64_t i = ch_cell[c];
  double v = lam[i];
  if (mB) {
    const int r = (int)(i % g.nr);
    const int64_t ju = i / g.nr;
    v += mt.wj[ju / g.nu] * mt.bu[ju % g.nu] * mB[r];
  }
  ring[ndrift % L] += v;
  double *slot = ring + (ndrift + L - 1) % L;
  tv[c] = *slot;
  *slot = 0.0;
}

// weight m of the cubic B-spline at fraction t (times 6): m = 0..3 are
// BV2(1-t), BV1(1-t), BV1(t), BV2(t), the drift's tap weights
__device__ __forceinline__ double bweight(int m, double t) {
  const double s = m < 2 ? 1.0 - t : t;
  return (m == 0 || m == 3) ? bv2d(s) : bv1d(s);
}

// Cb[j][p][q] = sum over the buckets (p - a, q - b), a, b = 0..3, of
// lam * w_a(y) w_b(x) / 36, by one of two gathers: lane_nodes (one lane per
// bucket column, entries read through their cell index) or sweep_nodes (a
// thread per block of node rows and columns, entries read in entry order).

// Entry order (FP32 handles whose lam does not fit in L2).  The packed
// footpoint word of each entry (a chain tail is GEO_TAIL, chain id) is
// stored once in entry order when the map is built, and each transposed
// step first permutes its values into entry order (vperm: lam plus the
// pending moment term, or the tail's ring adjoint), so that a visit of the
// gather reads two arrays at the same index.
constexpr uint32_t GEO_TAIL = 0xFFFFFFFFu;

__global__ void inv_geo_kernel(const uint32_t *__restrict__ ent,
                               const int64_t *__restrict__ ebase, const uint2 *__restrict__ fp2,
                               uint2 *__restrict__ geo, Geometry g) {
  const int j = blockIdx.y;
  const int64_t e0 = ebase[j], e1 = ebase[j + 1];
  const size_t cbase = (size_t)j * g.nr * g.nu;
  for (int64_t e = e0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < e1;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ent[e];
    if (id & INV_TAIL) {
      geo[e] = make_uint2(GEO_TAIL, id & ~INV_TAIL);
      continue;
    }
    geo[e] = fp2[cbase + (size_t)(id >> 16) * g.nr + (id & 0xffffu)];
  }
}

// values of this transposed step in entry order
__global__ void inv_perm_kernel(const uint32_t *__restrict__ ent,
                                const int64_t *__restrict__ ebase, const double *__restrict__ lam,
                                const double *__restrict__ mB, MomentTables mt,
                                const double *__restrict__ tv, double *__restrict__ vperm,
                                Geometry g) {
  const int j = blockIdx.y;
  const int64_t e0 = ebase[j], e1 = ebase[j + 1];
  const size_t cbase = (size_t)j * g.nr * g.nu;
  const double wjj = mB ? mt.wj[j] : 0.0;
  for (int64_t e = e0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < e1;
       e += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ent[e];
    double v;
    if (id & INV_TAIL) {
      v = tv[id & ~INV_TAIL];
    } else {
      const int u = (int)(id >> 16), r = (int)(id & 0xffffu);
      v = lam[cbase + (size_t)u * g.nr + r];
      if (mB) v += wjj * mt.bu[u] * mB[r];
    }
    vperm[e] = v;
  }
}

// The entry-ordered gather.  A thread sums the nodes of RB rows p0.. and Q
// columns q0.., walking the base rows p0-3 .. p0+RB-1 in order with the sums
// of the four node rows pb .. pb+3 in registers: node row pb is complete
// once base row pb is done (base rows pb-3 .. pb are the only ones reaching
// it) and is written then.  The buckets of one base row reaching the Q
// columns are adjacent, one contiguous run of entries.  Every node receives
// its contributions in a fixed order (base rows ascending, entries in
// bucket order), so the result does not depend on scheduling.  The sliding
// window keeps four rows of sums per column in registers (a block of RB
// rows held whole measured 8-12 % slower: more registers, fewer warps, more
// visits of each entry).  entry(e, v, x, y, rI) reads entry e of the slice.
template <int RB, int Q, class Entry>
__device__ __forceinline__ void sweep_nodes(const Entry &entry, double *__restrict__ Cbj,
                                            const uint32_t *__restrict__ endj, int p0, int q0,
                                            const Geometry &g) {
  const int qlo = max(q0 - 3, 0), qhi = min(q0 + Q - 1, g.nr - 1);
  double acc[4][Q];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int k = 0; k < Q; ++k) acc[a][k] = 0.0;
  const int pend = min(p0 + RB, g.nu + 3);
  for (int pb = p0 - 3; pb < pend; ++pb) {
    if (pb >= 0 && pb < g.nu && qlo <= qhi) {
      const size_t k0 = (size_t)pb * g.nr + qlo, k1 = (size_t)pb * g.nr + qhi;
      const uint32_t e1 = endj[k1];
      for (uint32_t e = k0 ? endj[k0 - 1] : 0u; e < e1; ++e) {
        double v, x, y;
        int rI;
        entry(e, v, x, y, rI);
        const double s = 1.0 - y;
        const double wy[4] = {bv2d(s), bv1d(s), bv1d(y), bv2d(y)};
#pragma unroll
        for (int k = 0; k < Q; ++k) {
          const int b = q0 + k - rI;
          const double c = (b >= 0 && b <= 3) ? v * bweight(b, x) : 0.0;
#pragma unroll
          for (int a = 0; a < 4; ++a) acc[a][k] += c * wy[a];
        }
      }
    }
    if (pb >= p0) {
      double *out = Cbj + (size_t)pb * g.pc + q0;
#pragma unroll
      for (int k = 0; k < Q; ++k)
        if (q0 + k < g.pc) out[k] = acc[0][k] * (1.0 / 36.0);
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      acc[0][k] = acc[1][k];
      acc[1][k] = acc[2][k];
      acc[2][k] = acc[3][k];
      acc[3][k] = 0.0;
    }
  }
}

template <int RB, int Q>
__global__ void __launch_bounds__(128)
    drift_adj_sweep_perm_kernel(const double *__restrict__ vperm, const uint2 *__restrict__ geo,
                                double *__restrict__ Cb, const uint32_t *__restrict__ ends,
                                const int64_t *__restrict__ ebase,
                                const int32_t *__restrict__ t_idx,
                                const double *__restrict__ t_x, const double *__restrict__ t_y,
                                Geometry g) {
  const int q0 = (blockIdx.x * 32 + threadIdx.x) * Q;
  const int p0 = (blockIdx.y * blockDim.y + threadIdx.y) * RB;
  const int j = blockIdx.z;
  if (q0 >= g.pc || p0 >= g.nu + 3) return;
  const size_t S = (size_t)g.nr * g.nu;
  const int64_t eb = ebase[j];
  const double *vj = vperm + eb;
  const uint2 *gj = geo + eb;
  sweep_nodes<RB, Q>(
      [&](uint32_t e, double &v, double &x, double &y, int &rI) {
        v = vj[e];
        const uint2 w = gj[e];
        if (w.x == GEO_TAIL) {
          rI = t_idx[w.y] & 0xffff;
          x = t_x[w.y];
          y = t_y[w.y];
        } else {
          rI = (int)(w.x >> AFP_FBITS);
          const uint32_t m = (1u << AFP_FBITS) - 1u;
          x = (double)(__uint_as_float(0x3F800000u | ((w.x & m) << 2)) - 1.0f);
          y = (double)(__uint_as_float(0x3F800000u | ((w.y & m) << 2)) - 1.0f);
        }
      },
      Cb + (size_t)j * (g.nu + 3) * g.pc, ends + (size_t)j * S, p0, q0, g);
}

// The cell-ordered gather.  A warp covers 32 consecutive bucket
// columns cb = c0 - 3 + lane of one block of node rows; each lane visits
// only its own bucket of each base row (every entry of the block once per
// pass, no per-column tests) and adds the entry's 4 x 4 products into the
// sums of the node rows pb .. pb + 3 and columns cb .. cb + 3 it holds.  A
// node row is complete once its own base row is done; node column q then
// sums the lanes q - b's column-offset-b sums, b = 0 .. 3, by shuffles in
// that order, and lanes 3 .. 31 write the 29 columns c0 .. c0 + 28.  The
// summation order is fixed.  entry(e, v, x, y) reads entry e of the slice
// (its bucket gives the base node).
template <int RB, class Entry>
__device__ __forceinline__ void lane_nodes(const Entry &entry, double *__restrict__ Cbj,
                                           const uint32_t *__restrict__ endj, int p0, int c0,
                                           const Geometry &g) {
  const int lane = threadIdx.x & 31;
  const int cb = c0 - 3 + lane;
  const bool col_ok = cb >= 0 && cb < g.nr;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  const int pend = min(p0 + RB, g.nu + 3);
  for (int pb = p0 - 3; pb < pend; ++pb) {
    if (col_ok && pb >= 0 && pb < g.nu) {
      const size_t k = (size_t)pb * g.nr + cb;
      const uint32_t e1 = endj[k];
      for (uint32_t e = k ? endj[k - 1] : 0u; e < e1; ++e) {
        double v, x, y;
        entry(e, v, x, y);
        const double sy = 1.0 - y, sx = 1.0 - x;
        const double wy[4] = {bv2d(sy), bv1d(sy), bv1d(y), bv2d(y)};
        const double vx[4] = {v * bv2d(sx), v * bv1d(sx), v * bv1d(x), v * bv2d(x)};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) acc[a][b] = fma(vx[b], wy[a], acc[a][b]);
      }
    }
    // node row pb is complete
    double t = acc[0][0];
    t += __shfl_up_sync(0xffffffffu, acc[0][1], 1);
    t += __shfl_up_sync(0xffffffffu, acc[0][2], 2);
    t += __shfl_up_sync(0xffffffffu, acc[0][3], 3);
    if (pb >= p0 && lane >= 3 && cb < g.pc) Cbj[(size_t)pb * g.pc + cb] = t * (1.0 / 36.0);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      acc[0][b] = acc[1][b];
      acc[1][b] = acc[2][b];
      acc[2][b] = acc[3][b];
      acc[3][b] = 0.0;
    }
  }
}

template <typename T, int RB>
__global__ void __launch_bounds__(128)
    drift_adj_lane_kernel(const double *__restrict__ lam, const double *__restrict__ mB,
                          MomentTables mt, const double *__restrict__ tv,
                          double *__restrict__ Cb, const uint32_t *__restrict__ ends,
                          const uint32_t *__restrict__ ent, const int64_t *__restrict__ ebase,
                          const T *__restrict__ fx, const T *__restrict__ fy,
                          const uint2 *__restrict__ fp2, const double *__restrict__ t_x,
                          const double *__restrict__ t_y, Geometry g) {
  const int c0 = blockIdx.x * 29;
  const int p0 = (blockIdx.y * blockDim.y + threadIdx.y) * RB;
  const int j = blockIdx.z;
  if (p0 >= g.nu + 3) return;  // the whole warp
  const size_t S = (size_t)g.nr * g.nu;
  const uint32_t *entj = ent + ebase[j];
  const size_t cbase = (size_t)j * S;
  const double wjj = mB ? mt.wj[j] : 0.0;
  lane_nodes<RB>(
      [&](uint32_t e, double &v, double &x, double &y) {
        const uint32_t id = entj[e];
        if (id & INV_TAIL) {
          const uint32_t c = id & ~INV_TAIL;
          v = tv[c];
          x = t_x[c];
          y = t_y[c];
          return;
        }
        const int u = (int)(id >> 16), r = (int)(id & 0xffffu);
        const size_t i = cbase + (size_t)u * g.nr + r;
        v = lam[i];
        if (mB) v += wjj * mt.bu[u] * mB[r];
        if (sizeof(T) == 8) {
          x = (double)fx[i];
          y = (double)fy[i];
        } else {
          const uint2 w = fp2[i];
          const uint32_t m = (1u << AFP_FBITS) - 1u;
          x = (double)(__uint_as_float(0x3F800000u | ((w.x & m) << 2)) - 1.0f);
          y = (double)(__uint_as_float(0x3F800000u | ((w.y & m) << 2)) - 1.0f);
        }
      },
      Cb + (size_t)j * (g.nu + 3) * g.pc, ends + (size_t)j * S, p0, c0, g);
}

template <int RB>
__global__ void __launch_bounds__(128)
    drift_adj_lane_perm_kernel(const double *__restrict__ vperm, const uint2 *__restrict__ geo,
                               double *__restrict__ Cb, const uint32_t *__restrict__ ends,
                               const int64_t *__restrict__ ebase, const double *__restrict__ t_x,
                               const double *__restrict__ t_y, Geometry g) {
  const int c0 = blockIdx.x * 29;
  const int p0 = (blockIdx.y * blockDim.y + threadIdx.y) * RB;
  const int j = blockIdx.z;
  if (p0 >= g.nu + 3) return;  // the whole warp
  const size_t S = (size_t)g.nr * g.nu;
  const int64_t eb = ebase[j];
  const double *vj = vperm + eb;
  const uint2 *gj = geo + eb;
  lane_nodes<RB>(
      [&](uint32_t e, double &v, double &x, double &y) {
        v = vj[e];
        const uint2 w = gj[e];
        if (w.x == GEO_TAIL) {
          x = t_x[w.y];
          y = t_y[w.y];
        } else {
          const uint32_t m = (1u << AFP_FBITS) - 1u;
          x = (double)(__uint_as_float(0x3F800000u | ((w.x & m) << 2)) - 1.0f);
          y = (double)(__uint_as_float(0x3F800000u | ((w.y & m) << 2)) - 1.0f);
        }
      },
      Cb + (size_t)j * (g.nu + 3) * g.pc, ends + (size_t)j * S, p0, c0, g);
}

}  // namespace

template <typename T>
cudaError_t launch_inv_fill(const int32_t *idx, const uint2 *fp2,
                            const int32_t *t_idx, int64_t nch, uint32_t *ends, uint32_t *ent,
                            const int64_t *ebase, const Geometry &g, cudaStream_t st) {
  const size_t n = (size_t)g.nr * g.nu * g.nj + (size_t)nch;
  inv_fill_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(idx, fp2, t_idx, nch, ends, ent,
                                                        ebase, g);
  return cudaGetLastError();
}

cudaError_t launch_inv_scan(uint32_t *ends, uint32_t *totals, const Geometry &g,
                            cudaStream_t st) {
  inv_scan_kernel<<<g.nj, 1024, 0, st>>>(ends, totals, (int64_t)g.nr * g.nu);
  return cudaGetLastError();
}

cudaError_t launch_inv_sort(const uint32_t *ends, uint32_t *ent, const int64_t *ebase,
                            const Geometry &g, cudaStream_t st) {
  const int64_t S = (int64_t)g.nr * g.nu;
  inv_sort_kernel<<<grid_for((size_t)S * g.nj, 256), 256, 0, st>>>(ends, ent, ebase, S,
                                                                   S * g.nj);
  return cudaGetLastError();
}

cudaError_t launch_chain_adj(const double *lam, const double *mB, const MomentTables &mt,
                             double *ringb, double *tv, const int64_t *ch_cell,
                             const int64_t *ch_start, const int32_t *ch_len, int64_t nch,
                             int64_t ndrift, const Geometry &g, cudaStream_t st) {
  if (nch <= 0) return cudaSuccess;
  chain_adj_kernel<<<(unsigned)((nch + 255) / 256), 256, 0, st>>>(
      lam, mB, mt, ringb, tv, ch_cell, ch_start, ch_len, nch, ndrift, g);
  return cudaGetLastError();
}

// SMs of the current device, looked up once per device
static int device_sms() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

// threads of a gather with R node rows and Q columns per thread, in waves of
// 1024 resident threads per SM
static double gather_waves(const Geometry &g, int Q, int R) {
  const double cols = 32.0 * ((g.pc + 32 * Q - 1) / (32 * Q));
  const double rows = 4.0 * ((g.nu + 3 + 4 * R - 1) / (4 * R));
  return cols * rows * g.nj / (1024.0 * device_sms());
}

// the same for the lane-per-bucket gather (29 node columns per warp)
static double lane_waves(const Geometry &g, int R) {
  const double cols = 32.0 * ((g.pc + 28) / 29);
  const double rows = 4.0 * ((g.nu + 3 + 4 * R - 1) / (4 * R));
  return cols * rows * g.nj / (1024.0 * device_sms());
}

template <typename T>
cudaError_t launch_drift_adj_gather(const double *lam, const double *mB, const MomentTables &mt,
                                    const double *tv, double *Cb, const uint32_t *ends,
                                    const uint32_t *ent, const int64_t *ebase, const T *fx,
                                    const T *fy, const uint2 *fp2, const double *t_x,
                                    const double *t_y, const Geometry &g, cudaStream_t st) {
  // 32 node rows per warp where that still gives 4 waves of threads, else
  // 16.  Per transposed step, FP64: 257 x 257 x 128 0.163 ms (8 / 32 rows
  // 0.168 / 0.167; the entry-ordered gather 0.190), 513 x 513 x 256 1.081 ms
  // (16 rows 1.114; entry-ordered 1.101), 1025 x 1025 x 64 1.056 ms (16 rows
  // 1.093; entry-ordered 1.044); FP32 257 x 257 x 128 0.155 ms (entry-ordered
  // with its permutation 0.184)
  auto go = [&](auto kern, int R) {
    const dim3 grid((unsigned)((g.pc + 28) / 29), (unsigned)((g.nu + 3 + 4 * R - 1) / (4 * R)),
                    (unsigned)g.nj);
    kern<<<grid, dim3(32, 4), 0, st>>>(lam, mB, mt, tv, Cb, ends, ent, ebase, fx, fy, fp2, t_x,
                                       t_y, g);
    return cudaGetLastError();
  };
  if (lane_waves(g, 32) >= 4.0) return go(drift_adj_lane_kernel<T, 32>, 32);
  return go(drift_adj_lane_kernel<T, 16>, 16);
}

static dim3 slice_grid(const Geometry &g) {
  const size_t per = ((size_t)g.nr * g.nu + 255) / 256;
  return dim3((unsigned)std::min<size_t>(per ? per : 1, 64), (unsigned)g.nj);
}

cudaError_t launch_inv_geo(const uint32_t *ent, const int64_t *ebase, const uint2 *fp2,
                           uint2 *geo, const Geometry &g, cudaStream_t st) {
  inv_geo_kernel<<<slice_grid(g), 256, 0, st>>>(ent, ebase, fp2, geo, g);
  return cudaGetLastError();
}

cudaError_t launch_inv_perm(const uint32_t *ent, const int64_t *ebase, const double *lam,
                            const double *mB, const MomentTables &mt, const double *tv,
                            double *vperm, const Geometry &g, cudaStream_t st) {
  inv_perm_kernel<<<slice_grid(g), 256, 0, st>>>(ent, ebase, lam, mB, mt, tv, vperm, g);
  return cudaGetLastError();
}

cudaError_t launch_drift_adj_gather_perm(const double *vperm, const uint2 *geo, double *Cb,
                                         const uint32_t *ends, const int64_t *ebase,
                                         const int32_t *t_idx, const double *t_x,
                                         const double *t_y, const Geometry &g, cudaStream_t st) {
  constexpr int Q = 2;
  auto go = [&](auto kern, int R) {
    const dim3 grid((unsigned)((g.pc + 32 * Q - 1) / (32 * Q)),
                    (unsigned)((g.nu + 3 + 4 * R - 1) / (4 * R)), (unsigned)g.nj);
    kern<<<grid, dim3(32, 4), 0, st>>>(vperm, geo, Cb, ends, ebase, t_idx, t_x, t_y, g);
    return cudaGetLastError();
  };
  if (gather_waves(g, Q, 32) >= 4.0) return go(drift_adj_sweep_perm_kernel<32, Q>, 32);
  return go(drift_adj_sweep_perm_kernel<16, Q>, 16);
}

#define VLS_INV_INST(T)                                                                       \
  template cudaError_t launch_inv_fill<T>(const int32_t *, const uint2 *,                      \
                                          const int32_t *, int64_t, uint32_t *, uint32_t *,    \
                                          const int64_t *, const Geometry &, cudaStream_t);    \
  template cudaError_t launch_drift_adj_gather<T>(                                            \
      const double *, const double *, const MomentTables &, const double *, double *,         \
      const uint32_t *, const uint32_t *, const int64_t *, const T *, const T *,              \
      const uint2 *, const double *, const double *, const Geometry &, cudaStream_t);
VLS_INV_INST(float)

VLS_INV_INST(double)
#undef VLS_INV_INST

cudaError_t launch_prer_adj(const double *Cb, double *Gb, const Geometry &g,
                            const DirTables &tr, cudaStream_t st) {
  const int64_t n = (int64_t)(g.nu + 2) * g.nj;
  prer_adj_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(Cb, Gb, g, tr);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ucol_adj(const T *f, double *Gb, double *A, double *B, double *lam,
                            double *sbar, const double *shift, const Geometry &g,
                            const DirTables &tu, cudaStream_t st) {
  const int64_t n = (int64_t)g.nr * g.nj;
  ucol_adj_kernel<T><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(f, Gb, A, B, lam, sbar,
                                                                   shift, g, tu);
  return cudaGetLastError();
}

cudaError_t launch_shift_adj(const double *sbar, double *beta, unsigned int *count,
                             const MomentTables &mt, const Geometry &g, cudaStream_t st) {
  if (g.nr > 2048) return cudaErrorInvalidValue;
  shift_adj_kernel<<<(g.nr + 31) / 32, 1024, 0, st>>>(sbar, beta, count, mt, g);
  return cudaGetLastError();
}

cudaError_t launch_moment_adj(double *lam, const double *beta, const MomentTables &mt,
                              const Geometry &g, cudaStream_t st) {
  const size_t n = (size_t)g.nr * g.nu * g.nj;
  moment_adj_kernel<<<grid_for(n, 256), 256, 0, st>>>(lam, beta, mt, g);
  return cudaGetLastError();
}

template cudaError_t launch_ucol_adj<float>(const float *, double *, double *, double *,
                                            double *, double *, const double *,
                                            const Geometry &, const DirTables &, cudaStream_t);
template cudaError_t launch_ucol_adj<double>(const double *, double *, double *, double *,
                                             double *, double *, const double *,
                                             const Geometry &, const DirTables &, cudaStream_t);

}  // namespace vls
