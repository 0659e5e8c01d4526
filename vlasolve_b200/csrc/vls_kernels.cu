// vls_kernels.cu -- sm_100a kernels of the split semi-Lagrangian step.
//
// Per step (linked mode, vlasovSolver21_spline.hxx:680-801):
//   scan      radial moment partials -> bins -> enclosed mass -> kick shift
//   ucol      per (J slice, strip of r columns): natural-BC spline solve along
//             u, kick gather at U+shift(r), second solve along u of the kicked
//             values -> G (u-direction coefficients of the kicked f)
//   prer      per (J slice, rows of G): solve along r -> C (2D coefficients)
//   drift     per cell: 4x4 gather of C at the host-tabulated footpoint, or the
//             delayed-kernel ring-buffer front, or 0; radial moment partials
//             of the result (the next step's moment) in the epilogue
//   tails     per delayed-kernel chain: spline value at the chain tail
//
// The 2D prefilter of the reference (r-solves, then u-solves on every column,
// localSpline.hxx:1238-1258) is applied here as u-solves then r-solves; the
// tensor-product operator is the same.  The Thomas recursion of one line
// (localSpline.hxx:953-1182) is split into segments that run in parallel:
// each segment first replays K rows of the recursion before its start (the
// forward and backward recursions contract by 2-sqrt(3) = 0.268 per row, so
// K = 32 rows reach FP64 rounding and K = 20 rows reach 1e-11).  The per-row
// coefficients are the reference's own (tabulated on the host in its
// operation order).  Recursions run in FP64 in both precisions.
#include <cstdio>
#include <cstdlib>

#include "vls_async.cuh"
#include "vls_dd.cuh"
#include "vls_internal.h"

namespace vls {

// warm-up rows of a segment: FP64 storage needs the recursion to contract to
// FP64 rounding (0.268^32 = 5e-19), FP32 storage to well below FP32 rounding
// (0.268^16 = 7e-10)
template <typename T>
struct Prec;
template <>
struct Prec<double> {
  static constexpr int K = 32;
};
template <>
struct Prec<float> {
  static constexpr int K = 16;
};

template <typename T>
__device__ __forceinline__ T bv2(T x) {
  return x * x * x;
}
template <typename T>
__device__ __forceinline__ T bv1(T x) {
  return T(1) + T(3) * x + T(3) * x * x - T(3) * x * x * x;
}

// s / 36 without the bias of a rounded 1/36 factor: in FP32 the constant is
// split in two floats (hi + lo = 1/36 to 1e-17), so the product carries only
// the final rounding.  A biased factor would scale every drifted value the
// same way in every step and show up as a steady mass drift.
template <typename T>
__device__ __forceinline__ T over36(T s) {
  return s * (T(1) / T(36));
}
template <>
__device__ __forceinline__ float over36<float>(float s) {
  return __fmaf_rn(s, 0.02777777798473835f, s * -2.0696057367874943e-10f);
}

// ----------------------------------------------------------- async copies
// cp.async (LDGSTS): element-wise global -> shared copies that stay in flight
// together; the tiles' global rows are only 4-byte aligned (r-pitch N_r).
template <typename T>
__device__ __forceinline__ void cp_async(T *smem, const T *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem),
               "n"((int)sizeof(T))
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ----------------------------------------------------------- segment solve
// One line of the padded natural-BC system lives at b[k*ks], k = 0..M-1.  On
// entry rows 1..M-2 hold the data; on exit rows 0..M-1 hold the coefficients.
// A thread owns interior rows [k0, k1).  The four stages are separated by
// __syncthreads() (see solve_lines).  R is the arithmetic of the recursion.
// The per-row coefficients rp_k, q_k are read from shared memory for rows
// below kc and replaced by their limits from row kc on (they are equal there
// in the recursion's precision), which removes two shared loads per element.
template <typename R>
struct Coef {
  const R *rp, *q;
  R rpi, qi, sixth;
  int kc;
  __device__ __forceinline__ R rpk(int k) const { return k < kc ? rp[k] : rpi; }
  __device__ __forceinline__ R qk(int k) const { return k < kc ? q[k] : qi; }
};

template <int K, typename R>
struct Seg {
  template <typename S>
  __device__ __forceinline__ static R fwd_warm(const S *b, int ks, int k0, const Coef<R> &cf) {
    R d = R(0);
    int ks0 = k0 - K;
    if (ks0 < 1) ks0 = 1;
#pragma unroll 4
    for (int k = ks0; k < k0; ++k) d = ((R)b[k * ks] - d * cf.sixth) * cf.rpk(k);
    return d;
  }
  template <typename S>
  __device__ __forceinline__ static void fwd_main(S *b, int ks, int k0, int k1, R d,
                                  const DirTables &t, const Coef<R> &cf) {
    R dprev = d;
    int k = k0;
    const int kt = min(k1, max(k0, cf.kc));
#pragma unroll 4
    for (; k < kt; ++k) {
      dprev = d;
      d = ((R)b[k * ks] - d * cf.sixth) * cf.rp[k];
      b[k * ks] = (S)d;
    }
#pragma unroll 4
    for (; k < k1; ++k) {
      dprev = d;
      d = ((R)b[k * ks] - d * cf.sixth) * cf.rpi;
      b[k * ks] = (S)d;
    }
    if (k1 == t.M - 1 && k1 > k0) {
      // last row (localSpline.hxx:1145-1152): d = d_{M-2}, dprev = d_{M-3}
      const R num = (R(0) - (R)t.hi2 * dprev) - (R)t.L1 * d;
      b[(t.M - 1) * ks] = (S)(num / (R)t.L2);
    }
  }
  template <typename S>
  __device__ __forceinline__ static R bwd_warm(const S *b, int ks, int k1, const DirTables &t,
                               const Coef<R> &cf) {
    int kst = k1 + K - 1;
    R c;
    if (kst >= t.M - 2) {
      kst = t.M - 2;
      c = (R)b[(t.M - 1) * ks];
    } else {
      c = R(0);
    }
#pragma unroll 4
    for (int k = kst; k >= k1; --k) c = (R)b[k * ks] - cf.qk(k) * c;
    return c;
  }
  template <typename S>
  __device__ __forceinline__ static void bwd_main(S *b, int ks, int k0, int k1, R c,
                                  const DirTables &t, const Coef<R> &cf) {
    R cnext = c;
    int k = k1 - 1;
    const int kt = max(k0, cf.kc);
#pragma unroll 4
    for (; k >= kt; --k) {
      cnext = c;
      c = (R)b[k * ks] - cf.qi * c;
      b[k * ks] = (S)c;
    }
#pragma unroll 4
    for (; k >= k0; --k) {
      cnext = c;
      c = (R)b[k * ks] - cf.q[k] * c;
      b[k * ks] = (S)c;
    }
    if (k0 == 1 && k1 > k0) {
      // first row (localSpline.hxx:1171): c_0 = (0 - a01 c_1) - a02 c_2
      b[0] = (S)((R(0) - (R)t.a01 * c) - (R)t.a02 * cnext);
    }
  }
};

// segment bounds: interior rows [1, M-1) split into nseg pieces of odd length
__device__ __forceinline__ void seg_bounds(int M, int nseg, int s, int &k0,
                                           int &k1) {
  int n = M - 2;
  int L = (n + nseg - 1) / nseg;
  L |= 1;
  k0 = 1 + s * L;
  k1 = k0 + L;
  if (k0 > M - 1) k0 = M - 1;
  if (k1 > M - 1) k1 = M - 1;
}

// rp, q: the direction's tables in the recursion type (shared memory)
template <int K, typename R, typename S>
__device__ __forceinline__ void solve_lines(S *base, int ks, int k0, int k1,
                            const DirTables &t, const R *rp, const R *q) {
  Coef<R> cf;
  cf.rp = rp;
  cf.q = q;
  cf.rpi = (R)t.rp_inf;
  cf.qi = (R)t.q_inf;
  cf.sixth = R(1) / R(6);
  cf.kc = sizeof(R) == 4 ? t.kc32 : t.kc64;
  R d = Seg<K, R>::fwd_warm(base, ks, k0, cf);
  __syncthreads();
  Seg<K, R>::fwd_main(base, ks, k0, k1, d, t, cf);
  __syncthreads();
  R c = Seg<K, R>::bwd_warm(base, ks, k1, t, cf);
  __syncthreads();
  Seg<K, R>::bwd_main(base, ks, k0, k1, c, t, cf);
  __syncthreads();
}

// copies the direction's Thomas tables into shared memory as type R
template <typename R>
__device__ __forceinline__ void load_tables(R *rp, R *q, const DirTables &t) {
  for (int k = threadIdx.x; k < t.M; k += blockDim.x) {
    rp[k] = (R)__ldg(t.rp + k);
    q[k] = (R)__ldg(t.q + k);
  }
}

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) / 16 * 16; }

// ------------------------------------------------------------------ ucol
// Block: TW columns (r) x NSEG segments (u), lane = column, so a shared row
// access by a warp is one (FP32) or two (FP64) wavefronts.  Shared memory:
// the Thomas tables and two buffers of (N_u+3) rows x TW in the recursion
// type R (row N_u+2 is an always-zero guard row); global f and G are type T,
// so T -> R and R -> T conversions happen once per element, at the tile load
// and at the tile store.
constexpr int UC_THREADS = 256;
template <typename R>
struct UcolCfg {
  static constexpr int TW = sizeof(R) == 4 ? 16 : 8;
  static constexpr int NSEG = UC_THREADS / TW;
};

// loads rows 1..nu of a TW-column tile of f (r0.., slice base fs) into buf
template <typename T, typename R, int TW>
__device__ __forceinline__ void load_col_tile(R *buf, const T *__restrict__ fs,
                                              int nu, int nr, int r0) {
  if constexpr (sizeof(T) == sizeof(R)) {
    for (int e = threadIdx.x; e < nu * TW; e += blockDim.x) {
      const int k = e / TW + 1, c = e % TW;
      const int rr = r0 + c;
      if (rr < nr)
        cp_async(reinterpret_cast<T *>(&buf[k * TW + c]), fs + (size_t)(k - 1) * nr + rr);
      else
        buf[k * TW + c] = R(0);
    }
    cp_async_wait_all();
  } else {
    // four loads in flight per thread, then convert
    const int n = nu * TW;
    for (int e0 = threadIdx.x; e0 < n; e0 += 4 * blockDim.x) {
      T v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = e0 + q * blockDim.x;
        const int k = e / TW + 1, c = e % TW, rr = r0 + c;
        v[q] = (e < n && rr < nr) ? __ldg(fs + (size_t)(k - 1) * nr + rr) : T(0);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = e0 + q * blockDim.x;
        if (e < n) buf[(e / TW + 1) * TW + e % TW] = (R)v[q];
      }
    }
  }
}

// exact per-cell kick index computation (vlasovSolver21_spline.hxx:760-762,
// localSpline.hxx:426-429), used where the column's fractional shift lies
// within 1e-9 of a node
template <typename R, int TW>
__device__ __forceinline__ R kick_exact(const R *cb, const Geometry &g, int u,
                                        double s) {
  const double newU = __ldg(g.U + u) + s;
  if (!(newU > g.u0 && newU < g.umax)) return R(0);  // outside (or NaN) -> 0
  const double y = (newU - g.su) * g.hu;
  const double fl = floor(y);
  const R fr = (R)(y - fl);
  const int Ny = 1 + (int)fl;
  return (bv2<R>(R(1) - fr) * cb[(Ny - 1) * TW] + bv1<R>(R(1) - fr) * cb[Ny * TW] +
          bv1<R>(fr) * cb[(Ny + 1) * TW] + bv2<R>(fr) * cb[(Ny + 2) * TW]) /
         R(6);
}

// TW columns per block (UcolCfg<R>::TW, or half of it where two buffers of
// that many long columns exceed a block's shared memory)
template <typename T, typename R, bool KICK, int TW>
__global__ void __launch_bounds__(UC_THREADS)
    ucol_kernel(const T *__restrict__ f, T *__restrict__ G,
                const double *__restrict__ shift, Geometry g, DirTables tu) {
  constexpr int NSEG = UC_THREADS / TW;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int M = g.nu + 2;
  const int rows = M + 1;
  R *rp = reinterpret_cast<R *>(smem_raw);
  R *qq = rp + M;
  R *bufA = reinterpret_cast<R *>(smem_raw + align16(2 * M * sizeof(R)));
  R *bufB = bufA + (size_t)rows * TW;
  const int tid = threadIdx.x;
  const int col = tid % TW;
  const int seg = tid / TW;
  const int r0 = blockIdx.x * TW;
  const int jl = blockIdx.y;        // slice within the batch (scratch index)
  const int j = g.j0 + jl;          // global slice
  const int r = r0 + col;

  load_tables<R>(rp, qq, tu);
  if (tid < TW) {
    bufA[0 * TW + tid] = R(0);
    bufA[(M - 1) * TW + tid] = R(0);
    bufA[M * TW + tid] = R(0);
    bufB[0 * TW + tid] = R(0);
    bufB[(M - 1) * TW + tid] = R(0);
    bufB[M * TW + tid] = R(0);
  }
  load_col_tile<T, R, TW>(bufA, f + (size_t)j * g.nu * g.nr, g.nu, g.nr, r0);
  __syncthreads();
  int k0, k1;
  seg_bounds(M, NSEG, seg, k0, k1);
  solve_lines<Prec<T>::K, R>(bufA + col, TW, k0, k1, tu, rp, qq);

  R *out = bufA;
  if (KICK) {
    // kick (vlasovSolver21_spline.hxx:758-763, localSpline.hxx:423-441 with
    // the r-direction (1,4,1)/6 weights folded into the u-only coefficients).
    // The shift is constant along the column and the u grid is uniform, so
    // y_u = u + s*hu: one fraction and one integer offset serve every row,
    // unless that fraction is within 1e-9 of a node (then every row takes
    // the exact per-cell path).
    const double s = (r < g.nr) ? __ldg(shift + r) : 0.0;
    const double qf = s * g.hu;
    const double fl = floor(qf);
    const double frd = qf - fl;
    const bool fast = frd > 1e-9 && frd < 1.0 - 1e-9 && fabs(qf) < 1e6;
    const int o = fast ? (int)fl : 0;
    const R fr = (R)frd;
    const R w0 = bv2<R>(R(1) - fr) / R(6), w1 = bv1<R>(R(1) - fr) / R(6);
    const R w2 = bv1<R>(fr) / R(6), w3 = bv2<R>(fr) / R(6);
    // rows with 0 < u + qf < nu - 1 are inside (strictly, as :761)
    const int ulo = fast ? (int)floor(-qf) + 1 : 0;
    const int uhi = fast ? (int)ceil((double)(g.nu - 1) - qf) - 1 : -1;
    const R *cb = bufA + col;
    if (fast) {
#pragma unroll 4
      for (int k = k0; k < k1; ++k) {
        const int u = k - 1;
        R v = R(0);
        if (u >= ulo && u <= uhi) {
          const R *p = cb + (k + o - 1) * TW;
          v = w0 * p[0] + w1 * p[TW] + w2 * p[2 * TW] + w3 * p[3 * TW];
        }
        bufB[k * TW + col] = v;
      }
    } else {
      for (int k = k0; k < k1; ++k) bufB[k * TW + col] = kick_exact<R, TW>(cb, g, k - 1, s);
    }
    __syncthreads();
    solve_lines<Prec<T>::K, R>(bufB + col, TW, k0, k1, tu, rp, qq);
    out = bufB;
  }
  T *Gs = G + (size_t)jl * M * g.gp;
  for (int e = tid; e < M * TW; e += UC_THREADS) {
    const int k = e / TW, c = e % TW;
    const int rr = r0 + c;
    if (rr < g.nr) Gs[(size_t)k * g.gp + rr] = (T)out[k * TW + c];
  }
}

template <typename T, typename R>
cudaError_t launch_ucol(bool kick, const T *f, T *G, const double *shift,
                        const Geometry &g, const DirTables &tu, cudaStream_t st) {
  constexpr int TW = UcolCfg<R>::TW;
  auto smem_for = [&](int tw) {
    return align16(2 * (size_t)(g.nu + 2) * sizeof(R)) + 2 * (size_t)(g.nu + 3) * tw * sizeof(R);
  };
  auto go = [&](auto kern, int tw) {
    const size_t smem = smem_for(tw);
    dim3 grid((g.nr + tw - 1) / tw, g.nb);
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, UC_THREADS, smem, st>>>(f, G, shift, g, tu);
    return cudaGetLastError();
  };
  // 227 KB per block: FP64 columns of more than ~1600 rows take half the columns
  if (smem_for(TW) > 232448)
    return kick ? go(ucol_kernel<T, R, true, TW / 2>, TW / 2)
                : go(ucol_kernel<T, R, false, TW / 2>, TW / 2);
  return kick ? go(ucol_kernel<T, R, true, TW>, TW) : go(ucol_kernel<T, R, false, TW>, TW);
}

// ------------------------------------------------------------------ prer
// Block: ROWS rows of G (lane = row) x NSEG long segments along r.  The
// shared row pitch is 1 mod 32 (FP32) or odd (FP64) so that the lanes, which
// walk different rows at the same column, hit distinct banks.  Shared rows
// are in the recursion type R.
template <typename R>
struct PrerCfg {
  static constexpr int ROWS = sizeof(R) == 4 ? 32 : 16;
  static constexpr int NSEG = 8;
  static constexpr int THREADS = ROWS * NSEG;
};

__host__ __device__ inline int prer_pitch(int M, int elem) {
  int P = M + 1;
  if (elem == 4)
    P = (P + 31) / 32 * 32 + 1;
  else
    P |= 1;
  return P;
}

// ROWS rows of G per block (PrerCfg<R>::ROWS, or half of it where a tile of
// that many long rows exceeds a block's shared memory)
template <typename T, typename R, int ROWS>
__global__ void __launch_bounds__(ROWS * PrerCfg<R>::NSEG)
    prer_kernel(const T *__restrict__ G, T *__restrict__ C, Geometry g,
                DirTables tr) {
  constexpr int NSEG = PrerCfg<R>::NSEG, NT = ROWS * NSEG;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int M = g.nr + 2;
  const int LS = prer_pitch(M, sizeof(R));
  R *rp = reinterpret_cast<R *>(smem_raw);
  R *qq = rp + M;
  R *buf = reinterpret_cast<R *>(smem_raw + align16(2 * M * sizeof(R)));
  const int tid = threadIdx.x;
  const int rho = tid % ROWS;
  const int seg = tid / ROWS;
  const int j = blockIdx.y;  // slice within the batch (G and C are batch scratch)
  const int kr0 = blockIdx.x * ROWS;
  const int nrows = g.nu + 2;
  const T *Gs = G + (size_t)j * nrows * g.gp;
  load_tables<R>(rp, qq, tr);
  // rows of the tile, each copied by the whole block (no index division)
  for (int p = 0; p < ROWS; ++p) {
    const int kr = kr0 + p;
    R *dst = buf + p * LS + 1;
    if (kr < nrows) {
      const T *src = Gs + (size_t)kr * g.gp;
      if constexpr (sizeof(T) == sizeof(R)) {
        for (int k = tid; k < g.nr; k += NT) cp_async(reinterpret_cast<T *>(dst + k), src + k);
      } else {
        for (int k = tid; k < g.nr; k += NT) dst[k] = (R)__ldg(src + k);
      }
    } else {
      for (int k = tid; k < g.nr; k += NT) dst[k] = R(0);
    }
  }
  if constexpr (sizeof(T) == sizeof(R)) cp_async_wait_all();
  __syncthreads();
  int k0, k1;
  seg_bounds(M, NSEG, seg, k0, k1);
  solve_lines<Prec<T>::K, R>(buf + rho * LS, 1, k0, k1, tr, rp, qq);
  T *Cs = C + (size_t)j * (g.nu + 3) * g.pc;
  for (int p = 0; p < ROWS; ++p) {
    const int kr = kr0 + p;
    if (kr >= nrows) break;
    T *dst = Cs + (size_t)kr * g.pc;
    const R *src = buf + p * LS;
    for (int k = tid; k < M; k += NT) dst[k] = (T)src[k];
  }
}

template <typename T, typename R>
cudaError_t launch_prer(const T *G, T *C, const Geometry &g, const DirTables &tr,
                        cudaStream_t st) {
  constexpr int ROWS = PrerCfg<R>::ROWS, NSEG = PrerCfg<R>::NSEG;
  const int M = g.nr + 2;
  auto smem_for = [&](int rows) {
    return align16(2 * (size_t)M * sizeof(R)) +
           (size_t)rows * prer_pitch(M, sizeof(R)) * sizeof(R);
  };
  // 227 KB per block: FP64 rows of more than ~1600 columns take half the rows
  if (smem_for(ROWS) > 232448) {
    constexpr int H = ROWS / 2;
    const size_t smem = smem_for(H);
    dim3 grid((g.nu + 2 + H - 1) / H, g.nb);
    cudaError_t e = cudaFuncSetAttribute(
        prer_kernel<T, R, H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    prer_kernel<T, R, H><<<grid, H * NSEG, smem, st>>>(G, C, g, tr);
    return cudaGetLastError();
  }
  const size_t smem = smem_for(ROWS);
  dim3 grid((g.nu + 2 + ROWS - 1) / ROWS, g.nb);
  cudaError_t e = cudaFuncSetAttribute(
      prer_kernel<T, R, ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  prer_kernel<T, R, ROWS><<<grid, ROWS * NSEG, smem, st>>>(G, C, g, tr);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ gather
// localSpline::evaluateC(int,double,int,double), localSpline.hxx:381-398:
// taps at padded columns rI..rI+3 and rows uI..uI+3 (FP64 form).
template <typename T>
__device__ __forceinline__ T eval2d(const T *__restrict__ Cj, int pc, int rI,
                                    T x, int uI, T y) {
  const T b2xI = bv2<T>(T(1) - x), b1xI = bv1<T>(T(1) - x);
  const T b1x = bv1<T>(x), b2x = bv2<T>(x);
  const T *p = Cj + (size_t)uI * pc + rI;
  const T s0 = __ldg(p) * b2xI + __ldg(p + 1) * b1xI + __ldg(p + 2) * b1x +
               __ldg(p + 3) * b2x;
  p += pc;
  const T s1 = __ldg(p) * b2xI + __ldg(p + 1) * b1xI + __ldg(p + 2) * b1x +
               __ldg(p + 3) * b2x;
  p += pc;
  const T s2 = __ldg(p) * b2xI + __ldg(p + 1) * b1xI + __ldg(p + 2) * b1x +
               __ldg(p + 3) * b2x;
  p += pc;
  const T s3 = __ldg(p) * b2xI + __ldg(p + 1) * b1xI + __ldg(p + 2) * b1x +
               __ldg(p + 3) * b2x;
  return over36<T>(bv2<T>(T(1) - y) * s0 + bv1<T>(T(1) - y) * s1 +
                           bv1<T>(y) * s2 + bv2<T>(y) * s3);
}

// FP32 form with packed f32x2 arithmetic: the x and y weights are computed
// pairwise, and rows (0,1) and (2,3) are accumulated pairwise.
//
// Difference form: with c the tap at (row 1, column 1), the value is
// c + (1/36) sum w_x w_y (C - c), which equals (1/36) sum w_x w_y C because
// the cubic B-spline weights of each direction sum to 6.  In FP32 the
// rounded weights do not sum to 6 exactly and the rounding of the 16 products
// is proportional to C; both errors are the same in every step of a nearly
// stationary state (the footpoints, hence the weights, never change), so
// they add up coherently over thousands of steps.  Taken on the differences
// C - c, which are small where f is smooth, they shrink by the same factor:
// over 2000 steps of the Plummer 257 x 257 x 128 case the energy drift of the
// FP32 path moves from 1.7e-6 to 1.5e-7 off the FP64 path's.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// tap (a, b) = row a, column b of the 4 x 4 block, from ld(a, b)
template <class Ld>
__device__ __forceinline__ float gather_f32x2(const Ld &ld, float x, float y) {
  const float2 t = f2(x, y);
  const float2 one = f2(1.f, 1.f), three = f2(3.f, 3.f), m3 = f2(-3.f, -3.f);
  const float2 sv = __fadd2_rn(one, f2(-t.x, -t.y));  // 1 - t
  const float2 t2 = __fmul2_rn(t, t), t3 = __fmul2_rn(t2, t);
  const float2 s2 = __fmul2_rn(sv, sv), s3 = __fmul2_rn(s2, sv);
  // BV1(v) = 1 + 3v + 3v^2 - 3v^3
  const float2 a1 = __ffma2_rn(m3, s3, __ffma2_rn(three, s2, __ffma2_rn(three, sv, one)));
  const float2 b1 = __ffma2_rn(m3, t3, __ffma2_rn(three, t2, __ffma2_rn(three, t, one)));
  // x weights: (s3.x, a1.x, b1.x, t3.x); y weights: (s3.y, a1.y, b1.y, t3.y)
  const float2 wx0 = f2(s3.x, s3.x), wx1 = f2(a1.x, a1.x), wx2 = f2(b1.x, b1.x),
               wx3 = f2(t3.x, t3.x);
  const float c = ld(1, 1);
  const float2 mc = f2(-c, -c);
  float2 r01 = __fmul2_rn(__fadd2_rn(f2(ld(0, 0), ld(1, 0)), mc), wx0);
  r01 = __ffma2_rn(__fadd2_rn(f2(ld(0, 1), c), mc), wx1, r01);
  r01 = __ffma2_rn(__fadd2_rn(f2(ld(0, 2), ld(1, 2)), mc), wx2, r01);
  r01 = __ffma2_rn(__fadd2_rn(f2(ld(0, 3), ld(1, 3)), mc), wx3, r01);
  float2 r23 = __fmul2_rn(__fadd2_rn(f2(ld(2, 0), ld(3, 0)), mc), wx0);
  r23 = __ffma2_rn(__fadd2_rn(f2(ld(2, 1), ld(3, 1)), mc), wx1, r23);
  r23 = __ffma2_rn(__fadd2_rn(f2(ld(2, 2), ld(3, 2)), mc), wx2, r23);
  r23 = __ffma2_rn(__fadd2_rn(f2(ld(2, 3), ld(3, 3)), mc), wx3, r23);
  // y weights (rows 0..3) applied pairwise, times 1/36
  const float2 acc = __ffma2_rn(r23, f2(b1.y, t3.y), __fmul2_rn(r01, f2(s3.y, a1.y)));
  return c + over36<float>(acc.x + acc.y);
}

// from C in global memory (row pitch pc), taps from Cj + off
__device__ __forceinline__ float eval2d_f32x2(const float *__restrict__ Cj, int pc,
                                              int off, float x, float y) {
  const float *p = Cj + off;
  return gather_f32x2([&](int a, int b) { return __ldg(p + a * pc + b); }, x, y);
}

// FP32 storage: every gather in the difference form
template <>
__device__ __forceinline__ float eval2d<float>(const float *__restrict__ Cj, int pc, int rI,
                                               float x, int uI, float y) {
  return eval2d_f32x2(Cj, pc, uI * pc + rI, x, y);
}

constexpr int DR_W = 8;  // warps per drift block

// FP32 tables, 8 bytes per cell: word = index << FP_FBITS | round(frac * 2^FP_FBITS)
// per direction; FP_OUT / FP_CHAIN in the first word mark the two special kinds
// (the second word then holds the chain id).  The 21 fraction bits are placed
// straight into a float mantissa (value 1.frac, minus 1): no int->float convert.
constexpr int FP_FBITS = 21;
constexpr uint32_t FP_FMASK = (1u << FP_FBITS) - 1u;
constexpr uint32_t FP_OUT = 0xFFFFFFFFu, FP_CHAIN = 0xFFFFFFFEu;

__device__ __forceinline__ float frac21(uint32_t w) {
  return __uint_as_float(0x3F800000u | ((w & FP_FMASK) << 2)) - 1.0f;
}

// ------------------------------------------------------- TMA-staged drift
// Most drift footpoints lie within a few cells of their own node, so each
// block (a strip of 32 r columns of one J slice) walks down the rows in
// chunks of DW_CH and has the tensor-memory accelerator bring the matching
// DW_ROWS x DW_COLS window of the coefficient slice into shared memory,
// double buffered and signalled through an mbarrier.  Taps inside the window
// are read from shared memory; footpoints outside it (far displacements) read
// the coefficients from global memory.  Every mbarrier wait is bounded: on
// timeout the block records an error flag and falls back to global reads.
constexpr int DW_COLS = 64, DW_ROWS = 40, DW_CH = 16, DW_XOFF = 16, DW_YOFF = 12;
constexpr int DT_THREADS = 256;  // 8 warps x 32 columns; 2 rows per warp per chunk
template <typename T>
struct Cell {
  int rI, uI, kind;
  uint32_t ch;
  T x, y;
};

// Footpoint words as loaded (decoded only where the cell is computed, so that
// prefetched loads stay in flight)
template <typename T>
struct RawCell;
template <>
struct RawCell<float> {
  uint2 w;
};
template <>
struct RawCell<double> {
  int code;
  double x, y;
};
__device__ __forceinline__ RawCell<float> load_raw(const int32_t *, const float *,
                                                   const float *,
                                                   const uint2 *__restrict__ fp2, size_t i) {
  RawCell<float> c;
  c.w = __ldg(fp2 + i);
  return c;
}
__device__ __forceinline__ RawCell<double> load_raw(const int32_t *__restrict__ idx,
                                                    const double *__restrict__ fx,
                                                    const double *__restrict__ fy,
                                                    const uint2 *, size_t i) {
  RawCell<double> c;
  c.code = __ldg(idx + i);
  c.x = __ldg(fx + i);
  c.y = __ldg(fy + i);
  return c;
}
// kinds: 0 gather, 1 outside (0), 2 delayed-kernel chain front
__device__ __forceinline__ Cell<float> decode(const RawCell<float> &r) {
  Cell<float> c;
  const uint2 w = r.w;
  const bool ok = w.x < FP_CHAIN;
  c.kind = ok ? 0 : (w.x == FP_OUT ? 1 : 2);
  c.ch = w.y;
  c.rI = ok ? (int)(w.x >> FP_FBITS) : 0;
  c.uI = ok ? (int)(w.y >> FP_FBITS) : 0;
  c.x = frac21(w.x);
  c.y = frac21(w.y);
  return c;
}
__device__ __forceinline__ Cell<double> decode(const RawCell<double> &r) {
  Cell<double> c;
  const int code = r.code;
  c.kind = code >= 0 ? 0 : (code == -1 ? 1 : 2);
  c.ch = (uint32_t)(-2 - code);
  c.rI = code >= 0 ? (code & 0xffff) : 0;
  c.uI = code >= 0 ? (code >> 16) : 0;
  c.x = code >= 0 ? r.x : 0.0;
  c.y = code >= 0 ? r.y : 0.0;
  return c;
}

// 4x4 gather from a shared window row-pitched DW_COLS (immediate offsets)
template <typename T>
__device__ __forceinline__ T eval_window(const T *p, T x, T y) {
  const T b2xI = bv2<T>(T(1) - x), b1xI = bv1<T>(T(1) - x);
  const T b1x = bv1<T>(x), b2x = bv2<T>(x);
  const T s0 = p[0] * b2xI + p[1] * b1xI + p[2] * b1x + p[3] * b2x;
  const T s1 = p[DW_COLS] * b2xI + p[DW_COLS + 1] * b1xI + p[DW_COLS + 2] * b1x +
               p[DW_COLS + 3] * b2x;
  const T s2 = p[2 * DW_COLS] * b2xI + p[2 * DW_COLS + 1] * b1xI +
               p[2 * DW_COLS + 2] * b1x + p[2 * DW_COLS + 3] * b2x;
  const T s3 = p[3 * DW_COLS] * b2xI + p[3 * DW_COLS + 1] * b1xI +
               p[3 * DW_COLS + 2] * b1x + p[3 * DW_COLS + 3] * b2x;
  return over36<T>(bv2<T>(T(1) - y) * s0 + bv1<T>(T(1) - y) * s1 +
                           bv1<T>(y) * s2 + bv2<T>(y) * s3);
}
template <>
__device__ __forceinline__ float eval_window<float>(const float *p, float x, float y) {
  return gather_f32x2([&](int a, int b) { return p[a * DW_COLS + b]; }, x, y);
}

template <typename T>
__global__ void __launch_bounds__(DT_THREADS)
    drift_tma_kernel(const __grid_constant__ CUtensorMap tmC, const T *__restrict__ C,
                     T *__restrict__ f, const int32_t *__restrict__ idx,
                     const T *__restrict__ fx, const T *__restrict__ fy,
                     const uint2 *__restrict__ fp2, const int64_t *__restrict__ ch_start,
                     const int32_t *__restrict__ ch_len, const T *__restrict__ ch_val,
                     int64_t ndrift, MomentTables mt, double *__restrict__ partial,
                     unsigned int *err, uint32_t spins, Geometry g) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T *win = reinterpret_cast<T *>(smem_raw);  // two windows
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + 2 * DW_COLS * DW_ROWS * sizeof(T));
  __shared__ double red[DT_THREADS / 32][32];
  constexpr uint32_t BYTES = DW_COLS * DW_ROWS * sizeof(T);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int r0 = blockIdx.x * 32, r = r0 + lane;
  const int jl = blockIdx.y, j = g.j0 + jl;  // batch-local / global slice
  const int nch = (g.nu + DW_CH - 1) / DW_CH;
  const int x0 = r0 - DW_XOFF;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
    for (int c = 0; c < 2 && c < nch; ++c) {
      mbar_expect_tx(&bar[c], BYTES);
      tma_load_3d(win + c * DW_COLS * DW_ROWS, &tmC, x0, c * DW_CH - DW_YOFF, jl, &bar[c]);
    }
  }
  __syncthreads();
  const T *Cj = C + (size_t)jl * (g.nu + 3) * g.pc;
  const size_t row0 = (size_t)j * g.nu * g.nr + r;
  const bool col_ok = r < g.nr;
  RawCell<T> nxt[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int u = w + 8 * q;
    nxt[q] = load_raw(idx, fx, fy, fp2, row0 + (size_t)(u < g.nu && col_ok ? u : 0) * g.nr);
  }
  double acc = 0.0;
  // copy bookkeeping (meaningful in thread 0, which issues every copy): the
  // chunk last sent to each buffer and whether its completion was observed
  int last0 = 0, last1 = 1;                   // chunk last sent to buffer 0 / 1
  unsigned pending = 1u | (nch > 1 ? 2u : 0u);  // bit b: buffer b's copy not yet seen
  bool issuing = true;
  for (int c = 0; c < nch; ++c) {
    const RawCell<T> cur[2] = {nxt[0], nxt[1]};
    if (c + 1 < nch) {
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int u = (c + 1) * DW_CH + w + 8 * q;
        nxt[q] = load_raw(idx, fx, fy, fp2, row0 + (size_t)(u < g.nu && col_ok ? u : 0) * g.nr);
      }
    }
    const int b = c & 1;
    // after one failed wait this thread waits no more (it reads C globally)
    const bool have = issuing && mbar_wait_bounded(&bar[b], (uint32_t)((c >> 1) & 1), spins);
    if (have) pending &= ~(1u << b);
    if (!have && issuing) {
      issuing = false;  // never stack a second copy onto an unfinished one
      atomicOr(err, 1u);
    }
    const T *wb = win + b * DW_COLS * DW_ROWS;
    const int y0 = c * DW_CH - DW_YOFF;
    T part = T(0);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int u = c * DW_CH + w + 8 * q;
      if (u < g.nu && col_ok) {
        const Cell<T> cl = decode(cur[q]);
        T v = T(0);
        if (cl.kind == 0) {
          const int wr = cl.uI - y0, wc = cl.rI - x0;
          if (have && wr >= 0 && wr <= DW_ROWS - 4 && wc >= 0 && wc <= DW_COLS - 4)
            v = eval_window<T>(wb + wr * DW_COLS + wc, cl.x, cl.y);
          else
            v = eval2d<T>(Cj, g.pc, cl.rI, cl.x, cl.uI, cl.y);
        } else if (cl.kind == 2) {
          const int L = __ldg(ch_len + cl.ch);
          v = ch_val[__ldg(ch_start + cl.ch) + ndrift % L];
        }
        f[row0 + (size_t)u * g.nr] = v;
        part += (T)__ldg(mt.bu + u) * v;
      }
    }
    acc += (double)part;
    __syncthreads();  // every warp is done with window b
    if (tid == 0 && issuing && c + 2 < nch) {
      fence_proxy_async();
      mbar_expect_tx(&bar[b], BYTES);
      tma_load_3d(win + b * DW_COLS * DW_ROWS, &tmC, x0, (c + 2) * DW_CH - DW_YOFF, jl,
                  &bar[b]);
      if (b) last1 = c + 2; else last0 = c + 2;
      pending |= 1u << b;
    }
  }
  // a copy whose wait timed out may still be in flight: wait for it (bounded)
  // before the block's shared memory is released
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      const int lb = b ? last1 : last0;
      if (((pending >> b) & 1u) && lb < nch &&
          !mbar_wait_bounded(&bar[b], (uint32_t)((lb >> 1) & 1)))
        atomicOr(err, 2u);
    }
  }
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0 && col_ok) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < DT_THREADS / 32; ++k) s += red[k][lane];
    partial[(size_t)j * g.nr + r] = __ldg(mt.wj + j) * s;
  }
}

template <typename T>
cudaError_t launch_drift_tma(const CUtensorMap *tmC, const T *C, T *f, const int32_t *idx,
                             const T *fx, const T *fy, const uint2 *fp2,
                             const int64_t *ch_start, const int32_t *ch_len,
                             const T *ch_val, int64_t ndrift, const MomentTables &mt,
                             double *partial, unsigned int *err, uint32_t spins,
                             const Geometry &g, cudaStream_t st) {
  const size_t smem = 2 * DW_COLS * DW_ROWS * sizeof(T) + 2 * sizeof(uint64_t);
  cudaError_t e = cudaFuncSetAttribute(drift_tma_kernel<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((g.nr + 31) / 32, g.nb);
  drift_tma_kernel<T><<<grid, DT_THREADS, smem, st>>>(*tmC, C, f, idx, fx, fy, fp2, ch_start,
                                                       ch_len, ch_val, ndrift, mt, partial,
                                                       err, spins, g);
  return cudaGetLastError();
}

// ------------------------------------------------------------ strip drift
// Block: 32 output columns x every row of one J slice.  The block's whole
// coefficient strip (WC columns starting (WC-32)/2 columns to the left, all
// N_u+3 rows) is staged once by TMA in DS_ROWS-row boxes, one mbarrier per
// box, so a cell can read any row of the strip: the footpoints' u
// displacements reach hundreds of rows while their r displacements stay
// within a few columns.  A cell waits only for the boxes its taps lie in
// (bounded; after a timeout the thread reads C in global memory).  No block
// barrier is taken inside the row loop.  Cells whose taps leave the strip's
// columns gather from global memory.
constexpr int DS_ROWS = 64;

template <typename T, int PITCH>
__device__ __forceinline__ T eval_pitch(const T *p, T x, T y) {
  const T b2xI = bv2<T>(T(1) - x), b1xI = bv1<T>(T(1) - x);
  const T b1x = bv1<T>(x), b2x = bv2<T>(x);
  const T s0 = p[0] * b2xI + p[1] * b1xI + p[2] * b1x + p[3] * b2x;
  const T s1 = p[PITCH] * b2xI + p[PITCH + 1] * b1xI + p[PITCH + 2] * b1x + p[PITCH + 3] * b2x;
  const T s2 = p[2 * PITCH] * b2xI + p[2 * PITCH + 1] * b1xI + p[2 * PITCH + 2] * b1x +
               p[2 * PITCH + 3] * b2x;
  const T s3 = p[3 * PITCH] * b2xI + p[3 * PITCH + 1] * b1xI + p[3 * PITCH + 2] * b1x +
               p[3 * PITCH + 3] * b2x;
  return over36<T>(bv2<T>(T(1) - y) * s0 + bv1<T>(T(1) - y) * s1 +
                           bv1<T>(y) * s2 + bv2<T>(y) * s3);
}
template <int PITCH>
__device__ __forceinline__ float eval_pitch_f32x2(const float *p, float x, float y) {
  return gather_f32x2([&](int a, int b) { return p[a * PITCH + b]; }, x, y);
}
template <typename T, int PITCH>
__device__ __forceinline__ T eval_strip(const T *p, T x, T y) {
  if constexpr (sizeof(T) == 4)
    return eval_pitch_f32x2<PITCH>(p, x, y);
  else
    return eval_pitch<T, PITCH>(p, x, y);
}

// Footpoint fields needed by the strip's fast path: the gather test and the
// tap position.  For non-gather words the values are unused.
template <typename T>
struct FastFoot {
  bool gather;
  int rI, uI;
  T x, y;
};
__device__ __forceinline__ FastFoot<float> fast_foot(const RawCell<float> &c) {
  FastFoot<float> p;
  p.gather = c.w.x < FP_CHAIN;
  p.rI = (int)(c.w.x >> FP_FBITS);
  p.uI = (int)(c.w.y >> FP_FBITS);
  // both fractions with one packed subtraction of 1 (values 1.frac21)
  const float2 xy = __fadd2_rn(
      make_float2(__uint_as_float(0x3F800000u | ((c.w.x & FP_FMASK) << 2)),
                  __uint_as_float(0x3F800000u | ((c.w.y & FP_FMASK) << 2))),
      make_float2(-1.f, -1.f));
  p.x = xy.x;
  p.y = xy.y;
  return p;
}
__device__ __forceinline__ FastFoot<double> fast_foot(const RawCell<double> &c) {
  FastFoot<double> p;
  p.gather = c.code >= 0;
  p.rI = c.code & 0xffff;
  p.uI = c.code >> 16;
  p.x = c.x;
  p.y = c.y;
  return p;
}

// The in-strip gather of one cell, run for every lane with the tap offset
// zeroed where it does not apply; `slow`: the cell takes strip_slow instead
// (outside, chain front, taps outside the strip's columns, or every cell
// after a failed wait: wcap = 0).
template <typename T, int WC>
__device__ __forceinline__ T strip_fast(const RawCell<T> &c, const T *win, int x0,
                                        uint32_t wcap, bool col_ok, bool &slow) {
  const FastFoot<T> p = fast_foot(c);
  const int wc = p.rI - x0;
  const bool in = col_ok && p.gather && (uint32_t)wc < wcap;
  const int so = in ? p.uI * WC + wc : 0;
  slow = col_ok && !in;
  return eval_strip<T, WC>(win + so, p.x, p.y);
}

// A cell the in-strip gather does not cover: the gather from C in global
// memory, a chain front, or zero outside.
template <typename T>
__device__ __forceinline__ T strip_slow(const RawCell<T> &c, const T *__restrict__ Cj,
                                        const int64_t *__restrict__ ch_start,
                                        const int32_t *__restrict__ ch_len,
                                        const T *__restrict__ ch_val, int64_t ndrift,
                                        const Geometry &g) {
  const Cell<T> cl = decode(c);
  T v = T(0);
  if (cl.kind == 0)
    v = eval2d<T>(Cj, g.pc, cl.rI, cl.x, cl.uI, cl.y);
  else if (cl.kind == 2)
    v = ch_val[__ldg(ch_start + cl.ch) + ndrift % __ldg(ch_len + cl.ch)];
  return v;
}

// One cell of the strip drift once every box has landed (wcap = WC - 3, or 0
// after a failed wait, which sends every cell to the global-memory gather).
// A warp vote sends the rare cells the in-strip gather does not cover through
// the general decode.  Every lane of the warp must call it.
template <typename T, int WC>
__device__ __forceinline__ T strip_cell(const RawCell<T> &c, const T *win, int x0,
                                        uint32_t wcap, bool col_ok, const T *__restrict__ Cj,
                                        const int64_t *__restrict__ ch_start,
                                        const int32_t *__restrict__ ch_len,
                                        const T *__restrict__ ch_val, int64_t ndrift,
                                        const Geometry &g) {
  bool slow;
  T v = strip_fast<T, WC>(c, win, x0, wcap, col_ok, slow);
  if (__any_sync(0xffffffffu, slow))
    if (slow) v = strip_slow<T>(c, Cj, ch_start, ch_len, ch_val, ndrift, g);
  return v;
}

// b_u in the storage type (a copy rounded once on the host for FP32)
template <typename T>
__device__ __forceinline__ T moment_bu(const MomentTables &mt, int u) {
  if constexpr (sizeof(T) == 4)
    return __ldg(mt.bu32 + u);
  else
    return __ldg(mt.bu + u);
}

// The rows of one strip column (lane) for warp w: rows w, w + NW, ...,
// footpoints PF rows ahead in flight.  Offsets are relative to slice j and
// 32-bit; the prefetch runs past the slice's last row into the next slice
// or the tables' padding (FOOT_PAD_ROWS rows and 32 cells), and lanes past
// N_r read the next row's words, which they do not use.
template <typename T, int WC, int NW, int PF>
__device__ __forceinline__ void strip_rows(
    const T *win, int x0, bool waits_ok, bool col_ok, int j, int r, int w,
    const T *__restrict__ Cj, T *__restrict__ f,
    const int32_t *__restrict__ idx, const T *__restrict__ fx, const T *__restrict__ fy,
    const uint2 *__restrict__ fp2, const int64_t *__restrict__ ch_start,
    const int32_t *__restrict__ ch_len, const T *__restrict__ ch_val, int64_t ndrift,
    const MomentTables &mt, const Geometry &g, double &acc) {
  static_assert(NW * PF + 1 <= FOOT_PAD_ROWS, "prefetch reaches past the padding rows");
  const size_t sb = (size_t)j * g.nu * g.nr;
  const int32_t *ids = idx;
  const T *fxs = fx, *fys = fy;
  const uint2 *fps = fp2;
  if constexpr (sizeof(T) == 4)
    fps += sb;
  else {
    ids += sb;
    fxs += sb;
    fys += sb;
  }
  T *fs = f + sb;
  const uint32_t step = (uint32_t)NW * (uint32_t)g.nr;
  const uint32_t ahead = (uint32_t)PF * step;
  const uint32_t wcap = waits_ok ? (uint32_t)(WC - 3) : 0u;
  uint32_t off = (uint32_t)w * (uint32_t)g.nr + (uint32_t)r;
  RawCell<T> q[PF];
#pragma unroll
  for (int k = 0; k < PF; ++k) q[k] = load_raw(ids, fxs, fys, fps, off + k * step);
  int u = w;
  // groups whose PF rows all lie in the slice: the PF in-strip gathers, one
  // warp vote for the group's rare cells, then the stores (an L2 prefetch of
  // the footpoint words further ahead measured 4 % slower)
  for (; u + NW * (PF - 1) < g.nu; u += NW * PF) {
    T v[PF];
    bool slow[PF];
    RawCell<T> c[PF];
    bool any = false;
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      c[k] = q[k];
      q[k] = load_raw(ids, fxs, fys, fps, off + ahead + k * step);
      v[k] = strip_fast<T, WC>(c[k], win, x0, wcap, col_ok, slow[k]);
      any |= slow[k];
    }
    if (__any_sync(0xffffffffu, any)) {
#pragma unroll
      for (int k = 0; k < PF; ++k)
        if (slow[k]) v[k] = strip_slow<T>(c[k], Cj, ch_start, ch_len, ch_val, ndrift, g);
    }
    T part = T(0);
#pragma unroll
    for (int k = 0; k < PF; ++k) {
      if (col_ok) {
        fs[off] = v[k];
        part += moment_bu<T>(mt, u + NW * k) * v[k];
      }
      off += step;
    }
    acc += (double)part;
  }
  // the last, partial group (u is warp-uniform, so the vote in strip_cell
  // sees the whole warp)
  T part = T(0);
#pragma unroll
  for (int k = 0; k < PF; ++k) {
    if (u + NW * k < g.nu) {
      const T v = strip_cell<T, WC>(q[k], win, x0, wcap, col_ok, Cj, ch_start, ch_len, ch_val,
                                    ndrift, g);
      if (col_ok) {
        fs[off] = v;
        part += moment_bu<T>(mt, u + NW * k) * v;
      }
      off += step;
    }
  }
  acc += (double)part;
}

template <typename T, int WC, int NW, int MINB, int PF = 2>
__global__ void __launch_bounds__(32 * NW, MINB)
    drift_strip_kernel(const __grid_constant__ CUtensorMap tmS, const T *__restrict__ C,
                       T *__restrict__ f, const int32_t *__restrict__ idx,
                       const T *__restrict__ fx, const T *__restrict__ fy,
                       const uint2 *__restrict__ fp2, const int64_t *__restrict__ ch_start,
                       const int32_t *__restrict__ ch_len, const T *__restrict__ ch_val,
                       int64_t ndrift, MomentTables mt, double *__restrict__ partial,
                       unsigned int *err, uint32_t spins, int extra, Geometry g) {
  constexpr int XL = (WC - 32) / 2;
  // PF: rows of footpoints in flight per thread.  16 warps with PF = 2 (two
  // blocks per SM) measured fastest on the 513 x 513 x 256 case: drift 0.309
  // ms against 0.318 / 0.361 (PF 3 / 1), 0.319 / 0.327 (12 warps, PF 2 / 3),
  // 0.398 / 0.316 (8 warps, PF 2 / 4)
  constexpr uint32_t BYTES = DS_ROWS * WC * sizeof(T);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ double red[NW][32];
  const int rows = g.nu + 3;
  const int nch = (rows + DS_ROWS - 1) / DS_ROWS;
  T *win = reinterpret_cast<T *>(smem_raw);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + (size_t)nch * BYTES);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int r0 = blockIdx.x * 32, r = r0 + lane;
  const int jl = blockIdx.y, j = g.j0 + jl;
  const int x0 = r0 - XL;
  if (tid == 0) {
    for (int c = 0; c < nch; ++c) mbar_init(&bar[c], 1);
    mbar_fence_init();
    for (int c = 0; c < nch; ++c) {
      mbar_expect_tx(&bar[c], BYTES);
      tma_load_3d(win + (size_t)c * DS_ROWS * WC, &tmS, x0, c * DS_ROWS, jl, &bar[c]);
    }
  }
  __syncthreads();
  const T *Cj = C + (size_t)jl * rows * g.pc;
  const bool col_ok = r < g.nr;
  int ready = 0;  // boxes [0, ready) seen complete by this thread
  bool waits_ok = true;
  // every box before the first cell (the other block on the SM computes
  // meanwhile); `spins` bounds each wait
  for (; ready < nch; ++ready)
    if (!mbar_wait_bounded(&bar[ready], 0u, spins)) {
      waits_ok = false;
      atomicOr(err, 1u);
      break;
    }
  double acc = 0.0;
  strip_rows<T, WC, NW, PF>(win, x0, waits_ok, col_ok, j, r, w, Cj, f, idx, fx, fy, fp2,
                            ch_start, ch_len, ch_val, ndrift, mt, g, acc);
  // extra: the grid has N_r / 32 blocks and N_r = 32 k + 1; the last block
  // also computes the last column from its strip (columns r0 - 8 .. r0 + 39
  // cover it), one row per thread, instead of a block of one column
  double acc2 = 0.0;
  const bool xblock = extra && blockIdx.x == gridDim.x - 1;
  if (xblock) {
    const int rx = r0 + 32;
    for (int u = tid; u < g.nu; u += 32 * NW) {
      const size_t cell = ((size_t)j * g.nu + u) * g.nr + rx;
      const Cell<T> cl = decode(load_raw(idx, fx, fy, fp2, cell));
      T v = T(0);
      if (cl.kind == 0) {
        const int wc = cl.rI - x0;
        bool inwin = waits_ok && wc >= 0 && wc <= WC - 4;
        if (inwin) {
          // every box was awaited above (ready == nch), so these bounded
          // waits never run; without the loop the compiler's register
          // allocation of this kernel spills (40 B a thread, the drift 8 %
          // slower on the 513 x 513 x 256 case)
          const int cb = (cl.uI + 3) / DS_ROWS;
          while (ready <= cb) {
            if (!mbar_wait_bounded(&bar[ready], 0u)) {
              waits_ok = false;
              inwin = false;
              atomicOr(err, 1u);
              break;
            }
            ++ready;
          }
        }
        v = inwin ? eval_strip<T, WC>(win + (size_t)cl.uI * WC + wc, cl.x, cl.y)
                  : eval2d<T>(Cj, g.pc, cl.rI, cl.x, cl.uI, cl.y);
      } else if (cl.kind == 2) {
        const int L = __ldg(ch_len + cl.ch);
        v = ch_val[__ldg(ch_start + cl.ch) + ndrift % L];
      }
      f[cell] = v;
      acc2 += (double)((T)__ldg(mt.bu + u) * v);
    }
  }
  // every box must have landed before the block's shared memory is released
  if (tid == 0) {
    for (int c = 0; c < nch; ++c)
      if (!mbar_wait_bounded(&bar[c], 0u)) atomicOr(err, 2u);
  }
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0 && col_ok) {
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) sum += red[k][lane];
    partial[(size_t)j * g.nr + r] = __ldg(mt.wj + j) * sum;
  }
  if (xblock) {
    // fixed-order reduction of the last column's terms over the block
    __syncthreads();
    red[w][lane] = acc2;
    __syncthreads();
    if (tid == 0) {
      double sum = 0.0;
      for (int k = 0; k < NW; ++k)
        for (int l = 0; l < 32; ++l) sum += red[k][l];
      partial[(size_t)j * g.nr + r0 + 32] = __ldg(mt.wj + j) * sum;
    }
  }
}

// Strip layouts (the DRIFT_* kinds): DRIFT_STRIP2, 48 columns, 16 warps, two
// blocks per SM; DRIFT_STRIP1, 48 columns, 32 warps, one block per SM;
// DRIFT_WINDOW: none, the windowed kernel.  `want` != DRIFT_AUTO asks for
// one kind, returned only if it fits (else DRIFT_WINDOW).  The default for
// FP32 storage is DRIFT_STRIP2 where it fits (4 % faster than per-cell box
// waits on the 513 x 513 x 256 case: the other block on the SM computes while
// this one's strip lands), else DRIFT_STRIP1 (strips of up to 1028 rows:
// 14 % faster than the windowed drift on 1025 x 1025 x 512), else the
// windowed kernel; FP64 takes the windowed kernel (its strips fit one block
// per SM only, which measured slower).
template <typename T>
int drift_strip_width(int nu, int want) {
  const int nch = (nu + 3 + DS_ROWS - 1) / DS_ROWS;
  if (nch > 32 || want == DRIFT_WINDOW) return DRIFT_WINDOW;
  auto dyn = [&](int wc) { return (size_t)nch * (DS_ROWS * wc * sizeof(T) + sizeof(uint64_t)); };
  // 228 KB of shared memory per SM, 1 KB of it reserved per block; at most
  // 227 KB per block; static reduction array NW x 32 doubles
  const bool fit2 = 2 * (dyn(48) + 16 * 32 * 8 + 1024) <= 233472;
  const bool fit1 = dyn(48) + 32 * 32 * 8 <= 232448;
  if (want == DRIFT_STRIP2) return fit2 ? DRIFT_STRIP2 : DRIFT_WINDOW;
  if (want == DRIFT_STRIP1) return fit1 ? DRIFT_STRIP1 : DRIFT_WINDOW;
  if (sizeof(T) != 4) return DRIFT_WINDOW;
  return fit2 ? DRIFT_STRIP2 : fit1 ? DRIFT_STRIP1 : DRIFT_WINDOW;
}

template <typename T, int WC, int NW, int MINB, int PF = 2>
static cudaError_t drift_strip_go(const CUtensorMap *tmS, const T *C, T *f, const int32_t *idx,
                                  const T *fx, const T *fy, const uint2 *fp2,
                                  const int64_t *ch_start, const int32_t *ch_len,
                                  const T *ch_val, int64_t ndrift, const MomentTables &mt,
                                  double *partial, unsigned int *err, uint32_t spins,
                                  const Geometry &g, cudaStream_t st) {
  const int nch = (g.nu + 3 + DS_ROWS - 1) / DS_ROWS;
  const size_t smem = (size_t)nch * DS_ROWS * WC * sizeof(T) + nch * sizeof(uint64_t);
  cudaError_t e = cudaFuncSetAttribute(drift_strip_kernel<T, WC, NW, MINB, PF>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // N_r = 32 k + 1 (every grid of the form 2^n + 1): k blocks, the last one
  // also takes the last column; 2.4 % faster than a block of one column on
  // the 513 x 513 x 256 case
  const int extra = (g.nr % 32 == 1 && g.nr > 32) ? 1 : 0;
  const dim3 grid(extra ? g.nr / 32 : (g.nr + 31) / 32, g.nb);
  drift_strip_kernel<T, WC, NW, MINB, PF><<<grid, 32 * NW, smem, st>>>(
      *tmS, C, f, idx, fx, fy, fp2, ch_start, ch_len, ch_val, ndrift, mt, partial, err, spins,
      extra, g);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_drift_strip(const CUtensorMap *tmS, int kind, const T *C, T *f,
                               const int32_t *idx, const T *fx, const T *fy, const uint2 *fp2,
                               const int64_t *ch_start, const int32_t *ch_len,
                               const T *ch_val, int64_t ndrift, const MomentTables &mt,
                               double *partial, unsigned int *err, uint32_t spins,
                               const Geometry &g, cudaStream_t st) {
  switch (kind) {
    case DRIFT_STRIP2:
      return drift_strip_go<T, 48, 16, 2>(tmS, C, f, idx, fx, fy, fp2, ch_start, ch_len,
                                          ch_val, ndrift, mt, partial, err, spins, g, st);
    case DRIFT_STRIP1:
      return drift_strip_go<T, 48, 32, 1>(tmS, C, f, idx, fx, fy, fp2, ch_start, ch_len,
                                          ch_val, ndrift, mt, partial, err, spins, g, st);
    default:
      return cudaErrorInvalidValue;
  }
}

template <typename T>
__global__ void chain_tail_kernel(const T *__restrict__ C, T *__restrict__ ch_val,
                                  const int64_t *__restrict__ ch_start,
                                  const int32_t *__restrict__ ch_len,
                                  const int32_t *__restrict__ t_idx,
                                  const double *__restrict__ t_x,
                                  const double *__restrict__ t_y,
                                  const int32_t *__restrict__ t_j, int64_t c_lo,
                                  int64_t c_hi, int64_t ndrift, Geometry g) {
  const int64_t c = c_lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c_hi) return;
  const int L = ch_len[c];
  const int code = t_idx[c];
  T v = T(0);
  if (code >= 0) {
    const T *Cj = C + (size_t)(t_j[c] - g.j0) * (g.nu + 3) * g.pc;
    v = eval2d<T>(Cj, g.pc, code & 0xffff, (T)t_x[c], code >> 16, (T)t_y[c]);
  }
  ch_val[ch_start[c] + (ndrift + L - 1) % L] = v;
}

template <typename T>
cudaError_t launch_chain_tails(const T *C, T *ch_val, const int64_t *ch_start,
                               const int32_t *ch_len, const int32_t *t_idx,
                               const double *t_x, const double *t_y,
                               int64_t nchains, int64_t c_lo, int64_t c_hi,
                               int64_t ndrift, const Geometry &g, cudaStream_t st) {
  if (c_hi <= c_lo) return cudaSuccess;
  // t_j (slice of each chain) is stored right after t_idx
  const int32_t *t_j = t_idx + nchains;
  const int threads = 256;
  const unsigned blocks = (unsigned)((c_hi - c_lo + threads - 1) / threads);
  chain_tail_kernel<T><<<blocks, threads, 0, st>>>(C, ch_val, ch_start, ch_len, t_idx,
                                                   t_x, t_y, t_j, c_lo, c_hi, ndrift, g);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ moment
template <typename T>
__global__ void __launch_bounds__(32 * DR_W)
    moment_kernel(const T *__restrict__ f, MomentTables mt,
                  double *__restrict__ partial, Geometry g) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  const int j = blockIdx.y;
  double acc = 0.0;
  if (r < g.nr)
    for (int u = w; u < g.nu; u += DR_W)
      acc += __ldg(mt.bu + u) * (double)f[((size_t)j * g.nu + u) * g.nr + r];
  __shared__ double red[DR_W][32];
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0 && r < g.nr) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < DR_W; ++k) s += red[k][lane];
    partial[(size_t)j * g.nr + r] = __ldg(mt.wj + j) * s;
  }
}

template <typename T>
cudaError_t launch_moment(const T *f, const MomentTables &mt, double *partial,
                          const Geometry &g, cudaStream_t st) {
  dim3 grid((g.nr + 31) / 32, g.nj);
  moment_kernel<T><<<grid, 32 * DR_W, 0, st>>>(f, mt, partial, g);
  return cudaGetLastError();
}

// -------------------------------------------------------------- scan
constexpr int SC_THREADS = 1024;
constexpr int SC_RB = 32;  // r columns per reduction block

// grid: ceil(N_r / SC_RB) blocks; each reduces partial[:, r-strip] over J
// (compensated) into T2.  The last block to finish (threadfence reduction
// pattern, no spin-wait) computes bins, the exclusive scan, mtot and shift.
// `count` is a per-handle device counter that the last block resets to 0.

__global__ void __launch_bounds__(SC_THREADS)
    scan_kernel(const double *__restrict__ partial, MomentTables mt,
                double *__restrict__ T2, double *__restrict__ bins,
                double *__restrict__ Mr, double *__restrict__ shift,
                double *__restrict__ mtot, unsigned int *count, unsigned int *status,
                Geometry g) {
  __shared__ dd sh[SC_THREADS];
  __shared__ bool last;
  const int tid = threadIdx.x;
  {
    const int lr = tid % SC_RB, jg = tid / SC_RB;  // 32 groups of J
    const int ngroups = SC_THREADS / SC_RB;
    const int r = blockIdx.x * SC_RB + lr;
    dd acc{0.0, 0.0};
    if (r < g.nr)
      for (int j = jg; j < g.nj; j += ngroups)
        acc = dd_add(acc, dd{partial[(size_t)j * g.nr + r], 0.0});
    sh[tid] = acc;
    __syncthreads();
    for (int s = ngroups / 2; s > 0; s >>= 1) {
      if (jg < s) sh[tid] = dd_add(sh[tid], sh[tid + s * SC_RB]);
      __syncthreads();
    }
    if (jg == 0 && r < g.nr) T2[r] = sh[tid].hi + sh[tid].lo;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    const unsigned int done = atomicAdd(count, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // bins (each thread up to 2 consecutive r), then a block-wide exclusive scan
  const int per = (g.nr + SC_THREADS - 1) / SC_THREADS;  // 1 or 2
  double b[2] = {0.0, 0.0};
  dd loc{0.0, 0.0};
  for (int q = 0; q < per; ++q) {
    const int r = tid * per + q;
    if (r < g.nr) {
      const double t2 = *((volatile double *)T2 + r);
      const double t3 = (r + 1 < g.nr) ? *((volatile double *)T2 + r + 1) : 0.0;
      b[q] = (r < g.nr - 1) ? __ldg(mt.dR4 + r) * (t2 + t3) : 0.0;
      bins[r] = b[q];
      loc = dd_add(loc, dd{b[q], 0.0});
    }
  }
  // inclusive warp scan of loc
  const int lane = tid & 31, wid = tid >> 5;
  dd inc = loc;
  for (int d = 1; d < 32; d <<= 1) {
    dd o = dd_shfl_up(inc, d);
    if (lane >= d) inc = dd_add(inc, o);
  }
  __shared__ dd wsum[SC_THREADS / 32];
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    dd x = wsum[lane];
    dd xi = x;
    for (int d = 1; d < 32; d <<= 1) {
      dd o = dd_shfl_up(xi, d);
      if (lane >= d) xi = dd_add(xi, o);
    }
    wsum[lane] = dd_add(xi, dd{-x.hi, -x.lo});  // exclusive
    if (lane == 31) {
      const double total = xi.hi + xi.lo;
      *mtot = total;
      // every cell enters the mass with a positive weight, so a NaN or an
      // infinity anywhere in f makes the total non-finite
      if (!isfinite(total)) atomicOr(status, 2u);
    }
  }
  __syncthreads();
  dd ex = dd_add(wsum[wid], dd_add(inc, dd{-loc.hi, -loc.lo}));
  for (int q = 0; q < per; ++q) {
    const int r = tid * per + q;
    if (r < g.nr) {
      const double m = ex.hi + ex.lo;
      Mr[r] = m;
      shift[r] = m * __ldg(mt.Rcoef + r);
      ex = dd_add(ex, dd{b[q], 0.0});
    }
  }
  if (tid == 0) *count = 0u;
}

cudaError_t launch_scan(const double *partial, const MomentTables &mt,
                        double *T2, double *bins, double *Mr, double *shift,
                        double *mtot, unsigned int *count, unsigned int *status,
                        const Geometry &g, cudaStream_t st) {
  if (g.nr > 2 * SC_THREADS) return cudaErrorInvalidValue;
  const unsigned blocks = (g.nr + SC_RB - 1) / SC_RB;
  scan_kernel<<<blocks, SC_THREADS, 0, st>>>(partial, mt, T2, bins, Mr, shift, mtot,
                                             count, status, g);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ stats
// integrate() of Ek, S, L1, L2 (quadrature21.hxx:56-85, integrand21.hxx:82-145)
// per block: one J slice, rows u = blockIdx.x*ST_U.., threads over r; block
// partials in double-double, 4 quantities x (hi, lo).
constexpr int ST_THREADS = 256;
constexpr int ST_U = 8;

template <typename T>
__global__ void __launch_bounds__(ST_THREADS)
    stats_kernel(const T *__restrict__ f, const double *__restrict__ R,
                 const double *__restrict__ U, const double *__restrict__ J,
                 const double *__restrict__ dR, const double *__restrict__ dU,
                 const double *__restrict__ Ct1, double *__restrict__ part,
                 Geometry g) {
  const int j = blockIdx.y;
  const int u0 = blockIdx.x * ST_U;
  dd acc[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
  const double Jj = J[j], ct = Ct1[j];
  for (int uu = 0; uu < ST_U; ++uu) {
    const int u = u0 + uu;
    if (u >= g.nu - 1) break;
    const double du = dU[u];
    if (du <= 0) continue;
    const double um = U[u] + 0.5 * du;
    for (int r = threadIdx.x; r < g.nr - 1; r += ST_THREADS) {
      const double dr = dR[r];
      if (dr <= 0) continue;
      const size_t i = ((size_t)j * g.nu + u) * g.nr + r;
      const double avg =
          ((double)f[i] + (double)f[i + 1] + (double)f[i + g.nr] +
           (double)f[i + g.nr + 1]) *
          0.25;
      const double rm = R[r] + 0.5 * dr;
      const double w = ct * du * dr;
      acc[0] = dd_add(acc[0], dd{w * (0.5 * avg * (um * um + Jj * Jj / (rm * rm))), 0});
      acc[1] = dd_add(acc[1], dd{w * ((avg <= 0) ? 0.0 : -avg * log(avg)), 0});
      acc[2] = dd_add(acc[2], dd{w * fabs(avg), 0});
      acc[3] = dd_add(acc[3], dd{w * (avg * avg), 0});
    }
  }
  for (int q = 0; q < 4; ++q)
    for (int d = 16; d > 0; d >>= 1) acc[q] = dd_add(acc[q], dd_shfl_down(acc[q], d));
  __shared__ dd ws[ST_THREADS / 32][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 4; ++q) ws[wid][q] = acc[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    for (int q = 0; q < 4; ++q) {
      dd s{0, 0};
      for (int k = 0; k < ST_THREADS / 32; ++k) s = dd_add(s, ws[k][q]);
      part[b * 8 + 2 * q] = s.hi;
      part[b * 8 + 2 * q + 1] = s.lo;
    }
  }
}

template <typename T>
cudaError_t launch_stats(const T *f, const double *R, const double *U,
                         const double *J, const double *dR, const double *dU,
                         const double *Ct1, double *part, double *out4,
                         const Geometry &g, cudaStream_t st) {
  (void)out4;
  dim3 grid((g.nu + ST_U - 1) / ST_U, g.nj);
  stats_kernel<T><<<grid, ST_THREADS, 0, st>>>(f, R, U, J, dR, dU, Ct1, part, g);
  return cudaGetLastError();
}

// ------------------------------------------------------------ conversions
template <typename T>
__global__ void convert_in_kernel(const double *__restrict__ s, T *__restrict__ d,
                                  size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    d[i] = (T)s[i];
}
template <typename T>
__global__ void convert_out_kernel(const T *__restrict__ s, double *__restrict__ d,
                                   size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    d[i] = (double)s[i];
}
template <typename T>
__global__ void nonfinite_kernel(const T *__restrict__ s, size_t n,
                                 unsigned int *flag) {
  unsigned int bad = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    bad |= !isfinite((double)s[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

static unsigned grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b == 0) b = 1;
  return (unsigned)b;
}

template <typename T>
cudaError_t launch_convert_in(const double *src, T *dst, size_t n,
                              cudaStream_t st) {
  convert_in_kernel<T><<<grid_for(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_convert_out(const T *src, double *dst, size_t n,
                               cudaStream_t st) {
  convert_out_kernel<T><<<grid_for(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_nonfinite(const T *f, size_t n, unsigned int *flag,
                             cudaStream_t st) {
  nonfinite_kernel<T><<<grid_for(n), 256, 0, st>>>(f, n, flag);
  return cudaGetLastError();
}

#define VLS_INST(T)                                                            \
  template int drift_strip_width<T>(int, int);                                  \
  template cudaError_t launch_drift_strip<T>(                                   \
      const CUtensorMap *, int, const T *, T *, const int32_t *, const T *, const T *, \
      const uint2 *, const int64_t *, const int32_t *, const T *, int64_t,       \
      const MomentTables &, double *, unsigned int *, uint32_t, const Geometry &, \
      cudaStream_t);                                                            \
  template cudaError_t launch_drift_tma<T>(                                     \
      const CUtensorMap *, const T *, T *, const int32_t *, const T *, const T *, \
      const uint2 *, const int64_t *, const int32_t *, const T *, int64_t,        \
      const MomentTables &, double *, unsigned int *, uint32_t, const Geometry &, \
      cudaStream_t);                                                            \
  template cudaError_t launch_chain_tails<T>(                                   \
      const T *, T *, const int64_t *, const int32_t *, const int32_t *,         \
      const double *, const double *, int64_t, int64_t, int64_t, int64_t,       \
      const Geometry &, cudaStream_t);                                          \
  template cudaError_t launch_moment<T>(const T *, const MomentTables &,        \
                                        double *, const Geometry &,             \
                                        cudaStream_t);                          \
  template cudaError_t launch_stats<T>(                                         \
      const T *, const double *, const double *, const double *,                \
      const double *, const double *, const double *, double *, double *,       \
      const Geometry &, cudaStream_t);                                          \
  template cudaError_t launch_convert_in<T>(const double *, T *, size_t,        \
                                            cudaStream_t);                      \
  template cudaError_t launch_convert_out<T>(const T *, double *, size_t,       \
                                             cudaStream_t);                     \
  template cudaError_t launch_nonfinite<T>(const T *, size_t, unsigned int *,   \
                                           cudaStream_t);

VLS_INST(float)
VLS_INST(double)

#define VLS_INST_TR(T, R)                                                       \
  template cudaError_t launch_ucol<T, R>(bool, const T *, T *, const double *,  \
                                         const Geometry &, const DirTables &,   \
                                         cudaStream_t);                         \
  template cudaError_t launch_prer<T, R>(const T *, T *, const Geometry &,      \
                                         const DirTables &, cudaStream_t);

VLS_INST_TR(double, double)
VLS_INST_TR(float, double)
VLS_INST_TR(float, float)

}  // namespace vls
