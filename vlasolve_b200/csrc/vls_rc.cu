// vls_rc.cu -- the cubic B-spline prefilter with register-resident lines.
//
// A line of the natural-BC system (localSpline::create_1D,
// localSpline.hxx:953-1182) has N data rows k = 1..N and M = N + 2
// coefficients.  It is cut into S = ceil(N / L) chunks of L rows; each
// thread holds one chunk of one line in registers and runs the Thomas
// recurrences there:
//
//   forward   d_k = (x_k - d_{k-1}/6) rp_k          (written d = d m_k + x rp_k)
//   last row  c_{M-1} = ((0 - hi2 d_{N-1}) - L1 d_N) / L2   (times 1/L2 from the host)
//   backward  c_k = d_k - q_k c_{k+1},  c_0 = (0 - a01 c_1) - a02 c_2
//
// Chunks other than the first start their recurrence from zero and are
// corrected afterwards: the true d_k differs from the local one by
// m^(k - k_first + 1) times the true d at the row before the chunk (the
// "carry"), and likewise backward with (-q)^(...).  From row L+1 on the
// coefficients are constant (rp_inf, q_inf) in the recursion's precision, so
// the correction factors are powers of one constant, held in the kernel
// parameters.  A carry is the neighbour chunk's local end value plus m^L (or
// (-q)^L) times the next one's; the remaining term is below m^(2L) (7e-18
// for L = 15) of the values and is dropped.  The first chunk (rows 1..L, where the
// coefficients still vary) runs the exact recurrences with the per-row
// tables; the last chunk computes c_{M-1} and starts the backward pass from
// it.
//
// Block layout (RcCfg): LN lines per block, 32/LN chunks per warp.  Warp 0
// holds the first chunk (lanes 0..LN-1) and the last chunk (lanes LN..2LN-1),
// the two chunks with their own code paths; every other warp holds 32/LN
// middle chunks.  L is odd so that the chunks of a warp, whose rows differ by
// multiples of L, fall on distinct shared-memory banks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "vls_async.cuh"
#include "vls_internal.h"
#include "vls_setup.h"

namespace vls {

namespace {

template <int L_, int LN_, int NT_, int MINB_>
struct RcCfg {
  static constexpr int L = L_, LN = LN_, CPW = 32 / LN_, NT = NT_, MINB = MINB_;
};
// most chunks one block holds in the adjoint kernels' layout: warp 0 (first
// and last chunk) + (NT/32 - 1) warps of CPW chunks
template <class C>
__host__ __device__ constexpr int rc_maxs() {
  return 2 + (C::NT / 32 - 1) * C::CPW;
}
// configuration ids (host and device agree on the order)
using CfgB = RcCfg<15, 8, 320, 3>;    // 15-row chunks, 8 lines, three blocks per SM
using CfgB1 = RcCfg<15, 8, 640, 1>;   // the same for up to 77 chunks
using CfgC = RcCfg<15, 16, 576, 2>;   // 15-row chunks, 16 lines, two blocks per SM
using CfgD = RcCfg<23, 8, 384, 2>;    // 23-row chunks, 8 lines, two blocks per SM (up to 45 chunks)
using CfgF = RcCfg<19, 8, 256, 3>;    // 19-row chunks, 8 lines, three blocks per SM (up to 29 chunks)
using CfgI = RcCfg<17, 16, 512, 2>;   // 17-row chunks, 16 lines, two blocks per SM (up to 31 chunks)

template <typename R>
struct Dev;
template <>
struct Dev<double> {
  static __device__ __forceinline__ double fma_(double a, double b, double c) {
    return __fma_rn(a, b, c);
  }
};
template <>
struct Dev<float> {
  static __device__ __forceinline__ float fma_(float a, float b, float c) {
    return __fmaf_rn(a, b, c);
  }
};

template <typename R>
__device__ __forceinline__ R rfma(R a, R b, R c) {
  return Dev<R>::fma_(a, b, c);
}

// cubic B-spline weights (localSpline.hxx:381-441): BV2(x) = x^3,
// BV1(x) = 1 + 3x + 3x^2 - 3x^3
template <typename T>
__device__ __forceinline__ T w_bv2(T x) {
  return x * x * x;
}
template <typename T>
__device__ __forceinline__ T w_bv1(T x) {
  return T(1) + T(3) * x + T(3) * x * x - T(3) * x * x * x;
}

// w / 6 without a division: FP32 multiplies by 1/6 split into a rounded
// head and its remainder (one multiply, one FMA), so the quotient carries no
// rounding bias of the constant; FP64 multiplies by the rounded 1/6
template <typename T>
__device__ __forceinline__ T over6(T w) {
  return w * (T(1) / T(6));
}
template <>
__device__ __forceinline__ float over6<float>(float w) {
  return __fmaf_rn(w, 0.1666666716337204f, w * -4.967053879312289e-09f);
}

__host__ __device__ constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }

// chunk index, role and activity of this thread
struct Role {
  int s;        // chunk
  bool active;  // holds a chunk
  int ln;       // line within the block
  int warp, grp;  // warp, chunk slot within the warp
};

template <class C>
__device__ __forceinline__ Role rc_role(int S) {
  Role o;
  const int lane = threadIdx.x & 31;
  o.warp = threadIdx.x >> 5;
  o.grp = lane / C::LN;
  o.ln = lane % C::LN;
  if (o.warp == 0) {
    o.s = o.grp == 0 ? 0 : S - 1;
    o.active = o.grp == 0 || (o.grp == 1 && S >= 2);
  } else {
    o.s = 1 + (o.warp - 1) * C::CPW + o.grp;
    o.active = o.s <= S - 2;
  }
  return o;
}

// The solve of one chunk per thread; v holds x on entry and c on exit.
// dend, cst: shared [S][LN] carry slots.  c0 (first chunk) and cM (last
// chunk) receive the two boundary coefficients.
template <typename R, class C>
__device__ __forceinline__ void rc_solve(R (&v)[C::L], const Role &ro, R *dend, R *cst,
                                         const RcDir<R> &t, R &c0, R &cM) {
  constexpr int L = C::L, LN = C::LN;
  const int S = t.S, N = t.N;
  const int s = ro.s;
  const int kfirst = 1 + s * L;
  const int slot = s * LN + ro.ln;
  // ---------------------------------------------------------- phase A
  if (s == 0) {
    // first chunk: per-row tables (this code path diverges within warp 0)
    R d = R(0);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      d = rfma(d, t.m0[1 + i], v[i] * t.rp0[1 + i]);
      v[i] = d;
    }
    if (ro.active && S >= 2) dend[slot] = d;
  } else {
    R d = R(0);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      d = rfma(d, t.m_inf, v[i] * t.rp_inf);
      v[i] = d;
    }
    if (ro.active) dend[slot] = d;
  }
  __syncthreads();
  // ---------------------------------------------------------- phase B
  if (ro.active) {
    if (S == 1) {
      // the only chunk is first and last: exact recurrences throughout
      const int iN = N - 1;
      R dl = v[0], dp = R(0);
#pragma unroll
      for (int i = 1; i < L; ++i)
        if (i == iN) {
          dl = v[i];
          dp = v[i - 1];
        }
      cM = ((R(0) - t.hi2 * dp) - t.L1 * dl) * t.inv_L2;
      R c = cM;
#pragma unroll
      for (int i = L - 1; i >= 0; --i)
        if (i <= iN) {
          c = rfma(-t.q0[1 + i], c, v[i]);
          v[i] = c;
        }
      c0 = (R(0) - t.a01 * v[0]) - t.a02 * (N >= 2 ? v[1] : cM);
    } else if (s > 0) {
      R carry = dend[slot - LN];
      if (s >= 2) carry = rfma(t.mpow[L], dend[slot - 2 * LN], carry);
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.mpow[i + 1], carry, v[i]);
      R c;
      if (s == S - 1) {
        const int iN = N - kfirst;  // 0 .. L-1
        R dl = v[0], dp = carry;
#pragma unroll
        for (int i = 1; i < L; ++i)
          if (i == iN) {
            dl = v[i];
            dp = v[i - 1];
          }
        cM = ((R(0) - t.hi2 * dp) - t.L1 * dl) * t.inv_L2;
        c = cM;
#pragma unroll
        for (int i = L - 1; i >= 0; --i)
          if (i <= iN) {
            c = rfma(-t.q_inf, c, v[i]);
            v[i] = c;
          }
      } else {
        c = R(0);
#pragma unroll
        for (int i = L - 1; i >= 0; --i) {
          c = rfma(-t.q_inf, c, v[i]);
          v[i] = c;
        }
      }
      cst[slot] = c;
    }
  }
  __syncthreads();
  // ---------------------------------------------------------- phase C
  if (ro.active && S >= 2 && s <= S - 2) {
    R carry = cst[slot + LN];
    if (s + 2 <= S - 1) carry = rfma(t.qpow[L], cst[slot + 2 * LN], carry);
    if (s == 0) {
      R c = carry;
#pragma unroll
      for (int i = L - 1; i >= 0; --i) {
        c = rfma(-t.q0[1 + i], c, v[i]);
        v[i] = c;
      }
      c0 = (R(0) - t.a01 * v[0]) - t.a02 * v[1];
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.qpow[L - i], carry, v[i]);
    }
  }
}

// ------------------------------------------------- forward solve layout
// The forward kernels use a second layout in which no warp runs two chunk
// kinds one after the other: warp 0 holds only the first chunk (lanes
// 0..LN-1; its other lanes compute the same chunk and store nothing), and
// the last chunk follows the middle chunks in the other warps.  Per phase:
//   A  every chunk: local forward recurrence (the first with its per-row
//      coefficients, exact since it starts at row 1)
//   B  first chunk: local backward from zero with its per-row q;
//      others: forward correction by the carry, then the backward from zero
//      (the last chunk from its boundary row, exact)
//   C  first chunk: backward correction qfirst[i] * carry (independent
//      products instead of the dependent exact backward), then c_0;
//      middle chunks: qpow[L - i] * carry
// so every warp's dependent chains are one forward and one backward pass.
template <class C>
__host__ __device__ constexpr int rc2_maxs() {
  return 1 + (C::NT / 32 - 1) * C::CPW;
}
template <class C>
int rc2_threads(int S) {
  return S == 1 ? 32 : 32 * (1 + (S - 1 + C::CPW - 1) / C::CPW);
}
template <class C>
__device__ __forceinline__ Role rc2_role(int S) {
  Role o;
  const int lane = threadIdx.x & 31;
  o.warp = threadIdx.x >> 5;
  o.grp = lane / C::LN;
  o.ln = lane % C::LN;
  if (o.warp == 0) {
    o.s = 0;
    o.active = o.grp == 0;
  } else {
    o.s = 1 + (o.warp - 1) * C::CPW + o.grp;
    o.active = o.s <= S - 1;
  }
  return o;
}

template <typename R, class C>
__device__ __forceinline__ void rc2_solve(R (&v)[C::L], const Role &ro, R *dend, R *cst,
                                          const RcDir<R> &t, R &c0, R &cM) {
  constexpr int L = C::L, LN = C::LN;
  const int S = t.S, N = t.N;
  const int s = ro.s;
  const int kfirst = 1 + s * L;
  const int slot = s * LN + ro.ln;
  // the warp holding the last chunk (its other lanes hold middle chunks)
  const bool lastwarp = ro.warp == (S - 2) / C::CPW + 1;
  // ---------------------------------------------------------- phase A
  if (s == 0) {
    R d = R(0);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      d = rfma(d, t.m0[1 + i], v[i] * t.rp0[1 + i]);
      v[i] = d;
    }
    if (ro.active && S >= 2) dend[slot] = d;
  } else {
    R d = R(0);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      d = rfma(d, t.m_inf, v[i] * t.rp_inf);
      v[i] = d;
    }
    if (ro.active) dend[slot] = d;
  }
  __syncthreads();
  // ---------------------------------------------------------- phase B
  if (S == 1) {
    // the only chunk is first and last: exact recurrences throughout
    const int iN = N - 1;
    R dl = v[0], dp = R(0);
#pragma unroll
    for (int i = 1; i < L; ++i)
      if (i == iN) {
        dl = v[i];
        dp = v[i - 1];
      }
    cM = ((R(0) - t.hi2 * dp) - t.L1 * dl) * t.inv_L2;
    R c = cM;
#pragma unroll
    for (int i = L - 1; i >= 0; --i)
      if (i <= iN) {
        c = rfma(-t.q0[1 + i], c, v[i]);
        v[i] = c;
      }
    c0 = (R(0) - t.a01 * v[0]) - t.a02 * (N >= 2 ? v[1] : cM);
  } else if (s == 0) {
    R c = R(0);
#pragma unroll
    for (int i = L - 1; i >= 0; --i) {
      c = rfma(-t.q0[1 + i], c, v[i]);
      v[i] = c;
    }
  } else {
    // lanes past the last chunk read nothing (their slots lie past dend)
    R carry = ro.active ? dend[slot - LN] : R(0);
    if (s >= 2 && ro.active) carry = rfma(t.mpow[L], dend[slot - 2 * LN], carry);
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = rfma(t.mpow[i + 1], carry, v[i]);
    R c = R(0);
    if (lastwarp) {
      // the last chunk starts from its boundary row; rows past N skipped
      const bool last = s == S - 1;
      const int iN = last ? N - kfirst : L - 1;  // 0 .. L-1
      if (last) {
        R dl = v[0], dp = carry;
#pragma unroll
        for (int i = 1; i < L; ++i)
          if (i == iN) {
            dl = v[i];
            dp = v[i - 1];
          }
        cM = ((R(0) - t.hi2 * dp) - t.L1 * dl) * t.inv_L2;
        c = cM;
      }
#pragma unroll
      for (int i = L - 1; i >= 0; --i)
        if (i <= iN) {
          c = rfma(-t.q_inf, c, v[i]);
          v[i] = c;
        }
    } else {
#pragma unroll
      for (int i = L - 1; i >= 0; --i) {
        c = rfma(-t.q_inf, c, v[i]);
        v[i] = c;
      }
    }
    if (ro.active) cst[slot] = c;
  }
  __syncthreads();
  // ---------------------------------------------------------- phase C
  if (S >= 2 && s <= S - 2) {
    R carry = cst[slot + LN];
    if (s + 2 <= S - 1) carry = rfma(t.qpow[L], cst[slot + 2 * LN], carry);
    if (s == 0) {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.qfirst[i], carry, v[i]);
      c0 = (R(0) - t.a01 * v[0]) - t.a02 * v[1];
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.qpow[L - i], carry, v[i]);
    }
  }
}

// ------------------------------------------------------------------ ucol
// Block: LN r columns of one J slice; a column is a u line.  With KICK: the
// u-solve of f, the kick gather (vlasovSolver21_spline.hxx:752-770 with the
// r-direction (1,4,1)/6 weights folded into the u-only coefficients) from a
// shared copy of the column's coefficients, and the u-solve of the kicked
// values; G receives the u-coefficients.
template <typename T, typename R, bool KICK, class CF>
__global__ void __launch_bounds__(CF::NT, CF::MINB)
    ucol_rc_kernel(const T *__restrict__ f, T *__restrict__ G,
                   const double *__restrict__ shift, Geometry g,
                   const __grid_constant__ RcDir<R> t) {
  constexpr int L = CF::L, LN = CF::LN;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = t.S, N = t.N;  // N == g.nu
  const int M = N + 2;
  R *dend = reinterpret_cast<R *>(smem_raw);
  R *cst = dend + S * LN;
  T *kb = reinterpret_cast<T *>(smem_raw + al16(2 * (size_t)S * LN * sizeof(R)));
  const Role ro = rc2_role<CF>(S);
  const int r = blockIdx.x * LN + ro.ln;
  const bool colok = r < g.nr;
  const int jl = blockIdx.y, j = g.j0 + jl;
  const int kfirst = 1 + ro.s * L;
  R v[L];
  {
    // unpredicated loads kept inside the slice (columns clamped to N_r - 1,
    // rows to N in the last chunk): values of rows beyond N and of idle
    // threads are never used.  Offsets within the slice are 32-bit.
    const T *fc = f + (size_t)j * g.nu * g.nr + (colok ? r : g.nr - 1);
    const uint32_t nr = (uint32_t)g.nr;
    if (kfirst + L - 1 <= N) {
      uint32_t o = (uint32_t)(kfirst - 1) * nr;
#pragma unroll
      for (int i = 0; i < L; ++i) {
        v[i] = (R)__ldg(fc + o);
        o += nr;
      }
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) {
        const int k = min(kfirst + i, N);
        v[i] = (R)__ldg(fc + (uint32_t)(k - 1) * nr);
      }
    }
  }
  R c0 = R(0), cM = R(0);
  rc2_solve<R, CF>(v, ro, dend, cst, t, c0, cM);
  if (KICK) {
    // chunks wholly inside the line (every chunk but the last) store without
    // per-row tests
    const bool full = kfirst + L - 1 <= N;
    if (ro.active) {
      if (full) {
#pragma unroll
        for (int i = 0; i < L; ++i) kb[(kfirst + i) * LN + ro.ln] = (T)v[i];
      } else {
#pragma unroll
        for (int i = 0; i < L; ++i) {
          const int k = kfirst + i;
          if (k <= N) kb[k * LN + ro.ln] = (T)v[i];
        }
      }
      if (ro.s == 0) kb[ro.ln] = (T)c0;
      if (ro.s == S - 1) {
        kb[(M - 1) * LN + ro.ln] = (T)cM;
        kb[M * LN + ro.ln] = T(0);
      }
    }
    __syncthreads();
    // The shift is constant along the column and the u grid is uniform, so
    // y_u = u + s*hu: one fraction and one integer offset serve every row,
    // unless that fraction is within 1e-9 of a node (then every row takes
    // the exact per-cell path).  Rows with 0 < u + s*hu < N-1 are inside
    // (strictly, vlasovSolver21_spline.hxx:761); outside rows get 0.
    const double sft = colok ? __ldg(shift + r) : 0.0;
    const double qf = sft * g.hu;
    const double fl = floor(qf);
    const double frd = qf - fl;
    const bool fast = frd > 1e-9 && frd < 1.0 - 1e-9 && fabs(qf) < 1e6;
    if (ro.active) {
      if (fast) {
        const int o = (int)fl;
        const T fr = (T)frd;
        // weights divided by 6 (a single rounded 1/6 factor would bias every
        // kick the same way, a steady mass drift in FP32)
        const T w0 = over6(w_bv2<T>(T(1) - fr)), w1 = over6(w_bv1<T>(T(1) - fr));
        const T w2 = over6(w_bv1<T>(fr)), w3 = over6(w_bv2<T>(fr));
        const int ulo = (int)floor(-qf) + 1;
        const int uhi = (int)ceil((double)(N - 1) - qf) - 1;
        // row k = kfirst + i (u = k - 1) reads coefficient rows k+o-1 .. k+o+2
        const int ilo = ulo - kfirst + 1, ihi = min(uhi, N - 1) - kfirst + 1;
        const T *base = kb + (ptrdiff_t)(kfirst + o - 1) * LN + ro.ln;
        if (ilo <= 0 && ihi >= L - 1) {
          // every row of the chunk inside
#pragma unroll
          for (int i = 0; i < L; ++i) {
            const T *p = base + i * LN;
            v[i] = (R)(w0 * p[0] + w1 * p[LN] + w2 * p[2 * LN] + w3 * p[3 * LN]);
          }
        } else {
#pragma unroll
          for (int i = 0; i < L; ++i) {
            T x = T(0);
            if (i >= ilo && i <= ihi) {
              const T *p = base + i * LN;
              x = w0 * p[0] + w1 * p[LN] + w2 * p[2 * LN] + w3 * p[3 * LN];
            }
            v[i] = (R)x;
          }
        }
      } else {
        // exact per-cell path (localSpline.hxx:426-429)
#pragma unroll
        for (int i = 0; i < L; ++i) {
          const int k = kfirst + i, u = k - 1;
          R x = R(0);
          if (k <= N) {
            const double newU = __ldg(g.U + u) + sft;
            if (newU > g.u0 && newU < g.umax) {
              const double y = (newU - g.su) * g.hu;
              const double yf = floor(y);
              const T fr = (T)(y - yf);
              const int Ny = 1 + (int)yf;
              const T *p = kb + (ptrdiff_t)(Ny - 1) * LN + ro.ln;
              x = (R)over6(w_bv2<T>(T(1) - fr) * p[0] + w_bv1<T>(T(1) - fr) * p[LN] +
                           w_bv1<T>(fr) * p[2 * LN] + w_bv2<T>(fr) * p[3 * LN]);
            }
          }
          v[i] = x;
        }
      }
    }
    rc2_solve<R, CF>(v, ro, dend, cst, t, c0, cM);
  }
  if (ro.active && colok) {
    T *Gc = G + (size_t)jl * M * g.gp + r;
    const uint32_t gp = (uint32_t)g.gp;
    if (kfirst + L - 1 <= N) {
      uint32_t o = (uint32_t)kfirst * gp;
#pragma unroll
      for (int i = 0; i < L; ++i) {
        Gc[o] = (T)v[i];
        o += gp;
      }
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) {
        const int k = kfirst + i;
        if (k <= N) Gc[(uint32_t)k * gp] = (T)v[i];
      }
    }
    if (ro.s == 0) Gc[0] = (T)c0;
    if (ro.s == S - 1) Gc[(uint32_t)(M - 1) * gp] = (T)cM;
  }
}

// ------------------------------------------------------------------ prer
// Block: LN rows of G (u lines of the padded grid) of one J slice; a row is
// an r line.  The rows are staged in shared memory, each thread moves its
// chunk into registers, solves, and writes it back; the block then stores the
// tile to C.
//
// Tile row pitch P: the lanes of a warp read (line ln, chunk slot m) at
// ln*P + m*L + const.  FP32 words: P = 2 mod 32 for 16 lines, 4 mod 32 for 8
// lines, so that the 32/LN lines times the chunk slots (L odd) cover the 32
// banks.  FP64 words (16 lanes per wavefront): odd P for 16 lines, 2 mod 16
// for 8 lines.
//
// With 8 lines the pitch is a multiple of 16 bytes, and whole rows move as
// bulk copies: G row -> tile row from word OFF = 16 bytes on (x_k at
// OFF - 1 + k), and tile row -> C row from word 0 (c_k at k, words M .. Pc-1
// zeroed).  A thread reads its whole chunk before the solve's first barrier
// and writes after its last one, so the two offsets do not race.  Otherwise
// (16 lines) the rows are copied element-wise with x_k at word k.
template <class CF>
__host__ __device__ constexpr bool rc_bulk_rows() {
  return CF::LN == 8;
}
__host__ __device__ inline int rc_tile_pitch(int M, int elem, int LN) {
  if (elem == 4) return (M + 31) / 32 * 32 + (LN == 16 ? 2 : 4);
  if (LN == 16) return M | 1;
  return (M + 15) / 16 * 16 + 2;
}
// the forward r-solve's tile: with bulk rows, room for OFF + Pg words in and
// Pc words out, at the same pitch residues
__host__ __device__ inline int rc_tile_pitch_rows(int M, int gp, int pc, int elem, int LN) {
  if (LN != 8) return rc_tile_pitch(M, elem, LN);
  const int need = max(max(16 / elem + gp, pc), M);
  return elem == 4 ? (need - 4 + 31) / 32 * 32 + 4 : (need - 2 + 15) / 16 * 16 + 2;
}

template <typename T>
__device__ __forceinline__ void cp_async_el(T *smem, const T *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem),
               "n"(sizeof(T))
               : "memory");
}

template <typename T, typename R, class CF>
__global__ void __launch_bounds__(CF::NT, CF::MINB)
    prer_rc_kernel(const T *__restrict__ G, T *__restrict__ C, Geometry g,
                   const __grid_constant__ RcDir<R> t, unsigned int *err) {
  constexpr int L = CF::L, LN = CF::LN;
  constexpr bool BULK = rc_bulk_rows<CF>();
  constexpr int OFF = BULK ? (int)(16 / sizeof(T)) : 1;  // word of x_1 in a tile row
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  const int S = t.S, N = t.N;  // N == g.nr
  const int M = N + 2;
  const int P = rc_tile_pitch_rows(M, g.gp, g.pc, sizeof(T), LN);
  R *dend = reinterpret_cast<R *>(smem_raw);
  R *cst = dend + S * LN;
  T *tile = reinterpret_cast<T *>(smem_raw + al16(2 * (size_t)S * LN * sizeof(R)));
  const Role ro = rc2_role<CF>(S);
  const int jl = blockIdx.y;
  const int rows = g.nu + 2;
  const int kr0 = blockIdx.x * LN;
  const int nrow = min(LN, rows - kr0);
  const T *Gs = G + ((size_t)jl * rows + kr0) * g.gp;
  bool landed = true;
  if constexpr (BULK) {
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      mbar_fence_init();
      const uint32_t bytes = (uint32_t)g.gp * sizeof(T);
      mbar_expect_tx(&bar, bytes * (uint32_t)nrow);
      for (int p = 0; p < nrow; ++p) bulk_load(tile + p * P + OFF, Gs + (size_t)p * g.gp, bytes, &bar);
    }
    __syncthreads();
    if (!mbar_wait_bounded(&bar, 0u)) {
      landed = false;
      atomicOr(err, 4u);
    }
  } else {
    for (int p = 0; p < nrow; ++p) {
      const T *src = Gs + (size_t)p * g.gp;
      T *dst = tile + p * P + OFF;
      for (int k = threadIdx.x; k < N; k += blockDim.x) cp_async_el(dst + k, src + k);
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
  }
  const bool lineok = ro.ln < nrow;
  const int kfirst = 1 + ro.s * L;
  R v[L];
  {
    // rows clamped to N in the last chunk; rows beyond N and lines beyond the
    // tile's last row are computed but never stored
    const T *row = tile + ro.ln * P + (OFF - 1);
    if (kfirst + L - 1 <= N) {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = (R)row[kfirst + i];
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = (R)row[min(kfirst + i, N)];
    }
  }
  R c0 = R(0), cM = R(0);
  rc2_solve<R, CF>(v, ro, dend, cst, t, c0, cM);
  if (ro.active && lineok) {
    T *row = tile + ro.ln * P;
    if (kfirst + L - 1 <= N) {
#pragma unroll
      for (int i = 0; i < L; ++i) row[kfirst + i] = (T)v[i];
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) {
        const int k = kfirst + i;
        if (k <= N) row[k] = (T)v[i];
      }
    }
    if (ro.s == 0) row[0] = (T)c0;
    if (ro.s == S - 1) {
      row[M - 1] = (T)cM;
      if (BULK)
        for (int k = M; k < g.pc; ++k) row[k] = T(0);
    }
  }
  T *Cs = C + ((size_t)jl * (g.nu + 3) + kr0) * g.pc;
  if constexpr (BULK) {
    fence_proxy_async();  // this thread's tile writes, visible to the bulk copies
    __syncthreads();
    if (threadIdx.x == 0) {
      if (landed) {
        const uint32_t bytes = (uint32_t)g.pc * sizeof(T);
        for (int p = 0; p < nrow; ++p) bulk_store(Cs + (size_t)p * g.pc, tile + p * P, bytes);
        bulk_commit();
        bulk_wait_read();
      } else if (!mbar_wait_bounded(&bar, 0u)) {
        // the rows never landed: nothing stored, and the block leaves only
        // after a second bounded wait for the copies in flight
        atomicOr(err, 8u);
      }
    }
  } else {
    __syncthreads();
    for (int p = 0; p < nrow; ++p) {
      const T *src = tile + p * P;
      T *dst = Cs + (size_t)p * g.pc;
      for (int k = threadIdx.x; k < M; k += blockDim.x) dst[k] = src[k];
    }
  }
}

// Persistent form of the bulk-row r-solve: each block walks groups of LN
// rows (gid = blockIdx.x, + gridDim.x, ...) through RC_PIPE_TILES row tiles,
// with the bulk loads of the next RC_PIPE_AHEAD groups in flight while it
// solves one: a group's solve is shorter than an HBM load, and three
// blocks of one group each keep too few bytes in flight per SM.  Thread 0
// issues the loads, and the bulk stores of each group after its solve; a
// tile is reloaded only once the stores issued from it have finished
// reading it.  Waits are bounded: after a timeout the block stores nothing
// more, waits (bounded) for its loads in flight and leaves, and the error
// word tells the host.
constexpr int RC_PIPE_TILES = 4, RC_PIPE_AHEAD = 2;

template <typename T, typename R, class CF>
__global__ void __launch_bounds__(CF::NT, CF::MINB)
    prer_pipe_kernel(const T *__restrict__ G, T *__restrict__ C, Geometry g,
                     const __grid_constant__ RcDir<R> t, unsigned int *err, int gps,
                     int ngroups) {
  constexpr int L = CF::L, LN = CF::LN;
  static_assert(rc_bulk_rows<CF>(), "the pipelined r-solve needs bulk rows");
  // the tile reloaded for group i + AHEAD was stored from at group
  // i + AHEAD - TILES, at least two groups before: wait_group.read 1
  static_assert(RC_PIPE_TILES - RC_PIPE_AHEAD >= 2, "tile reuse distance");
  constexpr int OFF = (int)(16 / sizeof(T));  // word of x_1 in a tile row
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar[RC_PIPE_TILES];
  __shared__ int bad;
  const int S = t.S, N = t.N;  // N == g.nr
  const int M = N + 2;
  const int P = rc_tile_pitch_rows(M, g.gp, g.pc, sizeof(T), LN);
  R *dend = reinterpret_cast<R *>(smem_raw);
  R *cst = dend + S * LN;
  T *tiles = reinterpret_cast<T *>(smem_raw + al16(2 * (size_t)S * LN * sizeof(R)));
  const Role ro = rc2_role<CF>(S);
  const int rows = g.nu + 2;
  const int cnt =
      (int)blockIdx.x < ngroups ? (ngroups - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const uint32_t gbytes = (uint32_t)g.gp * sizeof(T), cbytes = (uint32_t)g.pc * sizeof(T);
  auto group = [&](int i, int &jl, int &kr0, int &nrow) {
    const int gid = (int)blockIdx.x + i * (int)gridDim.x;
    jl = gid / gps;
    kr0 = (gid - jl * gps) * LN;
    nrow = min(LN, rows - kr0);
  };
  auto issue = [&](int i) {
    int jl, kr0, nrow;
    group(i, jl, kr0, nrow);
    const int b = i % RC_PIPE_TILES;
    T *tile = tiles + (size_t)b * LN * P;
    const T *Gs = G + ((size_t)jl * rows + kr0) * g.gp;
    mbar_expect_tx(&bar[b], gbytes * (uint32_t)nrow);
    for (int p = 0; p < nrow; ++p)
      bulk_load(tile + p * P + OFF, Gs + (size_t)p * g.gp, gbytes, &bar[b]);
  };
  int issued = 0;  // groups whose loads thread 0 issued
  if (threadIdx.x == 0) {
    for (int b = 0; b < RC_PIPE_TILES; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
    bad = 0;
    for (; issued < RC_PIPE_AHEAD && issued < cnt; ++issued) issue(issued);
  }
  __syncthreads();
  int i = 0;
  for (; i < cnt; ++i) {
    const int b = i % RC_PIPE_TILES;
    const uint32_t par = (uint32_t)(i / RC_PIPE_TILES) & 1u;
    T *tile = tiles + (size_t)b * LN * P;
    if (threadIdx.x == 0 && i + RC_PIPE_AHEAD < cnt) {
      asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
      issue(i + RC_PIPE_AHEAD);
      issued = i + RC_PIPE_AHEAD + 1;
    }
    if (!mbar_wait_bounded(&bar[b], par)) {
      atomicOr(err, 4u);
      bad = 1;
    }
    int jl, kr0, nrow;
    group(i, jl, kr0, nrow);
    const bool lineok = ro.ln < nrow;
    const int kfirst = 1 + ro.s * L;
    R v[L];
    {
      const T *row = tile + ro.ln * P + (OFF - 1);
      if (kfirst + L - 1 <= N) {
#pragma unroll
        for (int k = 0; k < L; ++k) v[k] = (R)row[kfirst + k];
      } else {
#pragma unroll
        for (int k = 0; k < L; ++k) v[k] = (R)row[min(kfirst + k, N)];
      }
    }
    R c0 = R(0), cM = R(0);
    rc2_solve<R, CF>(v, ro, dend, cst, t, c0, cM);
    if (ro.active && lineok) {
      T *row = tile + ro.ln * P;
      if (kfirst + L - 1 <= N) {
#pragma unroll
        for (int k = 0; k < L; ++k) row[kfirst + k] = (T)v[k];
      } else {
#pragma unroll
        for (int k = 0; k < L; ++k) {
          const int kk = kfirst + k;
          if (kk <= N) row[kk] = (T)v[k];
        }
      }
      if (ro.s == 0) row[0] = (T)c0;
      if (ro.s == S - 1) {
        row[M - 1] = (T)cM;
        for (int k = M; k < g.pc; ++k) row[k] = T(0);
      }
    }
    fence_proxy_async();  // this thread's tile writes, visible to the bulk copies
    __syncthreads();
    const bool stop = bad != 0;
    if (threadIdx.x == 0 && !stop) {
      T *Cs = C + ((size_t)jl * (g.nu + 3) + kr0) * g.pc;
      for (int p = 0; p < nrow; ++p) bulk_store(Cs + (size_t)p * g.pc, tile + p * P, cbytes);
      bulk_commit();
    }
    if (stop) break;
  }
  if (threadIdx.x == 0) {
    bulk_wait_read();
    // after a timeout: the loads issued beyond the failed group must land
    // before the block's shared memory is released
    for (int k = i + 1; k < issued; ++k)
      if (!mbar_wait_bounded(&bar[k % RC_PIPE_TILES], (uint32_t)(k / RC_PIPE_TILES) & 1u))
        atomicOr(err, 8u);
  }
}

template <class CF>
int rc_threads(int S) {
  const int warps = S == 1 ? 1 : 1 + (S - 2 + CF::CPW - 1) / CF::CPW;
  return 32 * warps;
}

template <class CF>
bool cfg_fits(int N, int kc) {
  const int S = (N + CF::L - 1) / CF::L;
  return N >= 2 && kc <= 1 + CF::L && S <= rc_maxs<CF>();
}
// the same for the forward kernels' layout (rc2_role)
template <class CF>
bool cfg2_fits(int N, int kc) {
  const int S = (N + CF::L - 1) / CF::L;
  return N >= 2 && kc <= 1 + CF::L && S <= rc2_maxs<CF>();
}

template <typename K>
cudaError_t rc_attr(K kern, size_t smem) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <typename T, typename R, bool KICK, class CF>
cudaError_t ucol_rc_go(const T *f, T *G, const double *shift, const Geometry &g,
                       const RcDir<R> &tu, cudaStream_t st) {
  const int nt = rc2_threads<CF>(tu.S);
  if (tu.N != g.nu || nt > CF::NT || tu.L != CF::L) return cudaErrorInvalidValue;
  const size_t smem = al16(2 * (size_t)tu.S * CF::LN * sizeof(R)) +
                      (size_t)(tu.N + 3) * CF::LN * sizeof(T);
  const dim3 grid((g.nr + CF::LN - 1) / CF::LN, g.nb);
  auto k = ucol_rc_kernel<T, R, KICK, CF>;
  cudaError_t e = rc_attr(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, nt, smem, st>>>(f, G, shift, g, tu);
  return cudaGetLastError();
}

// occupancy of the persistent r-solve per (device, kernel, shared memory,
// threads), computed on first use
struct PipeOcc {
  int nsm = 0, per = 0;
};
struct PipeOccKey {
  int dev;
  const void *k;
  size_t smem;
  int nt;
  bool operator<(const PipeOccKey &o) const {
    return std::tie(dev, k, smem, nt) < std::tie(o.dev, o.k, o.smem, o.nt);
  }
};
std::mutex g_occ_mutex;
std::map<PipeOccKey, PipeOcc> g_occ;
bool pipe_occ_lookup(int dev, const void *k, size_t smem, int nt, PipeOcc &o) {
  std::lock_guard<std::mutex> lk(g_occ_mutex);
  auto it = g_occ.find(PipeOccKey{dev, k, smem, nt});
  if (it == g_occ.end()) return false;
  o = it->second;
  return true;
}
void pipe_occ_store(int dev, const void *k, size_t smem, int nt, const PipeOcc &o) {
  std::lock_guard<std::mutex> lk(g_occ_mutex);
  g_occ[PipeOccKey{dev, k, smem, nt}] = o;
}

template <typename T, typename R, class CF>
cudaError_t prer_rc_go(const T *G, T *C, const Geometry &g, const RcDir<R> &tr,
                       unsigned int *err, cudaStream_t st) {
  const int nt = rc2_threads<CF>(tr.S);
  if (tr.N != g.nr || nt > CF::NT || tr.L != CF::L) return cudaErrorInvalidValue;
  // bulk rows: 16-byte rows of G and C, 16-byte aligned slices
  if (rc_bulk_rows<CF>() &&
      ((g.gp * sizeof(T)) % 16 != 0 || (g.pc * sizeof(T)) % 16 != 0 ||
       reinterpret_cast<uintptr_t>(G) % 16 != 0 || reinterpret_cast<uintptr_t>(C) % 16 != 0))
    return cudaErrorInvalidValue;
  const int M = tr.N + 2;
  const size_t smem =
      al16(2 * (size_t)tr.S * CF::LN * sizeof(R)) +
      (size_t)CF::LN * rc_tile_pitch_rows(M, g.gp, g.pc, sizeof(T), CF::LN) * sizeof(T);
  if constexpr (rc_bulk_rows<CF>()) {
    {
      // persistent blocks, as many as fit on the device at once
      const size_t psmem = al16(2 * (size_t)tr.S * CF::LN * sizeof(R)) +
                           (size_t)RC_PIPE_TILES * CF::LN *
                               rc_tile_pitch_rows(M, g.gp, g.pc, sizeof(T), CF::LN) * sizeof(T);
      auto kp = prer_pipe_kernel<T, R, CF>;
      int dev = 0;
      cudaError_t e;
      if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
      // blocks per SM of the persistent kernel for this tile size, found once
      // per device (occupancy queries cost host time at every step otherwise)
      PipeOcc o;
      if (!pipe_occ_lookup(dev, (const void *)kp, psmem, nt, o)) {
        int smax = 0;
        if ((e = cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
            cudaSuccess)
          return e;
        // four tiles of long FP64 rows (1025 columns: 272 KB) do not fit a
        // block: the plain kernel below then takes the rows
        if (psmem <= (size_t)smax) {
          if ((e = rc_attr(kp, psmem)) != cudaSuccess) return e;
          if ((e = cudaDeviceGetAttribute(&o.nsm, cudaDevAttrMultiProcessorCount, dev)) !=
              cudaSuccess)
            return e;
          if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per, kp, nt, psmem)) !=
              cudaSuccess)
            return e;
        }
        pipe_occ_store(dev, (const void *)kp, psmem, nt, o);
      } else if (o.per >= CF::MINB && (e = rc_attr(kp, psmem)) != cudaSuccess) {
        return e;
      }
      const int nsm = o.nsm, per = o.per;
      // only where it keeps the plain kernel's blocks per SM (four FP64
      // tiles of a 513-column row group hold one block per SM)
      if (per >= CF::MINB) {
        const int gps = (g.nu + 2 + CF::LN - 1) / CF::LN;
        const int ngroups = gps * g.nb;
        const int blocks = std::max(1, std::min(ngroups, nsm * per));
        kp<<<blocks, nt, psmem, st>>>(G, C, g, tr, err, gps, ngroups);
        return cudaGetLastError();
      }
    }
  }
  const dim3 grid((g.nu + 2 + CF::LN - 1) / CF::LN, g.nb);
  auto k = prer_rc_kernel<T, R, CF>;
  cudaError_t e = rc_attr(k, smem);
  if (e != cudaSuccess) return e;
  k<<<grid, nt, smem, st>>>(G, C, g, tr, err);
  return cudaGetLastError();
}

// ----------------------------------------------------------- adjoint
// Transposed natural-BC solve (the adjoint of the forward solve above, read
// backwards): for c̄ at rows 0..M-1, x̄ at the data rows 1..N is
//   ascending   e_1 = c̄_1 - a01 c̄_0, e_2 = c̄_2 - a02 c̄_0 - q_1 e_1,
//               e_k = c̄_k - q_{k-1} e_{k-1};  c̄_{M-1} -= q_N e_N
//   last row    d̄_{N-1} = e_{N-1} - (hi2/L2) c̄_{M-1},  d̄_N = e_N - (L1/L2) c̄_{M-1}
//   descending  f_N = d̄_N,  f_k = d̄_k + m_{k+1} f_{k+1}  (m = -rp/6)
//   x̄_k = rp_k f_k
// in the same chunked form: local recurrences from zero corrected by carries.
// The ascending carry enters a chunk through the factor -q at the row before
// it (q_{16} for the second chunk, a table value; the limit beyond).  v holds
// c̄ of the chunk's rows on entry and x̄ on exit; c0b (first chunk) and cMb
// (last chunk) are c̄_0 and c̄_{M-1}.  Lines of at least two chunks only
// (rc_adj_supported); shorter lines use the one-thread-per-line kernels.
template <class C>
__device__ __forceinline__ double adj_first_factor(int s, const RcDir<double> &t) {
  const int k = s * C::L;  // the row before chunk s
  return -t.q0[k < 31 ? k : 31];
}

template <class C>
__device__ __forceinline__ void rc_solve_adj(double (&v)[C::L], const Role &ro, double *E,
                                             double *F, const RcDir<double> &t, double c0b,
                                             double cMb_in) {
  constexpr int L = C::L, LN = C::LN;
  const int S = t.S, N = t.N;
  const int s = ro.s;
  const int kfirst = 1 + s * L;
  const int slot = s * LN + ro.ln;
  // ---------------------------------------------------------- phase A
  if (s == 0) {
    v[0] -= t.a01 * c0b;
    if (N >= 2) v[1] -= t.a02 * c0b;
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
      e = rfma(-t.q0[i], e, v[i]);  // factor -q_{k-1}, k = 1 + i
      v[i] = e;
    }
    if (ro.active && S >= 2) E[slot] = e;
  } else {
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
      e = rfma(-t.q_inf, e, v[i]);
      v[i] = e;
    }
    if (ro.active && s <= S - 2) E[slot] = e;
  }
  __syncthreads();
  // ---------------------------------------------------------- phase B
  if (ro.active) {
    if (s > 0) {
      double ein = E[slot - LN];
      if (s >= 2) ein = rfma(adj_first_factor<C>(s - 1, t) * t.qpow[L - 1], E[slot - 2 * LN], ein);
      const double af = adj_first_factor<C>(s, t) * ein;
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.qpow[i], af, v[i]);
      double fk = 0.0;
      if (s == S - 1) {
        const int iN = N - kfirst;  // 0 .. L-1
        double eN = v[0];
#pragma unroll
        for (int i = 1; i < L; ++i)
          if (i == iN) eN = v[i];
        const double cMb = cMb_in - t.q0[N < 31 ? N : 31] * eN;
        const double Bn = -(t.L1 / t.L2) * cMb, Bp = -(t.hi2 / t.L2) * cMb;
#pragma unroll
        for (int i = 0; i < L; ++i) {
          if (i == iN) v[i] += Bn;
          if (i + 1 == iN) v[i] += Bp;
        }
#pragma unroll
        for (int i = L - 1; i >= 0; --i)
          if (i <= iN) {
            fk = (i == iN) ? v[i] : rfma(t.m_inf, fk, v[i]);
            v[i] = fk;
          }
        // with one row here, d̄_{N-1} belongs to the previous chunk: pass its
        // term through the carry (m T' = m T + Bp)
        F[slot] = v[0] + (iN == 0 ? Bp / t.m_inf : 0.0);
      } else {
#pragma unroll
        for (int i = L - 1; i >= 0; --i) {
          fk = rfma(t.m_inf, fk, v[i]);
          v[i] = fk;
        }
        F[slot] = fk;
      }
    }
  }
  __syncthreads();
  // ---------------------------------------------------------- phase C
  if (ro.active && S >= 2 && s <= S - 2) {
    double T = F[slot + LN];
    if (s + 2 <= S - 1) T = rfma(t.mpow[L], F[slot + 2 * LN], T);
    if (s == 0) {
      double fk = T;
#pragma unroll
      for (int i = L - 1; i >= 0; --i) {
        fk = rfma(t.m0[i + 2], fk, v[i]);
        v[i] = fk;
      }
    } else {
#pragma unroll
      for (int i = 0; i < L; ++i) v[i] = rfma(t.mpow[L - i], T, v[i]);
    }
  }
  // x̄ = rp f
  if (s == 0) {
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] *= t.rp0[i + 1];
  } else {
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] *= t.rp_inf;
  }
}

// adjoint of the kick weights: w_m(fr) and dw_m/dfr
__device__ __forceinline__ void adj_kick_weights(double fr, double w[4], double dw[4]) {
  const double a = 1.0 - fr;
  w[0] = w_bv2<double>(a) / 6.0;
  w[1] = w_bv1<double>(a) / 6.0;
  w[2] = w_bv1<double>(fr) / 6.0;
  w[3] = w_bv2<double>(fr) / 6.0;
  dw[0] = -3.0 * a * a / 6.0;
  dw[1] = -(3.0 + 6.0 * a - 9.0 * a * a) / 6.0;
  dw[2] = (3.0 + 6.0 * fr - 9.0 * fr * fr) / 6.0;
  dw[3] = 3.0 * fr * fr / 6.0;
}

// u lines of the adjoint step, per (16 r columns, J slice):
//   g = P_u f_n          (recomputed; kept in shared memory GS)
//   f̄' = P_u^T Ḡ        (rows of the kicked values)
//   ḡ = Kick^T f̄', s̄   (gather in shift-fraction form, or shared-memory
//                          scatter when a column takes the exact per-row path)
//   λ = P_u^T ḡ
template <typename T, class CF>
__global__ void __launch_bounds__(CF::NT, CF::MINB)
    ucol_adj_rc_kernel(const T *__restrict__ f, const double *__restrict__ Gb,
                       double *__restrict__ lam, double *__restrict__ sbar,
                       const double *__restrict__ shift, Geometry g,
                       const __grid_constant__ RcDir<double> t) {
  constexpr int L = CF::L, LN = CF::LN;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = t.S, N = t.N;  // N == g.nu
  const int M = N + 2;
  double *E = reinterpret_cast<double *>(smem_raw);
  double *F = E + S * LN;
  double *GS = F + S * LN;              // (M + 1) rows x LN
  double *FB = GS + (size_t)(M + 1) * LN;  // N rows x LN
  const Role ro = rc_role<CF>(S);
  const int r = blockIdx.x * LN + ro.ln;
  const bool colok = r < g.nr;
  const int j = blockIdx.y;
  const int kfirst = 1 + ro.s * L;
  const int rc = colok ? r : g.nr - 1;
  double v[L];
  // 1. g = P_u f_n
  {
    const T *fc = f + (size_t)j * N * g.nr + rc;
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = (double)__ldg(fc + (size_t)(min(kfirst + i, N) - 1) * g.nr);
  }
  double c0 = 0.0, cM = 0.0;
  rc_solve<double, CF>(v, ro, E, F, t, c0, cM);
  if (ro.active) {
#pragma unroll
    for (int i = 0; i < L; ++i)
      if (kfirst + i <= N) GS[(kfirst + i) * LN + ro.ln] = v[i];
    if (ro.s == 0) GS[ro.ln] = c0;
    if (ro.s == S - 1) {
      GS[(M - 1) * LN + ro.ln] = cM;
      GS[M * LN + ro.ln] = 0.0;
    }
  }
  // 2. f̄' = P_u^T Ḡ
  const double *Gc = Gb + (size_t)j * M * g.nr + rc;
#pragma unroll
  for (int i = 0; i < L; ++i) v[i] = Gc[(size_t)min(kfirst + i, N) * g.nr];
  const double c0b = ro.s == 0 ? Gc[0] : 0.0;
  const double cMb = ro.s == S - 1 ? Gc[(size_t)(M - 1) * g.nr] : 0.0;
  __syncthreads();  // E, F reused
  rc_solve_adj<CF>(v, ro, E, F, t, c0b, cMb);
  if (ro.active) {
#pragma unroll
    for (int i = 0; i < L; ++i)
      if (kfirst + i <= N) FB[(kfirst + i - 1) * LN + ro.ln] = v[i];
  }
  __syncthreads();
  // 3. kick, transposed
  const double sft = colok ? __ldg(shift + r) : 0.0;
  const double qf = sft * g.hu;
  const double fl = floor(qf);
  const double frd = qf - fl;
  const bool fast = frd > 1e-9 && frd < 1.0 - 1e-9 && fabs(qf) < 1e6;
  double w[4], dw[4];
  adj_kick_weights(frd, w, dw);
  const int o = (int)fl;
  // inside rows of the fraction form, clipped to the grid's rows
  const int ulo = fast ? max((int)floor(-qf) + 1, 0) : 0;
  const int uhi = fast ? min((int)ceil((double)(N - 1) - qf) - 1, N - 1) : -1;
  double sb = 0.0;
  double g0 = 0.0, gM = 0.0;
  // gather when every column of the block is in fraction form
  const bool scatter = __syncthreads_or(ro.active && colok && !fast);
  if (!scatter) {
    // Fraction form, from registers: row u of f̄' (u in [ulo, uhi], else 0)
    // kicks to rows u + o .. u + o + 3 of g.  The thread's own rows
    // u = kfirst - 1 + i are in v; the taps of the derivative, g rows
    // kfirst - 1 + o + t (t = 0 .. L + 2), and the rows of f̄' the gather
    // reads, kfirst - o - 3 + t, are read once each, in order (outside
    // [0, M] the g index is clamped: its f̄' factor is zero there).
    const int gb = kfirst - 1 + o;
    auto gtap = [&](int t) { return GS[min(max(gb + t, 0), M) * LN + ro.ln]; };
    double t0 = gtap(0), t1 = gtap(1), t2 = gtap(2);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      const double t3 = gtap(i + 3);
      const int u = kfirst - 1 + i;
      const double fb = (u >= ulo && u <= uhi) ? FB[u * LN + ro.ln] : 0.0;
      sb = rfma(fb, dw[0] * t0 + dw[1] * t1 + dw[2] * t2 + dw[3] * t3, sb);
      t0 = t1;
      t1 = t2;
      t2 = t3;
    }
    const int fbase = kfirst - o - 3;
    auto ftap = [&](int t) {
      const int u = fbase + t;
      return (u >= ulo && u <= uhi) ? FB[u * LN + ro.ln] : 0.0;
    };
    double a0 = ftap(0), a1 = ftap(1), a2 = ftap(2);
#pragma unroll
    for (int i = 0; i < L; ++i) {
      // row k = kfirst + i takes f̄' rows k - o - m, m = 0 .. 3
      const double a3 = ftap(i + 3);
      v[i] = w[0] * a3 + w[1] * a2 + w[2] * a1 + w[3] * a0;
      a0 = a1;
      a1 = a2;
      a2 = a3;
    }
    if (ro.s == 0)
      for (int m = 0; m < 4; ++m) {
        const int u = 0 - o - m;
        if (u >= ulo && u <= uhi) g0 += w[m] * FB[u * LN + ro.ln];
      }
    if (ro.s == S - 1)
      for (int m = 0; m < 4; ++m) {
        const int u = M - 1 - o - m;
        if (u >= ulo && u <= uhi) gM += w[m] * FB[u * LN + ro.ln];
      }
  } else {
    // shift derivative: sum over this thread's kicked rows
    if (ro.active) {
#pragma unroll 1
      for (int i = 0; i < L; ++i) {
        const int u = kfirst + i - 1;
        if (u >= N) break;
        const double fb = FB[u * LN + ro.ln];
        if (fast) {
          if (u < ulo || u > uhi) continue;
          const double *gp = GS + (ptrdiff_t)(u + o) * LN + ro.ln;
          sb += fb * (dw[0] * gp[0] + dw[1] * gp[LN] + dw[2] * gp[2 * LN] + dw[3] * gp[3 * LN]);
        } else {
          const double newU = __ldg(g.U + u) + sft;
          if (!(newU > g.u0 && newU < g.umax)) continue;
          const double y = (newU - g.su) * g.hu;
          const double yf = floor(y);
          double ww[4], dd[4];
          adj_kick_weights(y - yf, ww, dd);
          const int Ny = 1 + (int)yf;
          for (int m = 0; m < 4; ++m)
            if (Ny - 1 + m < M) sb += fb * dd[m] * GS[(Ny - 1 + m) * LN + ro.ln];
        }
      }
    }
    // shared-memory scatter into GS (g is no longer needed)
    __syncthreads();
    for (int e = threadIdx.x; e < (M + 1) * LN; e += blockDim.x) GS[e] = 0.0;
    __syncthreads();
    if (ro.active) {
#pragma unroll 1
      for (int i = 0; i < L; ++i) {
        const int u = kfirst + i - 1;
        if (u >= N) break;
        const double fb = FB[u * LN + ro.ln];
        if (fast) {
          if (u < ulo || u > uhi) continue;
          for (int m = 0; m < 4; ++m) atomicAdd(&GS[(u + o + m) * LN + ro.ln], w[m] * fb);
        } else {
          const double newU = __ldg(g.U + u) + sft;
          if (!(newU > g.u0 && newU < g.umax)) continue;
          const double y = (newU - g.su) * g.hu;
          const double yf = floor(y);
          double ww[4], dd[4];
          adj_kick_weights(y - yf, ww, dd);
          const int Ny = 1 + (int)yf;
          for (int m = 0; m < 4; ++m)
            if (Ny - 1 + m < M) atomicAdd(&GS[(Ny - 1 + m) * LN + ro.ln], ww[m] * fb);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < L; ++i) v[i] = GS[min(kfirst + i, M) * LN + ro.ln];
    g0 = GS[ro.ln];
    gM = GS[(M - 1) * LN + ro.ln];
  }
  sb *= g.hu;
  // s̄ of the column, summed over its chunks in chunk order
  __syncthreads();
  if (ro.active) F[ro.s * LN + ro.ln] = sb;
  __syncthreads();
  if (ro.active && ro.s == 0 && colok) {
    double tot = 0.0;
    for (int c = 0; c < S; ++c) tot += F[c * LN + ro.ln];
    sbar[(size_t)j * g.nr + r] = tot;
  }
  __syncthreads();
  // 4. λ = P_u^T ḡ (ḡ in v)
  rc_solve_adj<CF>(v, ro, E, F, t, ro.s == 0 ? g0 : 0.0, ro.s == S - 1 ? gM : 0.0);
  if (ro.active && colok) {
    double *lc = lam + (size_t)j * N * g.nr + r;
#pragma unroll
    for (int i = 0; i < L; ++i)
      if (kfirst + i <= N) lc[(size_t)(kfirst + i - 1) * g.nr] = v[i];
  }
}

// r lines of the adjoint step: rows of C̄ (all slices) -> P_r^T -> rows of Ḡ
template <class CF>
__global__ void __launch_bounds__(CF::NT, CF::MINB)
    prer_adj_rc_kernel(const double *__restrict__ Cb, double *__restrict__ Gb, Geometry g,
                       const __grid_constant__ RcDir<double> t) {
  constexpr int L = CF::L, LN = CF::LN;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int S = t.S, N = t.N;  // N == g.nr
  const int M = N + 2;
  const int P = rc_tile_pitch(M, sizeof(double), LN);
  double *E = reinterpret_cast<double *>(smem_raw);
  double *F = E + S * LN;
  double *tile = reinterpret_cast<double *>(smem_raw + al16(2 * (size_t)S * LN * sizeof(double)));
  const Role ro = rc_role<CF>(S);
  const int j = blockIdx.y;
  const int rows = g.nu + 2;
  const int kr0 = blockIdx.x * LN;
  const int nrow = min(LN, rows - kr0);
  const double *Cs = Cb + ((size_t)j * (g.nu + 3) + kr0) * g.pc;
  for (int p = 0; p < nrow; ++p)
    for (int k = threadIdx.x; k < M; k += blockDim.x)
      cp_async_el(tile + p * P + k, Cs + (size_t)p * g.pc + k);
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  const int kfirst = 1 + ro.s * L;
  double v[L];
  const double *row = tile + ro.ln * P;
#pragma unroll
  for (int i = 0; i < L; ++i) v[i] = row[min(kfirst + i, N)];
  const double c0b = ro.s == 0 ? row[0] : 0.0;
  const double cMb = ro.s == S - 1 ? row[M - 1] : 0.0;
  __syncthreads();  // every thread has its chunk before rows are overwritten
  rc_solve_adj<CF>(v, ro, E, F, t, c0b, cMb);
  if (ro.active && ro.ln < nrow) {
    double *wr = tile + ro.ln * P;
#pragma unroll
    for (int i = 0; i < L; ++i)
      if (kfirst + i <= N) wr[kfirst + i] = v[i];
  }
  __syncthreads();
  double *Gs = Gb + ((size_t)j * rows + kr0) * g.nr;
  for (int p = 0; p < nrow; ++p)
    for (int k = threadIdx.x; k < N; k += blockDim.x) Gs[(size_t)p * g.nr + k] = tile[p * P + 1 + k];
}

// u lines: 15-row chunks in 8-line blocks (up to 70 chunks; 12 % faster than
// 16-line blocks on 513-row lines, and 0.835 against 1.193 ms per
// transposed step for 4-line blocks on 1025 x 1025 x 64); r lines: 15-row
// chunks in 8-line blocks up to 38 chunks, longer lines in 4-line blocks of
// up to 82 chunks (two blocks of 320 threads per SM on 1025-row lines: 0.284
// against 0.332 ms per transposed step on 1025 x 1025 x 64 for one block of
// 8 lines)
using CfgAdjU = RcCfg<15, 8, 576, 1>;
using CfgAdjR = RcCfg<15, 8, 320, 2>;
using CfgAdjR2 = RcCfg<15, 4, 352, 1>;

}  // namespace

// ------------------------------------------------------------- host side
// configuration for one direction (u_lines: the ucol kernel's columns, else
// the prer kernel's rows), -1 when no configuration takes the shape (the
// shared-memory segment kernels then solve the lines).  Ids: 2 = B (15-row
// chunks, 8 lines), 3 = B1 (the same, one block per SM), 4 = C (15-row, 16
// lines), 5 = D (23-row, 8 lines), 6 = F (19-row, 8 lines), 7 = I (17-row,
// 16 lines).
template <typename R>
int rc_config(const HostDirTables &t, bool u_lines) {
  const int N = t.M - 2;
  const int kc = sizeof(R) == 8 ? t.kc64 : t.kc32;
  const int b = cfg2_fits<CfgB>(N, kc) ? 2 : cfg2_fits<CfgB1>(N, kc) ? 3 : -1;
  // the fastest measured on 513 x 513 x 256: 16-line blocks of 17-row
  // chunks for the u lines (15, 19 and 23 rows measured 1 %, 3 % and 28 %
  // slower), 8-line blocks of 19-row chunks for the r lines (prer 0.142 ->
  // 0.120 ms against 15-row chunks; 17 and 21 rows 0.130 and 0.128 ms);
  // lines too long for those take 23-row chunks with two blocks per SM
  // (1025-row lines: ucol 2.85 -> 1.85 ms, prer 1.17 -> 0.97 ms against
  // 15-row chunks at one block per SM)
  if (u_lines && cfg2_fits<CfgI>(N, kc)) return 7;
  if (u_lines && cfg2_fits<CfgC>(N, kc)) return 4;
  if (!u_lines && cfg2_fits<CfgF>(N, kc)) return 6;
  if (cfg2_fits<CfgB>(N, kc)) return 2;
  if (cfg2_fits<CfgD>(N, kc)) return 5;
  return b;
}

static int cfg_L(int cfg) {
  switch (cfg) {
    case 5:
      return CfgD::L;
    case 6:
      return CfgF::L;
    case 7:
      return CfgI::L;
    default:
      return CfgB::L;
  }
}

template <typename R>
RcDir<R> rc_dir(const HostDirTables &t, int cfg) {
  RcDir<R> o{};
  const int M = t.M, N = M - 2;
  const int L = cfg_L(cfg < 0 ? 0 : cfg);
  const double sixth = 1.0 / 6.0;
  for (int k = 0; k < 32; ++k) {
    const double rp = (k >= 1 && k <= M - 2) ? t.rp[k] : t.rp_inf;
    const double q = (k >= 1 && k <= M - 2) ? t.q[k] : t.q_inf;
    o.rp0[k] = (R)rp;
    o.m0[k] = (R)(-(sixth * rp));
    o.q0[k] = (R)q;
  }
  o.rp_inf = (R)t.rp_inf;
  o.m_inf = (R)(-(sixth * t.rp_inf));
  o.q_inf = (R)t.q_inf;
  const double m = -(sixth * t.rp_inf);
  double pm = 1.0, pq = 1.0;
  for (int i = 0; i <= 32; ++i) {
    o.mpow[i] = (R)pm;
    o.qpow[i] = (R)pq;
    pm *= m;
    pq *= -t.q_inf;
  }
  // first chunk's backward correction factors prod_{k=i}^{L-1} (-q_{1+k})
  {
    double pf = 1.0;
    for (int i = 31; i >= 0; --i) {
      if (i < L) {
        const int k = 1 + i;
        const double q = (k >= 1 && k <= M - 2) ? t.q[k] : t.q_inf;
        pf *= -q;
        o.qfirst[i] = (R)pf;
      } else {
        o.qfirst[i] = (R)0;
      }
    }
  }
  o.a01 = (R)t.a01;
  o.a02 = (R)t.a02;
  o.hi2 = (R)t.hi2;
  o.L1 = (R)t.L1;
  o.L2 = (R)t.L2;
  o.inv_L2 = (R)(1.0 / t.L2);
  o.N = N;
  o.L = L;
  o.S = (N + L - 1) / L;
  return o;
}

template <typename T, typename R>
cudaError_t launch_ucol_rc(int cfg, bool kick, const T *f, T *G, const double *shift,
                           const Geometry &g, const RcDir<R> &tu, cudaStream_t st) {
#define VLS_UCOL_CFG(ID, CF)                                                    \
  case ID:                                                                      \
    return kick ? ucol_rc_go<T, R, true, CF>(f, G, shift, g, tu, st)            \
                : ucol_rc_go<T, R, false, CF>(f, G, shift, g, tu, st);
  switch (cfg) {
    VLS_UCOL_CFG(2, CfgB)
    VLS_UCOL_CFG(3, CfgB1)
    VLS_UCOL_CFG(4, CfgC)
    VLS_UCOL_CFG(5, CfgD)
    VLS_UCOL_CFG(6, CfgF)
    VLS_UCOL_CFG(7, CfgI)
    default:
      return cudaErrorInvalidValue;
  }
#undef VLS_UCOL_CFG
}

template <typename T, typename R>
cudaError_t launch_prer_rc(int cfg, const T *G, T *C, const Geometry &g, const RcDir<R> &tr,
                           unsigned int *err, cudaStream_t st) {
  switch (cfg) {
    case 2:
      return prer_rc_go<T, R, CfgB>(G, C, g, tr, err, st);
    case 3:
      return prer_rc_go<T, R, CfgB1>(G, C, g, tr, err, st);
    case 4:
      return prer_rc_go<T, R, CfgC>(G, C, g, tr, err, st);
    case 5:
      return prer_rc_go<T, R, CfgD>(G, C, g, tr, err, st);
    case 6:
      return prer_rc_go<T, R, CfgF>(G, C, g, tr, err, st);
    case 7:
      return prer_rc_go<T, R, CfgI>(G, C, g, tr, err, st);
    default:
      return cudaErrorInvalidValue;
  }
}

// adjoint line kernels (FP64), layouts CfgAdjU / CfgAdjR / CfgAdjR2; tables
// from rc_dir<double>(t, 2)
bool rc_adj_supported(const HostDirTables &tu, const HostDirTables &tr) {
  return tu.M - 2 > CfgAdjU::L && tr.M - 2 > CfgAdjR::L &&
         cfg_fits<CfgAdjU>(tu.M - 2, tu.kc64) &&
         (cfg_fits<CfgAdjR>(tr.M - 2, tr.kc64) || cfg_fits<CfgAdjR2>(tr.M - 2, tr.kc64));
}

template <typename T, class CF>
static cudaError_t ucol_adj_go(const T *f, const double *Gb, double *lam, double *sbar,
                               const double *shift, const Geometry &g, const RcDir<double> &tu,
                               cudaStream_t st) {
  const int nt = rc_threads<CF>(tu.S);
  if (tu.N != g.nu || nt > CF::NT || tu.L != CF::L) return cudaErrorInvalidValue;
  const int M = tu.N + 2;
  const size_t smem = 2 * (size_t)tu.S * CF::LN * sizeof(double) +
                      (size_t)(M + 1 + tu.N) * CF::LN * sizeof(double);
  auto k = ucol_adj_rc_kernel<T, CF>;
  cudaError_t e = rc_attr(k, smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((g.nr + CF::LN - 1) / CF::LN, g.nj);
  k<<<grid, nt, smem, st>>>(f, Gb, lam, sbar, shift, g, tu);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ucol_adj_rc(const T *f, const double *Gb, double *lam, double *sbar,
                               const double *shift, const Geometry &g, const RcDir<double> &tu,
                               cudaStream_t st) {
  return ucol_adj_go<T, CfgAdjU>(f, Gb, lam, sbar, shift, g, tu, st);
}

template <class CF>
static cudaError_t prer_adj_go(const double *Cb, double *Gb, const Geometry &g,
                               const RcDir<double> &tr, cudaStream_t st) {
  const int nt = rc_threads<CF>(tr.S);
  if (tr.N != g.nr || nt > CF::NT || tr.L != CF::L) return cudaErrorInvalidValue;
  const int M = tr.N + 2;
  const size_t smem = al16(2 * (size_t)tr.S * CF::LN * sizeof(double)) +
                      (size_t)CF::LN * rc_tile_pitch(M, sizeof(double), CF::LN) * sizeof(double);
  auto k = prer_adj_rc_kernel<CF>;
  cudaError_t e = rc_attr(k, smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((g.nu + 2 + CF::LN - 1) / CF::LN, g.nj);
  k<<<grid, nt, smem, st>>>(Cb, Gb, g, tr);
  return cudaGetLastError();
}

cudaError_t launch_prer_adj_rc(const double *Cb, double *Gb, const Geometry &g,
                               const RcDir<double> &tr, cudaStream_t st) {
  if (tr.S <= rc_maxs<CfgAdjR>()) return prer_adj_go<CfgAdjR>(Cb, Gb, g, tr, st);
  return prer_adj_go<CfgAdjR2>(Cb, Gb, g, tr, st);
}

template cudaError_t launch_ucol_adj_rc<float>(const float *, const double *, double *, double *,
                                               const double *, const Geometry &,
                                               const RcDir<double> &, cudaStream_t);
template cudaError_t launch_ucol_adj_rc<double>(const double *, const double *, double *,
                                                double *, const double *, const Geometry &,
                                                const RcDir<double> &, cudaStream_t);

#define VLS_RC_INST(T, R)                                                                 \
  template cudaError_t launch_ucol_rc<T, R>(int, bool, const T *, T *, const double *,   \
                                            const Geometry &, const RcDir<R> &,          \
                                            cudaStream_t);                               \
  template cudaError_t launch_prer_rc<T, R>(int, const T *, T *, const Geometry &,       \
                                            const RcDir<R> &, unsigned int *, cudaStream_t);
VLS_RC_INST(double, double)
VLS_RC_INST(float, double)
VLS_RC_INST(float, float)
template int rc_config<double>(const HostDirTables &, bool);
template int rc_config<float>(const HostDirTables &, bool);
int rc_chunk_rows(int cfg) { return cfg < 0 ? 0 : cfg_L(cfg); }
template RcDir<double> rc_dir<double>(const HostDirTables &, int);
template RcDir<float> rc_dir<float>(const HostDirTables &, int);

}  // namespace vls
