// vls_profile.cu -- the analytic initial distribution functions on the
// device, for the derivative of the initial state with respect to the
// profile parameters that the adjoint's users take by central differences.
//
// The formulas are Profile::value's (vls_setup.cpp, after
// initGen_UniformDensitySphere.hxx:158-173, initGen_PowerLawDensitySphere.hxx
// :181-189, initGen_Plummer.hxx:126-131, initGen_Hernquist.hxx:133-155),
// evaluated with the device's FP64 math functions.  The initial grid itself
// comes from that host code, bit for bit as the reference makes it; the
// grids here differ from it in the last bits, which a central difference
// over a 1e-6 relative step does not resolve.  Every sum is taken in a
// fixed order.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/vlasolve_b200.h"
#include "vls_internal.h"

namespace vls {

namespace {

__device__ double profile_value(const ProfileConsts &p, double r, double u, double j) {
  switch (p.type) {
    case VLS_INIT_UDF: {
      const double sm = 0.5 * (1. + erf((p.R0 - r) / p.smoothingRadius));
      double res = sm * p.C1 * exp(-(u * u + (j * j) / (r * r)) / p.C2);
      if (p.gap1 > 0) {
        const double sm0 = 0.5 * (1. + erf((p.gap0 - r) / 0.15));
        const double sm1 = 0.5 * (1. + erf(-(p.gap1 - r) / 0.15));
        res *= (sm0 + sm1);
      }
      return res < 1.E-200 ? 1.E-200 : res;
    }
    case VLS_INIT_PLDF: {
      const double sm = 0.5 * (1. + erf((p.R0 - r) / p.smoothingRadius));
      const double res =
          sm * p.C0 * exp(-u * u * p.C1 - ((j * j) / (r * r)) * p.C2) * pow(r, -p.n);
      return res < 1.E-200 ? 1.E-200 : res;
    }
    case VLS_INIT_PLUMMER: {
      const double phi = -(p.G * p.M) / sqrt(r * r + p.R0 * p.R0);
      const double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      if (eps >= 0) return 0;
      return pow(-2. * eps, 3.5) * (3. / (M_PI * M_PI * M_PI * 7.));
    }
    case VLS_INIT_HERNQUIST: {
      const double phi = -(p.G * p.M) / (p.R0 + r);
      double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      if (p.Ra > 0) eps = eps + (j * j) / (2 * p.Ra * p.Ra);
      if (eps >= 0) return 0;
      const double q = sqrt(-(p.R0) / (p.G * p.M) * eps);
      const double q2 = q * q;
      double A1 = (p.M) / (8. * sqrt(2.) * pow(M_PI * p.R0 * p.Vg, 3.)) * pow(1. - q2, -2.5);
      double A2 = 3 * asin(q) + q * sqrt(1. - q2) * (1. - 2 * q2) * (8 * q2 * q2 - 8 * q2 - 3);
      double result = A1 * A2;
      if (p.Ra > 0) {
        A1 = (p.M) / (sqrt(2.) * pow(M_PI * p.R0 * p.Vg, 3)) * pow(p.R0 / p.Ra, 2);
        A2 = q * (1. - 2 * q2);
        result += A1 * A2;
      }
      return result;
    }
  }
  return 0;
}

// f of every cell, [j][u][r]; xyz: R (nr), U (nu), J (nj)
__global__ void profile_grid_kernel(ProfileConsts p, const double *__restrict__ xyz,
                                    double *__restrict__ f, int nr, int nu, int nj) {
  const size_t n = (size_t)nr * nu * nj;
  const double *R = xyz, *U = xyz + nr, *J = xyz + nr + nu;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i % nr);
    const size_t ju = i / nr;
    const int u = (int)(ju % nu), j = (int)(ju / nu);
    f[i] = profile_value(p, __ldg(R + r), __ldg(U + u), __ldg(J + j));
  }
}

// The mass quadrature of vls_init_profile (quadrature21.hxx:56-85) per (j,
// u) row, one warp per row: rows[j nu + u] = 8 pi^2 J_j dJ_j dU_u sum_r dR_r
// (f at the cell's 4 corners) / 4, the lanes' sums added by shuffles in a
// fixed order.  xyz: R, U, J, then JV (nj + 1).
__global__ void profile_rows_kernel(const double *__restrict__ f,
                                    const double *__restrict__ xyz, double *__restrict__ rows,
                                    int nr, int nu, int nj) {
  const double *R = xyz, *U = xyz + nr, *J = xyz + nr + nu, *JV = xyz + nr + nu + nj;
  const int lane = threadIdx.x & 31;
  const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (row >= nu * nj) return;  // the whole warp
  const int u = row % nu, j = row / nu;
  const double dU = (u >= nu - 1) ? 0 : (U[u + 1] - U[u]);
  const double dJ = (j >= nu - 1) ? 0 : (JV[j + 1] - JV[j]);
  double s = 0.0;
  if (dU > 0) {
    const double *fr = f + ((size_t)j * nu + u) * nr;
    for (int r = lane; r < nr - 1; r += 32) {
      const double dR = R[r + 1] - R[r];
      if (dR > 0) s += dR * ((fr[r] + fr[r + 1] + fr[nr + r] + fr[nr + r + 1]) * 0.25);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) rows[row] = 8 * M_PI * M_PI * J[j] * dJ * dU * s;
}

constexpr int DOT_BLOCKS = 1184, DOT_THREADS = 256;

// partial[b] = sum over block b's cells of w (a fp - b fm), fixed order
__global__ void __launch_bounds__(DOT_THREADS)
    profile_dot_kernel(const double *__restrict__ w, const double *__restrict__ fp,
                       const double *__restrict__ fm, double a, double b, size_t n,
                       double *__restrict__ partial) {
  __shared__ double red[DOT_THREADS];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    s += w[i] * (a * fp[i] - b * fm[i]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = DOT_THREADS / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace

int profile_dot_blocks() { return DOT_BLOCKS; }

cudaError_t launch_profile_grid(const ProfileConsts &p, const double *xyz, double *f, int nr,
                                int nu, int nj, cudaStream_t st) {
  const size_t n = (size_t)nr * nu * nj;
  const size_t b = std::min<size_t>((n + 255) / 256, (size_t)148 * 32);
  profile_grid_kernel<<<(unsigned)(b ? b : 1), 256, 0, st>>>(p, xyz, f, nr, nu, nj);
  return cudaGetLastError();
}

cudaError_t launch_profile_rows(const double *f, const double *xyz, double *rows, int nr,
                                int nu, int nj, cudaStream_t st) {
  const size_t warps = (size_t)nu * nj;
  profile_rows_kernel<<<(unsigned)((warps + 7) / 8), 256, 0, st>>>(f, xyz, rows, nr, nu, nj);
  return cudaGetLastError();
}

cudaError_t launch_profile_dot(const double *w, const double *fp, const double *fm, double a,
                               double b, size_t n, double *partial, cudaStream_t st) {
  profile_dot_kernel<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(w, fp, fm, a, b, n, partial);
  return cudaGetLastError();
}

}  // namespace vls
