// vls_noalloc.cu -- radial moment and enclosed mass of a caller-owned device
// grid, computed without allocating any memory.
//
// Who needs this: applications that own every byte of device memory and hand
// the library only pointers (a host framework with its own pool, or a process
// that reserves its whole memory budget at start-up) cannot let a library
// call cudaMalloc behind their back.  This entry point takes the grid and the
// output buffers from the caller and keeps its working space in one
// file-scope device array of fixed size instead.
//
// Scratch: g_noalloc_scratch, VLS_NOALLOC_SCRATCH_DOUBLES doubles (512 KiB).
// Every GPU that loads this library holds that array until the process exits.
// All calls share it and it keeps the last call's contents; each call
// writes every word it later reads (coordinates, weights, partial sums), so
// nothing needs clearing between calls.  Calls that overlap on the GPU
// (different streams, or different host threads, on one device) race on the
// array and must be serialised by the caller.
//
// The device address of the array is looked up once per device, with that
// device current, on the first call on that device (cudaGetSymbolAddress).
// That first call therefore should come before any stream capture is begun
// on the device.  The address belongs to the device's current context: after
// cudaDeviceReset the next call on that device finds a new context (by its
// context id) and looks the address up again.
//
// Every call copies the coordinate arrays R, U, J and JV from host memory
// into the scratch array with cudaMemcpyAsync on the caller's stream.
//
// Error messages are kept per host thread (vls_noalloc_last_error returns the
// message of the calling thread's last failed call).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/vlasolve_b200.h"

namespace {

constexpr int64_t VLS_NOALLOC_SCRATCH_DOUBLES = 65536;  // 512 KiB
constexpr int NA_MAXN = 2048;  // at most 2048 vertices/cells per direction
constexpr int NA_GROUPS = 16;  // slice groups of the partial sums
constexpr int NA_MAX_DEVICES = 64;

// layout (in doubles): R, U, J, JV (raw coordinates), bu, wj, dR4 (weights),
// partial[NA_GROUPS][nr], T2[nr]
constexpr int64_t OFF_R = 0;
constexpr int64_t OFF_U = OFF_R + NA_MAXN;
constexpr int64_t OFF_J = OFF_U + NA_MAXN;
constexpr int64_t OFF_JV = OFF_J + NA_MAXN;
constexpr int64_t OFF_BU = OFF_JV + NA_MAXN + 1;
constexpr int64_t OFF_WJ = OFF_BU + NA_MAXN;
constexpr int64_t OFF_DR4 = OFF_WJ + NA_MAXN;
constexpr int64_t OFF_PART = OFF_DR4 + NA_MAXN;
constexpr int64_t OFF_T2 = OFF_PART + (int64_t)NA_GROUPS * NA_MAXN;
static_assert(OFF_T2 + NA_MAXN <= VLS_NOALLOC_SCRATCH_DOUBLES, "scratch layout too large");

}  // namespace

static __device__ __align__(256) double g_noalloc_scratch[VLS_NOALLOC_SCRATCH_DOUBLES];

namespace {

std::mutex g_na_mutex;
double *g_na_ptr[NA_MAX_DEVICES] = {nullptr};
unsigned long long g_na_ctx[NA_MAX_DEVICES] = {0};  // context id the address belongs to
thread_local std::string g_na_error;

int na_fail(int code, const std::string &m) {
  g_na_error = m;
  return code;
}

// get_dU / get_dR / get_dJ (slice21Iterator.hxx:84-86) and the radial-bin
// weights of quadrature21::integrate1D (quadrature21.hxx:111-119), rewritten as
// in the step: bins[r] = dR_r/4 (T[r] + T[r+1]), T[r] = sum_j w_j sum_u b_u f
__global__ void na_tables(double *s, int nr, int nu, int nj) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double *R = s + OFF_R, *U = s + OFF_U, *J = s + OFF_J, *JV = s + OFF_JV;
  if (i < nu) {
    const double a = (i >= nu - 1) ? 0.0 : (U[i + 1] - U[i]);
    const double b = (i == 0) ? 0.0 : ((i - 1 >= nu - 1) ? 0.0 : (U[i] - U[i - 1]));
    s[OFF_BU + i] = a + b;
  }
  if (i < nj) {
    const double dJ = (i >= nu - 1) ? 0.0 : (JV[i + 1] - JV[i]);
    s[OFF_WJ + i] = 8 * M_PI * M_PI * J[i] * dJ;
  }
  if (i < nr) s[OFF_DR4 + i] = ((i >= nr - 1) ? 0.0 : (R[i + 1] - R[i])) * 0.25;
}

// block (strip of 32 r columns, slice group g): partial[g][r] = sum over the
// group's slices j (j = g mod NA_GROUPS) and all u of w_j b_u f[j][u][r]
template <typename T>
__global__ void __launch_bounds__(256)
    na_moment(const T *__restrict__ f, double *s, int nr, int nu, int nj) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  const int grp = blockIdx.y;
  const double *bu = s + OFF_BU, *wj = s + OFF_WJ;
  double acc = 0.0;
  if (r < nr)
    for (int j = grp; j < nj; j += NA_GROUPS) {
      double a = 0.0;
      for (int u = w; u < nu; u += 8) a += bu[u] * (double)f[((size_t)j * nu + u) * nr + r];
      acc += wj[j] * a;
    }
  __shared__ double red[8][32];
  red[w][lane] = acc;
  __syncthreads();
  if (w == 0 && r < nr) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += red[k][lane];
    s[OFF_PART + (int64_t)grp * NA_MAXN + r] = t;
  }
}

// compensated (TwoSum) pair arithmetic
struct dd2 {
  double hi, lo;
};
__device__ __forceinline__ dd2 add(dd2 a, dd2 b) {
  const double t = a.hi + b.hi;
  const double bb = t - a.hi;
  double e = (a.hi - (t - bb)) + (b.hi - bb);
  e += a.lo + b.lo;
  const double h = t + e;
  return dd2{h, e - (h - t)};
}

// one block of 1024 threads: T2 from the group partials, bins, exclusive scan
// (enclosed mass strictly inside R_r, grid_handler.hxx:387-407) and total
__global__ void __launch_bounds__(1024)
    na_scan(double *s, int nr, double *bins, double *Mr, double *mtot) {
  __shared__ dd2 wsum[32];
  const int tid = threadIdx.x;
  for (int r = tid; r < nr; r += 1024) {
    dd2 a{0.0, 0.0};
    for (int g = 0; g < NA_GROUPS; ++g) a = add(a, dd2{s[OFF_PART + (int64_t)g * NA_MAXN + r], 0.0});
    s[OFF_T2 + r] = a.hi + a.lo;
  }
  __syncthreads();
  const int per = (nr + 1023) / 1024;  // 1 or 2 consecutive r per thread
  double b[2] = {0.0, 0.0};
  dd2 loc{0.0, 0.0};
  for (int q = 0; q < per; ++q) {
    const int r = tid * per + q;
    if (r < nr) {
      b[q] = (r < nr - 1) ? s[OFF_DR4 + r] * (s[OFF_T2 + r] + s[OFF_T2 + r + 1]) : 0.0;
      bins[r] = b[q];
      loc = add(loc, dd2{b[q], 0.0});
    }
  }
  const int lane = tid & 31, wid = tid >> 5;
  dd2 inc = loc;
  for (int d = 1; d < 32; d <<= 1) {
    dd2 o{__shfl_up_sync(0xffffffffu, inc.hi, d), __shfl_up_sync(0xffffffffu, inc.lo, d)};
    if (lane >= d) inc = add(inc, o);
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const dd2 x = wsum[lane];
    dd2 xi = x;
    for (int d = 1; d < 32; d <<= 1) {
      dd2 o{__shfl_up_sync(0xffffffffu, xi.hi, d), __shfl_up_sync(0xffffffffu, xi.lo, d)};
      if (lane >= d) xi = add(xi, o);
    }
    wsum[lane] = add(xi, dd2{-x.hi, -x.lo});
    if (lane == 31) *mtot = xi.hi + xi.lo;
  }
  __syncthreads();
  dd2 ex = add(wsum[wid], add(inc, dd2{-loc.hi, -loc.lo}));
  for (int q = 0; q < per; ++q) {
    const int r = tid * per + q;
    if (r < nr) {
      Mr[r] = ex.hi + ex.lo;
      ex = add(ex, dd2{b[q], 0.0});
    }
  }
}

// id of the context current on this thread (0 if it cannot be read); the
// driver calls are reached through the runtime, without a libcuda link
unsigned long long current_ctx_id() {
  static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    fn = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(fn);
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// device address of the scratch array on `device`: looked up with the device
// current on the first call, and again when the device's context has changed
// (cudaDeviceReset)
int scratch_on(int device, double **out) {
  if (device < 0 || device >= NA_MAX_DEVICES)
    return na_fail(VLS_EINVAL, "device ordinal out of range");
  const unsigned long long ctx = current_ctx_id();
  std::lock_guard<std::mutex> lk(g_na_mutex);
  if (!g_na_ptr[device] || ctx == 0 || ctx != g_na_ctx[device]) {
    double *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return na_fail(VLS_ECUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch: ") +
                                    cudaGetErrorString(e));
    g_na_ptr[device] = p;
    g_na_ctx[device] = ctx;
  }
  *out = g_na_ptr[device];
  return VLS_OK;
}

}  // namespace

extern "C" const char *vls_noalloc_last_error(void) { return g_na_error.c_str(); }

extern "C" int vls_radial_mass_noalloc(const void *f_dev, int32_t precision, int64_t nr,
                                       int64_t nu, int64_t nj, const double *R,
                                       const double *U, const double *J, const double *JV,
                                       double *bins_dev, double *Mr_dev, double *mtot_dev,
                                       void *stream, int32_t device) {
  if (!f_dev || !R || !U || !J || !JV || !bins_dev || !Mr_dev || !mtot_dev)
    return na_fail(VLS_EINVAL, "vls_radial_mass_noalloc: NULL argument");
  if (precision != VLS_FP64 && precision != VLS_FP32_BULK && precision != VLS_FP32_ALL)
    return na_fail(VLS_EINVAL, "vls_radial_mass_noalloc: unknown precision");
  if (nr < 2 || nu < 2 || nj < 1)
    return na_fail(VLS_EINVAL, "vls_radial_mass_noalloc: grid too small");
  if (nr > NA_MAXN || nu > NA_MAXN || nj > NA_MAXN)
    return na_fail(VLS_EINVAL,
                   "vls_radial_mass_noalloc: grid exceeds the fixed scratch (at most 2048 "
                   "r vertices, 2048 u vertices and 2048 J cells)");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return na_fail(VLS_ECUDA, "vls_radial_mass_noalloc: cudaSetDevice failed");
  }
  int rc = VLS_OK;
  double *s = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  auto ck = [&](cudaError_t e, const char *what) {
    if (rc == VLS_OK && e != cudaSuccess)
      rc = na_fail(VLS_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  rc = scratch_on(device, &s);
  if (rc == VLS_OK) {
    ck(cudaMemcpyAsync(s + OFF_R, R, sizeof(double) * nr, cudaMemcpyHostToDevice, st), "copy R");
    ck(cudaMemcpyAsync(s + OFF_U, U, sizeof(double) * nu, cudaMemcpyHostToDevice, st), "copy U");
    ck(cudaMemcpyAsync(s + OFF_J, J, sizeof(double) * nj, cudaMemcpyHostToDevice, st), "copy J");
    ck(cudaMemcpyAsync(s + OFF_JV, JV, sizeof(double) * (nj + 1), cudaMemcpyHostToDevice, st),
       "copy JV");
  }
  if (rc == VLS_OK) {
    const int n = (int)std::max(nr, std::max(nu, nj));
    na_tables<<<(n + 255) / 256, 256, 0, st>>>(s, (int)nr, (int)nu, (int)nj);
    ck(cudaGetLastError(), "na_tables");
    dim3 grid((unsigned)((nr + 31) / 32), NA_GROUPS);
    if (precision == VLS_FP64)
      na_moment<double><<<grid, 256, 0, st>>>((const double *)f_dev, s, (int)nr, (int)nu,
                                              (int)nj);
    else
      na_moment<float><<<grid, 256, 0, st>>>((const float *)f_dev, s, (int)nr, (int)nu,
                                             (int)nj);
    ck(cudaGetLastError(), "na_moment");
    na_scan<<<1, 1024, 0, st>>>(s, (int)nr, bins_dev, Mr_dev, mtot_dev);
    ck(cudaGetLastError(), "na_scan");
  }
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}
