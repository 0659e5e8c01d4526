// vls_spline.cu -- the spline-level surface of the step: batches of 2D
// natural-BC cubic B-splines (localSpline<2>, localSpline.hxx:60-503) and
// the einspline-shaped interpolSpline (interpol_spline.hxx:49-189), both
// resident on one GPU.
//
// A vls_spline2d holds nslices data slices [slice][dim1][dim0] (dim0
// fastest, as localSpline::assign reads them, localSpline.hxx:210-246) and
// their padded coefficient slices in the step's C layout
// [slice][dim1+3][pitch], coefficient (a, b) of slice s at row a, column b,
// i.e. the reference's data[b + a (dim0+2)].  build() runs the step's
// prefilter kernels (u-direction solves, then r-direction solves; the
// tensor operator of create_2D, localSpline.hxx:1238-1258).  The gathers run
// one point per thread from the coefficients in global memory; the
// decomposition of a position into (index, fraction) (pos2Coord,
// localSpline.hxx:352-358) runs on the host in FP64 with the host libm, so
// that the indices are the reference's bit for bit.
//
// Only the natural boundary condition is built (the one the step uses,
// vlasovSolver21_spline.hxx:296-374); the others are rejected with
// VLS_EINVAL.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vlasolve_b200.h"
#include "vls_internal.h"
#include "vls_setup.h"

using namespace vls;

struct vls_spline2d {
  vls_spline2d_desc d{};
  int dim[2] = {0, 0};      // values per direction (genScale sizes)
  double start[2], step_inv[2];  // localSpline::start / step_inv (rescaled)
  int64_t ns = 0;           // slices
  int pc = 0, gp = 0;       // row pitches of C and G
  size_t esize = 8;
  cudaStream_t st = nullptr;
  void *f = nullptr, *G = nullptr, *C = nullptr;
  double *rp[2] = {nullptr, nullptr}, *q[2] = {nullptr, nullptr};
  unsigned int *flag = nullptr;
  HostDirTables tab[2];
  int rc_cfg[2] = {-1, -1};  // register layouts of the u (dim1) and r (dim0) lines
  RcDir<double> rcd[2];
  bool assigned = false, built = false;
  // point buffers of the gathers (grown on demand)
  void *pts = nullptr;
  size_t pts_bytes = 0;
  std::vector<void *> allocs;
  std::string err;
};

namespace {

thread_local std::string g_spline_create_error;

int sfail(vls_spline2d *s, int code, const std::string &m) {
  if (s)
    s->err = m;
  else
    g_spline_create_error = m;
  return code;
}

#define SCK(s, call)                                                              \
  do {                                                                            \
    const cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                        \
      return sfail(s, VLS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename P>
int salloc(vls_spline2d *s, P **p, size_t bytes) {
  void *q = nullptr;
  const cudaError_t e = cudaMalloc(&q, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return sfail(s, VLS_ENOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
  }
  s->allocs.push_back(q);
  *p = reinterpret_cast<P *>(q);
  return VLS_OK;
}

void sfree(vls_spline2d *s) {
  if (s->st) cudaStreamSynchronize(s->st);
  for (void *p : s->allocs) cudaFree(p);
  s->allocs.clear();
  if (s->pts) cudaFree(s->pts);
  s->pts = nullptr;
  if (s->st) cudaStreamDestroy(s->st);
  s->st = nullptr;
}

Geometry spline_geometry(const vls_spline2d *s) {
  Geometry g{};
  g.nr = s->dim[0];
  g.nu = s->dim[1];
  g.nj = (int)s->ns;
  g.pc = s->pc;
  g.gp = s->gp;
  g.j0 = 0;
  g.nb = (int)s->ns;
  return g;
}

DirTables spline_dir(const vls_spline2d *s, int k) {
  const HostDirTables &t = s->tab[k];
  DirTables d{};
  d.rp = s->rp[k];
  d.q = s->q[k];
  d.a01 = t.a01;
  d.a02 = t.a02;
  d.hi2 = t.hi2;
  d.L1 = t.L1;
  d.L2 = t.L2;
  d.M = t.M;
  d.kc64 = t.kc64;
  d.kc32 = t.kc32;
  d.rp_inf = t.rp_inf;
  d.q_inf = t.q_inf;
  return d;
}

}  // namespace

extern "C" const char *vls_spline2d_last_error(const vls_spline2d *s) {
  return s ? s->err.c_str() : g_spline_create_error.c_str();
}

extern "C" int vls_spline2d_create(const vls_spline2d_desc *d, int64_t nslices,
                                   vls_spline2d **out) {
  if (!d || !out) return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: NULL argument");
  *out = nullptr;
  if (nslices < 1) return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: nslices < 1");
  if (d->precision != VLS_FP64 && d->precision != VLS_FP32_BULK)
    return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: precision FP64 or FP32_BULK");
  for (int k = 0; k < 2; ++k) {
    if (d->bCond[k][0] != VLS_BC_NATURAL || d->bCond[k][1] != VLS_BC_NATURAL)
      return sfail(nullptr, VLS_EINVAL,
                   "vls_spline2d_create: only the natural boundary condition is built");
    if (d->scaleType[k] < VLS_SCALE_LINEAR || d->scaleType[k] > VLS_SCALE_QUADRATIC)
      return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: unknown scale type");
  }
  {
    const int s = vls_device_ok(d->device);
    if (s != VLS_OK) return sfail(nullptr, s, vls_last_error(nullptr));
  }
  std::unique_ptr<vls_spline2d> s(new vls_spline2d());
  s->d = *d;
  s->ns = nslices;
  s->esize = d->precision == VLS_FP64 ? 8 : 4;
  // localSpline::init (localSpline.hxx:60-93)
  for (int k = 0; k < 2; ++k) {
    const std::vector<double> scl =
        gen_scale(d->start[k], d->stop[k], d->N[k], d->scaleType[k], d->vlType[k] != 0);
    s->dim[k] = (int)scl.size();
    if (s->dim[k] < 2 || s->dim[k] > 2048)
      return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: 2 to 2048 values per direction");
    double a = scl.front(), b = scl.back();
    a = rescale(a, d->scaleType[k]);
    b = rescale(b, d->scaleType[k]);
    const double step = (b - a) / (s->dim[k] - 1);
    s->start[k] = a;
    s->step_inv[k] = 1. / step;
    s->tab[k] = thomas_tables(s->dim[k], s->step_inv[k]);
  }
  if ((double)s->dim[0] * s->dim[1] * (double)nslices > 4.0e9)
    return sfail(nullptr, VLS_EINVAL, "vls_spline2d_create: more than 4e9 values");
  s->pc = ((s->dim[0] + 3) + 3) / 4 * 4;
  {
    const int per16 = (int)(16 / s->esize);
    s->gp = (s->dim[0] + per16 - 1) / per16 * per16;
  }
  for (int k = 0; k < 2; ++k) {
    // k = 0: r lines (dim0, the prer kernel), k = 1: u lines (dim1, ucol)
    s->rc_cfg[k] = rc_config<double>(s->tab[k], k == 1);
    s->rcd[k] = rc_dir<double>(s->tab[k], s->rc_cfg[k]);
  }
  if (cudaSetDevice(d->device) != cudaSuccess)
    return sfail(nullptr, VLS_ECUDA, "cudaSetDevice failed");
  vls_spline2d *sp = s.get();
  int rc = VLS_OK;
  auto A = [&](int r) {
    if (rc == VLS_OK) rc = r;
  };
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess)
    return sfail(nullptr, VLS_ECUDA, "cudaStreamCreate failed");
  const size_t n = (size_t)s->dim[0] * s->dim[1] * nslices;
  A(salloc(sp, &s->f, s->esize * n));
  A(salloc(sp, &s->G, s->esize * (size_t)nslices * (s->dim[1] + 2) * s->gp));
  A(salloc(sp, &s->C, s->esize * (size_t)nslices * (s->dim[1] + 3) * s->pc));
  for (int k = 0; k < 2; ++k) {
    A(salloc(sp, &s->rp[k], sizeof(double) * s->tab[k].M));
    A(salloc(sp, &s->q[k], sizeof(double) * s->tab[k].M));
  }
  A(salloc(sp, &s->flag, sizeof(unsigned int) * 4));
  if (rc != VLS_OK) {
    g_spline_create_error = sp->err;
    sfree(sp);
    return rc;
  }
  bool ok = true;
  for (int k = 0; k < 2; ++k) {
    ok = ok && cudaMemcpy(s->rp[k], s->tab[k].rp.data(), sizeof(double) * s->tab[k].M,
                          cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(s->q[k], s->tab[k].q.data(), sizeof(double) * s->tab[k].M,
                          cudaMemcpyHostToDevice) == cudaSuccess;
  }
  // rows and columns past the coefficients stay zero (the gathers of points
  // on the last node read them with weight 0)
  ok = ok && cudaMemset(s->C, 0, s->esize * (size_t)nslices * (s->dim[1] + 3) * s->pc) ==
                 cudaSuccess;
  ok = ok && cudaMemset(s->flag, 0, sizeof(unsigned int) * 4) == cudaSuccess;
  if (!ok) {
    sfree(sp);
    return sfail(nullptr, VLS_ECUDA, "vls_spline2d_create: table upload failed");
  }
  *out = s.release();
  return VLS_OK;
}

extern "C" int vls_spline2d_destroy(vls_spline2d *s) {
  if (!s) return VLS_OK;
  cudaSetDevice(s->d.device);
  sfree(s);
  delete s;
  return VLS_OK;
}

extern "C" int vls_spline2d_dims(const vls_spline2d *s, int32_t *dim0, int32_t *dim1,
                                 int64_t *nslices) {
  if (!s) return VLS_EINVAL;
  if (dim0) *dim0 = s->dim[0];
  if (dim1) *dim1 = s->dim[1];
  if (nslices) *nslices = s->ns;
  return VLS_OK;
}

extern "C" int vls_spline2d_scale(const vls_spline2d *s, double *start, double *step_inv) {
  if (!s) return VLS_EINVAL;
  for (int k = 0; k < 2; ++k) {
    if (start) start[k] = s->start[k];
    if (step_inv) step_inv[k] = s->step_inv[k];
  }
  return VLS_OK;
}

// localSpline::assign (localSpline.hxx:210-246): the values of nslices
// slices [slice][dim1][dim0] (host, FP64; rounded once to FP32 for
// VLS_FP32_BULK objects)
extern "C" int vls_spline2d_assign(vls_spline2d *s, const double *data, int64_t nslices) {
  if (!s || !data) return sfail(s, VLS_EINVAL, "vls_spline2d_assign: NULL argument");
  if (nslices != s->ns) return sfail(s, VLS_EINVAL, "vls_spline2d_assign: slice count mismatch");
  SCK(s, cudaSetDevice(s->d.device));
  const size_t n = (size_t)s->dim[0] * s->dim[1] * s->ns;
  if (s->esize == 8) {
    SCK(s, cudaMemcpyAsync(s->f, data, sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
    SCK(s, cudaStreamSynchronize(s->st));
  } else {
    std::vector<float> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = (float)data[i];
    SCK(s, cudaMemcpyAsync(s->f, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s->st));
    SCK(s, cudaStreamSynchronize(s->st));
  }
  s->assigned = true;
  s->built = false;
  return VLS_OK;
}

namespace {
template <typename T>
cudaError_t spline_build(vls_spline2d *s) {
  const Geometry g = spline_geometry(s);
  const T *f = (const T *)s->f;
  T *G = (T *)s->G, *C = (T *)s->C;
  cudaError_t e;
  // solves along dim1 (the step's u lines), then along dim0 (r lines)
  if (s->rc_cfg[1] >= 0)
    e = launch_ucol_rc<T, double>(s->rc_cfg[1], false, f, G, nullptr, g, s->rcd[1], s->st);
  else
    e = launch_ucol<T, double>(false, f, G, nullptr, g, spline_dir(s, 1), s->st);
  if (e != cudaSuccess) return e;
  if (s->rc_cfg[0] >= 0)
    return launch_prer_rc<T, double>(s->rc_cfg[0], G, C, g, s->rcd[0], s->flag + 1, s->st);
  return launch_prer<T, double>(G, C, g, spline_dir(s, 0), s->st);
}
}  // namespace

// localSpline::build / create_2D (localSpline.hxx:248-260, :1238-1258): the
// coefficients of every slice
extern "C" int vls_spline2d_build(vls_spline2d *s) {
  if (!s) return VLS_EINVAL;
  if (!s->assigned) return sfail(s, VLS_ESTATE, "vls_spline2d_build before assign");
  SCK(s, cudaSetDevice(s->d.device));
  SCK(s, s->esize == 8 ? spline_build<double>(s) : spline_build<float>(s));
  unsigned int fl[4];
  SCK(s, cudaMemcpyAsync(fl, s->flag, sizeof(fl), cudaMemcpyDeviceToHost, s->st));
  SCK(s, cudaStreamSynchronize(s->st));
  if (fl[1]) {
    SCK(s, cudaMemset(s->flag, 0, sizeof(fl)));
    return sfail(s, VLS_ECUDA, "a bounded device wait timed out in the r-solve kernel");
  }
  s->built = true;
  return VLS_OK;
}

// the padded coefficients of one slice as the reference's spline buffer
// holds them (localSpline.hxx:222): (dim0+2) x (dim1+2) FP64, dim0 fastest
extern "C" int vls_spline2d_coefficients(vls_spline2d *s, int64_t slice, double *coef) {
  if (!s || !coef) return sfail(s, VLS_EINVAL, "vls_spline2d_coefficients: NULL argument");
  if (!s->built) return sfail(s, VLS_ESTATE, "vls_spline2d_coefficients before build");
  if (slice < 0 || slice >= s->ns)
    return sfail(s, VLS_EINVAL, "vls_spline2d_coefficients: slice out of range");
  SCK(s, cudaSetDevice(s->d.device));
  const int w = s->dim[0] + 2, hgt = s->dim[1] + 2;
  const char *src = (const char *)s->C + s->esize * (size_t)slice * (s->dim[1] + 3) * s->pc;
  if (s->esize == 8) {
    SCK(s, cudaMemcpy2DAsync(coef, sizeof(double) * w, src, sizeof(double) * s->pc,
                             sizeof(double) * w, hgt, cudaMemcpyDeviceToHost, s->st));
    SCK(s, cudaStreamSynchronize(s->st));
  } else {
    std::vector<float> h((size_t)w * hgt);
    SCK(s, cudaMemcpy2DAsync(h.data(), sizeof(float) * w, src, sizeof(float) * s->pc,
                             sizeof(float) * w, hgt, cudaMemcpyDeviceToHost, s->st));
    SCK(s, cudaStreamSynchronize(s->st));
    for (size_t i = 0; i < h.size(); ++i) coef[i] = h[i];
  }
  return VLS_OK;
}

// localSpline::pos2Coord (localSpline.hxx:352-358) of n positions along
// direction dir, on the host (FP64, host libm: the reference's indices)
extern "C" int vls_spline2d_pos2coord(const vls_spline2d *sc, int32_t dir, int64_t n,
                                      const double *p, int32_t *I, double *F) {
  vls_spline2d *s = const_cast<vls_spline2d *>(sc);
  if (!s || (n > 0 && (!p || !I || !F)))
    return sfail(s, VLS_EINVAL, "vls_spline2d_pos2coord: NULL argument");
  if (dir != 0 && dir != 1) return sfail(s, VLS_EINVAL, "vls_spline2d_pos2coord: dir 0 or 1");
  for (int64_t i = 0; i < n; ++i) {
    double ip;
    const double x = std::modf((rescale(p[i], s->d.scaleType[dir]) - s->start[dir]) *
                                   s->step_inv[dir],
                               &ip);
    I[i] = (ip > -2.0e9 && ip < 2.0e9) ? (int32_t)ip : INT32_MIN;
    F[i] = x;
  }
  return VLS_OK;
}

// ------------------------------------------------------------ gathers
namespace {

enum { EV_VALUE = 0, EV_GRAD = 1, EV_HESS = 2, EV_NXPY = 3 };

// cubic B-spline weights (x6) of the four taps at fraction t, and their
// first and second derivatives with respect to t:
//   w0 = (1-t)^3, w1 = 1 + 3s + 3s^2 - 3s^3 (s = 1-t), w2 = the same in t,
//   w3 = t^3 (localSpline.hxx BV1 / BV2 at 1-t, 1-t, t, t)
__device__ __forceinline__ void bweights(double t, double (&w)[4], double (&d)[4],
                                         double (&dd)[4]) {
  const double s = 1.0 - t;
  w[0] = s * s * s;
  w[1] = 1.0 + 3.0 * s + 3.0 * s * s - 3.0 * s * s * s;
  w[2] = 1.0 + 3.0 * t + 3.0 * t * t - 3.0 * t * t * t;
  w[3] = t * t * t;
  d[0] = -3.0 * s * s;
  d[1] = -(3.0 + 6.0 * s - 9.0 * s * s);
  d[2] = 3.0 + 6.0 * t - 9.0 * t * t;
  d[3] = 3.0 * t * t;
  dd[0] = 6.0 * s;
  dd[1] = 6.0 - 18.0 * s;
  dd[2] = 6.0 - 18.0 * t;
  dd[3] = 6.0 * t;
}

// One point per thread: taps at padded columns Nx..Nx+3 (Nx..Nx+2 with the
// node weights 1, 4, 1 for EV_NXPY) and rows Ny..Ny+3 of the point's slice,
// all inside the coefficient array for 0 <= Nx < dim0, 0 <= Ny < dim1 (the
// host checks those before the launch).  v = sum wy wx C / 36; g =
// (dv/dy, dv/dx) and h = (yy, yx, xy, xx) in rescaled coordinates (hx, hy:
// 1 / node spacing), in that order as einspline returns them for its
// (y, x) call (interpol_spline.hxx:133-160).
template <typename T, int MODE>
__global__ void spline_points_kernel(const T *__restrict__ C, int pc, int rows, int64_t n,
                                     const int64_t *__restrict__ slice,
                                     const int32_t *__restrict__ NX,
                                     const double *__restrict__ X,
                                     const int32_t *__restrict__ NY,
                                     const double *__restrict__ Y, double hx, double hy,
                                     double *__restrict__ v, double *__restrict__ g,
                                     double *__restrict__ h) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t j = slice ? slice[i] : 0;
  const T *p = C + ((size_t)j * rows + NY[i]) * (size_t)pc + NX[i];
  double wx[4], dx[4], ddx[4], wy[4], dy[4], ddy[4];
  if (MODE == EV_NXPY) {
    wx[0] = 1.0;
    wx[1] = 4.0;
    wx[2] = 1.0;
    wx[3] = 0.0;
  } else {
    bweights(X[i], wx, dx, ddx);
  }
  bweights(Y[i], wy, dy, ddy);
  double s[4], sx[4], sxx[4];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const T *row = p + (size_t)a * pc;
    s[a] = 0.0;
    sx[a] = 0.0;
    sxx[a] = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (MODE == EV_NXPY && b == 3) break;
      const double c = (double)row[b];
      s[a] += wx[b] * c;
      if (MODE == EV_GRAD || MODE == EV_HESS) sx[a] += dx[b] * c;
      if (MODE == EV_HESS) sxx[a] += ddx[b] * c;
    }
  }
  const double k = 1.0 / 36.0;
  double val = 0.0;
#pragma unroll
  for (int a = 0; a < 4; ++a) val += wy[a] * s[a];
  v[i] = k * val;
  if (MODE == EV_GRAD || MODE == EV_HESS) {
    double vx = 0.0, vy = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      vx += wy[a] * sx[a];
      vy += dy[a] * s[a];
    }
    g[2 * i] = k * hy * vy;
    g[2 * i + 1] = k * hx * vx;
    if (MODE == EV_HESS) {
      double vxx = 0.0, vyy = 0.0, vxy = 0.0;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        vxx += wy[a] * sxx[a];
        vyy += ddy[a] * s[a];
        vxy += dy[a] * sx[a];
      }
      h[4 * i] = k * hy * hy * vyy;
      h[4 * i + 1] = k * hx * hy * vxy;
      h[4 * i + 2] = k * hx * hy * vxy;
      h[4 * i + 3] = k * hx * hx * vxx;
    }
  }
}

template <typename T>
cudaError_t launch_points(const vls_spline2d *s, int mode, int64_t n, const int64_t *slice,
                          const int32_t *NX, const double *X, const int32_t *NY,
                          const double *Y, double *v, double *g, double *h) {
  const unsigned blocks = (unsigned)((n + 255) / 256);
  const T *C = (const T *)s->C;
  const int rows = s->dim[1] + 3;
  const double hx = s->step_inv[0], hy = s->step_inv[1];
  switch (mode) {
    case EV_VALUE:
      spline_points_kernel<T, EV_VALUE><<<blocks, 256, 0, s->st>>>(C, s->pc, rows, n, slice, NX,
                                                                  X, NY, Y, hx, hy, v, g, h);
      break;
    case EV_GRAD:
      spline_points_kernel<T, EV_GRAD><<<blocks, 256, 0, s->st>>>(C, s->pc, rows, n, slice, NX,
                                                                 X, NY, Y, hx, hy, v, g, h);
      break;
    case EV_HESS:
      spline_points_kernel<T, EV_HESS><<<blocks, 256, 0, s->st>>>(C, s->pc, rows, n, slice, NX,
                                                                 X, NY, Y, hx, hy, v, g, h);
      break;
    default:
      spline_points_kernel<T, EV_NXPY><<<blocks, 256, 0, s->st>>>(C, s->pc, rows, n, slice, NX,
                                                                 X, NY, Y, hx, hy, v, g, h);
  }
  return cudaGetLastError();
}

// n points, host arrays in and out: checks the indices, uploads, gathers,
// downloads.  slice may be NULL (every point on slice 0); g (2n) and h (4n)
// are written for EV_GRAD / EV_HESS.
int run_points(vls_spline2d *s, int mode, int64_t n, const int64_t *slice, const int32_t *NX,
               const double *X, const int32_t *NY, const double *Y, double *v, double *g,
               double *h) {
  if (!s->built) return sfail(s, VLS_ESTATE, "spline evaluated before build");
  if (n < 0) return sfail(s, VLS_EINVAL, "negative point count");
  if (n == 0) return VLS_OK;
  for (int64_t i = 0; i < n; ++i) {
    if (NX[i] < 0 || NX[i] >= s->dim[0] || NY[i] < 0 || NY[i] >= s->dim[1])
      return sfail(s, VLS_EINVAL,
                   "point " + std::to_string(i) + " lies outside the spline's nodes");
    if (slice && (slice[i] < 0 || slice[i] >= s->ns))
      return sfail(s, VLS_EINVAL, "point " + std::to_string(i) + ": slice out of range");
  }
  SCK(s, cudaSetDevice(s->d.device));
  const size_t nn = (size_t)n;
  const int nout = mode == EV_HESS ? 7 : mode == EV_GRAD ? 3 : 1;
  const size_t bytes = nn * (8 * 3 + 4 * 2 + 8 * (size_t)nout) + 64;
  if (bytes > s->pts_bytes) {
    if (s->pts) cudaFree(s->pts);
    s->pts = nullptr;
    s->pts_bytes = 0;
    if (cudaMalloc(&s->pts, bytes) != cudaSuccess) {
      cudaGetLastError();
      return sfail(s, VLS_ENOMEM, "cudaMalloc of the point buffers failed");
    }
    s->pts_bytes = bytes;
  }
  char *b = (char *)s->pts;
  int64_t *d_sl = slice ? (int64_t *)b : nullptr;
  double *d_x = (double *)(b + 8 * nn), *d_y = (double *)(b + 16 * nn);
  double *d_v = (double *)(b + 24 * nn);
  double *d_g = d_v + nn, *d_h = d_v + 3 * nn;
  int32_t *d_nx = (int32_t *)(b + 24 * nn + 8 * nn * (size_t)nout);
  int32_t *d_ny = d_nx + nn;
  if (slice) SCK(s, cudaMemcpyAsync(d_sl, slice, 8 * nn, cudaMemcpyHostToDevice, s->st));
  if (mode != EV_NXPY) SCK(s, cudaMemcpyAsync(d_x, X, 8 * nn, cudaMemcpyHostToDevice, s->st));
  SCK(s, cudaMemcpyAsync(d_y, Y, 8 * nn, cudaMemcpyHostToDevice, s->st));
  SCK(s, cudaMemcpyAsync(d_nx, NX, 4 * nn, cudaMemcpyHostToDevice, s->st));
  SCK(s, cudaMemcpyAsync(d_ny, NY, 4 * nn, cudaMemcpyHostToDevice, s->st));
  SCK(s, s->esize == 8 ? launch_points<double>(s, mode, n, d_sl, d_nx, d_x, d_ny, d_y, d_v, d_g,
                                               d_h)
                       : launch_points<float>(s, mode, n, d_sl, d_nx, d_x, d_ny, d_y, d_v, d_g,
                                              d_h));
  SCK(s, cudaMemcpyAsync(v, d_v, 8 * nn, cudaMemcpyDeviceToHost, s->st));
  if (mode == EV_GRAD || mode == EV_HESS)
    SCK(s, cudaMemcpyAsync(g, d_g, 16 * nn, cudaMemcpyDeviceToHost, s->st));
  if (mode == EV_HESS) SCK(s, cudaMemcpyAsync(h, d_h, 32 * nn, cudaMemcpyDeviceToHost, s->st));
  SCK(s, cudaStreamSynchronize(s->st));
  return VLS_OK;
}

}  // namespace

// localSpline::evaluateC(int, double, int, double) (localSpline.hxx:381-398)
// at n points of the given slices
extern "C" int vls_spline2d_evaluate_c(vls_spline2d *s, int64_t n, const int64_t *slice,
                                       const int32_t *Nx, const double *x, const int32_t *Ny,
                                       const double *y, double *v) {
  if (!s || (n > 0 && (!Nx || !x || !Ny || !y || !v)))
    return sfail(s, VLS_EINVAL, "vls_spline2d_evaluate_c: NULL argument");
  return run_points(s, EV_VALUE, n, slice, Nx, x, Ny, y, v, nullptr, nullptr);
}

// localSpline::evaluateNxPy (localSpline.hxx:423-441): at node Nx along dim0
// and position yy along dim1 (decomposed on the host as the reference does)
extern "C" int vls_spline2d_evaluate_nxpy(vls_spline2d *s, int64_t n, const int64_t *slice,
                                          const int32_t *Nx, const double *yy, double *v) {
  if (!s || (n > 0 && (!Nx || !yy || !v)))
    return sfail(s, VLS_EINVAL, "vls_spline2d_evaluate_nxpy: NULL argument");
  std::vector<int32_t> NY((size_t)std::max<int64_t>(n, 0));
  std::vector<double> Y(NY.size());
  const int rc = vls_spline2d_pos2coord(s, 1, n, yy, NY.data(), Y.data());
  if (rc != VLS_OK) return rc;
  return run_points(s, EV_NXPY, n, slice, Nx, nullptr, NY.data(), Y.data(), v, nullptr,
                    nullptr);
}

// localSpline::evaluate(double, double) (localSpline.hxx:477-488): pos2Coord
// of both coordinates on the host, then the gather
extern "C" int vls_spline2d_evaluate(vls_spline2d *s, int64_t n, const int64_t *slice,
                                     const double *xx, const double *yy, double *v) {
  if (!s || (n > 0 && (!xx || !yy || !v)))
    return sfail(s, VLS_EINVAL, "vls_spline2d_evaluate: NULL argument");
  const size_t nn = (size_t)std::max<int64_t>(n, 0);
  std::vector<int32_t> NX(nn), NY(nn);
  std::vector<double> X(nn), Y(nn);
  int rc = vls_spline2d_pos2coord(s, 0, n, xx, NX.data(), X.data());
  if (rc == VLS_OK) rc = vls_spline2d_pos2coord(s, 1, n, yy, NY.data(), Y.data());
  if (rc != VLS_OK) return rc;
  return run_points(s, EV_VALUE, n, slice, NX.data(), X.data(), NY.data(), Y.data(), v,
                    nullptr, nullptr);
}

// ---------------------------------------------------------- interpolSpline
// interpolSpline (interpol_spline.hxx:49-189) over einspline, a third-party
// library the reference does not vendor (and compiles out): a uniform cubic
// B-spline in rescaled coordinates whose last node sits 1e-10 of a cell past
// the data's last node.  With natural ends (NATURAL, or DERIV2 with value
// 0: the same boundary row) its coefficients are those of the natural-BC
// solve above, so the object is a one-slice vls_spline2d on that grid.
struct vls_interp {
  vls_interp_init ini{};
  vls_spline2d *sp = nullptr;
  std::string err;
};

namespace {
thread_local std::string g_interp_error;
int ifail(vls_interp *s, int code, const std::string &m) {
  if (s)
    s->err = m;
  else
    g_interp_error = m;
  return code;
}
bool natural_end(int32_t code, double val) {
  return code == VLS_EBC_NATURAL || (code == VLS_EBC_DERIV2 && val == 0.0);
}
}  // namespace

extern "C" const char *vls_interp_last_error(const vls_interp *s) {
  return s ? s->err.c_str() : g_interp_error.c_str();
}

// interpolSpline::createInit (interpol_spline.hxx:49-91), on the host
extern "C" int vls_interp_create_init(double xstart, double xstop, int32_t Nx, double ystart,
                                      double ystop, int32_t Ny, int32_t xbctL, int32_t xbctR,
                                      int32_t ybctL, int32_t ybctR, int32_t xscaleType,
                                      int32_t yscaleType, int32_t vltype, int32_t useLog,
                                      double xbcvL, double xbcvR, double ybcvL, double ybcvR,
                                      vls_interp_init *g) {
  if (!g) return ifail(nullptr, VLS_EINVAL, "vls_interp_create_init: NULL argument");
  if (xscaleType < VLS_SCALE_LINEAR || xscaleType > VLS_SCALE_QUADRATIC ||
      yscaleType < VLS_SCALE_LINEAR || yscaleType > VLS_SCALE_QUADRATIC)
    return ifail(nullptr, VLS_EINVAL, "vls_interp_create_init: unknown scale type");
  std::memset(g, 0, sizeof(*g));
  const double se[2] = {xstart, ystart}, so[2] = {xstop, ystop};
  const int32_t N[2] = {Nx, Ny}, sct[2] = {xscaleType, yscaleType};
  double *gs[2] = {&g->xstart, &g->ystart}, *ge[2] = {&g->xend, &g->yend};
  int32_t *num[2] = {&g->nx, &g->ny};
  g->rescaleNeeded = 0;
  for (int k = 0; k < 2; ++k) {
    std::vector<double> t = gen_scale(se[k], so[k], N[k], sct[k], vltype != 0);
    if (t.size() < 2) return ifail(nullptr, VLS_EINVAL, "vls_interp_create_init: grid too small");
    t.back() += (t[t.size() - 1] - t[t.size() - 2]) * 1.E-10;
    *gs[k] = rescale(t.front(), sct[k]);
    *ge[k] = rescale(t.back(), sct[k]);
    *num[k] = (int32_t)t.size();
    if (sct[k] != VLS_SCALE_LINEAR) g->rescaleNeeded = 1;
  }
  g->xbc[0] = xbctL;
  g->xbc[1] = xbctR;
  g->ybc[0] = ybctL;
  g->ybc[1] = ybctR;
  g->xbcv[0] = xbcvL;
  g->xbcv[1] = xbcvR;
  g->ybcv[0] = ybcvL;
  g->ybcv[1] = ybcvR;
  g->xscaleType = xscaleType;
  g->yscaleType = yscaleType;
  g->useLog = useLog ? 1 : 0;
  return VLS_OK;
}

// interpolSpline::create (interpol_spline.hxx:93-110): data [y][x], x
// fastest (ny x nx values; their logarithm is interpolated with useLog)
extern "C" int vls_interp_create(const vls_interp_init *ini, const double *data, int32_t device,
                                 vls_interp **out) {
  if (!ini || !data || !out) return ifail(nullptr, VLS_EINVAL, "vls_interp_create: NULL argument");
  *out = nullptr;
  if (!natural_end(ini->xbc[0], ini->xbcv[0]) || !natural_end(ini->xbc[1], ini->xbcv[1]) ||
      !natural_end(ini->ybc[0], ini->ybcv[0]) || !natural_end(ini->ybc[1], ini->ybcv[1]))
    return ifail(nullptr, VLS_EINVAL,
                 "vls_interp_create: only natural ends (NATURAL, or DERIV2 with value 0) are built");
  if (ini->nx < 2 || ini->ny < 2 || ini->nx > 2048 || ini->ny > 2048)
    return ifail(nullptr, VLS_EINVAL, "vls_interp_create: 2 to 2048 nodes per direction");
  std::unique_ptr<vls_interp> s(new vls_interp());
  s->ini = *ini;
  vls_spline2d_desc d{};
  // a linear grid of nx (ny) vertices from start to end, in the rescaled
  // coordinates the evaluation maps points into
  d.start[0] = ini->xstart;
  d.stop[0] = ini->xend;
  d.N[0] = ini->nx - 1;
  d.start[1] = ini->ystart;
  d.stop[1] = ini->yend;
  d.N[1] = ini->ny - 1;
  for (int k = 0; k < 2; ++k) {
    d.scaleType[k] = VLS_SCALE_LINEAR;
    d.vlType[k] = 1;
    d.bCond[k][0] = d.bCond[k][1] = VLS_BC_NATURAL;
  }
  d.precision = VLS_FP64;
  d.device = device;
  int rc = vls_spline2d_create(&d, 1, &s->sp);
  if (rc != VLS_OK) return ifail(nullptr, rc, vls_spline2d_last_error(nullptr));
  const size_t n = (size_t)ini->nx * ini->ny;
  std::vector<double> tmp;
  const double *src = data;
  if (ini->useLog) {
    tmp.assign(data, data + n);
    for (double &x : tmp) x = std::log(x);
    src = tmp.data();
  }
  rc = vls_spline2d_assign(s->sp, src, 1);
  if (rc == VLS_OK) rc = vls_spline2d_build(s->sp);
  if (rc != VLS_OK) {
    const std::string m = vls_spline2d_last_error(s->sp);
    vls_spline2d_destroy(s->sp);
    return ifail(nullptr, rc, m);
  }
  *out = s.release();
  return VLS_OK;
}

// interpolSpline::evaluate (interpol_spline.hxx:112-183) at n points: v, and
// with g (2 per point: dv/dy, dv/dx) the gradient, with h (4 per point: yy,
// yx, xy, xx) the Hessian, in rescaled coordinates as einspline returns them.
// Points are rescaled (scale types) and clamped to the grid as the reference
// does when a scale is not linear; on linear grids the reference leaves them
// as they are and einspline reads outside its coefficients for points
// outside the grid, here they are clamped in every case.  useLog: v =
// exp(max(v, -700)) and g = -g v (the reference's formula); a Hessian of a
// useLog spline is an error (the reference exits there).
extern "C" int vls_interp_evaluate(vls_interp *s, int64_t n, const double *x, const double *y,
                                   double *v, double *g, double *h) {
  if (!s || (n > 0 && (!x || !y || !v)))
    return ifail(s, VLS_EINVAL, "vls_interp_evaluate: NULL argument");
  if (h && !g) return ifail(s, VLS_EINVAL, "vls_interp_evaluate: a Hessian needs g too");
  if (h && s->ini.useLog)
    return ifail(s, VLS_EINVAL,
                 "second derivative evaluation for spline with log valued function not "
                 "implemented (interpol_spline.hxx:172-176)");
  if (n <= 0) return n < 0 ? ifail(s, VLS_EINVAL, "negative point count") : VLS_OK;
  const vls_interp_init &I = s->ini;
  const size_t nn = (size_t)n;
  std::vector<int32_t> NX(nn), NY(nn);
  std::vector<double> X(nn), Y(nn);
  double st[2], hi[2];
  vls_spline2d_scale(s->sp, st, hi);
  for (size_t i = 0; i < nn; ++i) {
    double px = x[i], py = y[i];
    if (I.rescaleNeeded) {
      px = rescale(px, I.xscaleType);
      py = rescale(py, I.yscaleType);
    }
    px = std::min(std::max(px, I.xstart), I.xend);
    py = std::min(std::max(py, I.ystart), I.yend);
    double ip;
    X[i] = std::modf((px - st[0]) * hi[0], &ip);
    NX[i] = std::min((int32_t)ip, I.nx - 1);
    Y[i] = std::modf((py - st[1]) * hi[1], &ip);
    NY[i] = std::min((int32_t)ip, I.ny - 1);
  }
  const int mode = h ? EV_HESS : g ? EV_GRAD : EV_VALUE;
  const int rc = run_points(s->sp, mode, n, nullptr, NX.data(), X.data(), NY.data(), Y.data(),
                            v, g, h);
  if (rc != VLS_OK) return ifail(s, rc, vls_spline2d_last_error(s->sp));
  if (I.useLog)
    for (size_t i = 0; i < nn; ++i) {
      v[i] = std::exp(std::max(v[i], -700.0));
      if (g) {
        g[2 * i] = -g[2 * i] * v[i];
        g[2 * i + 1] = -g[2 * i + 1] * v[i];
      }
    }
  return VLS_OK;
}

// interpolSpline::destroy (interpol_spline.hxx:185-189)
extern "C" int vls_interp_destroy(vls_interp *s) {
  if (!s) return VLS_OK;
  vls_spline2d_destroy(s->sp);
  delete s;
  return VLS_OK;
}
