// vls_api.cpp -- the C-ABI of include/vlasolve_b200.h: handle life cycle,
// host set-up upload, step orchestration on the handle's CUDA stream,
// moments, statistics and NDfield I/O.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <omp.h>

#include <cstdlib>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vlasolve_b200.h"
#include "vls_internal.h"
#include "vls_setup.h"

using namespace vls;

struct vls_handle {
  vls_grid_desc grid{};
  vls_solver_desc solver{};
  Coords co;
  HostDirTables tr, tu;
  int prec = VLS_FP64;
  size_t esize = 8;
  size_t cells = 0;
  int pc = 0;
  int gp = 0;  // row pitch of G: N_r rounded up to 16 bytes
  cudaStream_t st = nullptr;
  // device buffers
  void *f = nullptr, *G = nullptr, *C = nullptr;
  float *bu32 = nullptr;         // the moment weights b_u in FP32
  int32_t *idx = nullptr;        // FP64 footpoints
  void *fx = nullptr, *fy = nullptr;
  uint2 *fp2 = nullptr;          // FP32 packed footpoints
  int64_t nch = 0, nel = 0;
  int64_t *ch_start = nullptr;
  int32_t *ch_len = nullptr;
  void *ch_val = nullptr;
  int32_t *t_idx = nullptr;  // [nch] codes then [nch] slice index
  double *t_x = nullptr, *t_y = nullptr;
  double *rp_r = nullptr, *q_r = nullptr, *rp_u = nullptr, *q_u = nullptr;
  double *dU_val = nullptr, *dR_val = nullptr, *dJ_val = nullptr;
  double *d_dR = nullptr, *d_dU = nullptr, *d_Ct1 = nullptr;
  double *bu = nullptr, *wj = nullptr, *dR4 = nullptr, *Rcoef = nullptr;
  double *partial = nullptr, *T2 = nullptr, *bins = nullptr, *Mr = nullptr,
         *shift = nullptr, *mtot = nullptr;
  unsigned int *count = nullptr, *flag = nullptr;
  double *stats_part = nullptr;
  size_t stats_nblk = 0;
  double *staging = nullptr;
  size_t staging_n = 0;
  // host copies of the chain layout
  std::vector<int64_t> ch_cell_h, ch_start_h;
  std::vector<int32_t> ch_len_h;
  std::vector<double> ch_R_h, ch_U_h;
  // state
  bool have_f = false;
  bool moments_valid = false;
  int64_t ndrift = 0;
  double time = 0;
  int64_t step = 0;
  int64_t launches = 0;
  // slice batches: batch b covers slices [b*B, b*B+B) and runs on batch
  // stream b mod NS with its own ring slot of G and C scratch
  int B = 1, nbatch = 1, NS = 1;
  cudaStream_t bst[8] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[8] = {};
  std::vector<int64_t> chain_lo;  // first chain of slice j (size nj + 1)
  // register-resident prefilter tables (per direction and recursion type)
  // and whether its kernels take this grid (-1: the shared-memory segment
  // kernels, for longer lines or the segment prefilter layout)
  RcDir<double> rcu_d{}, rcr_d{};
  RcDir<float> rcu_f{}, rcr_f{};
  int rcu_cfg = -1, rcr_cfg = -1;
  // TMA descriptors of each slot of C for the drift's staged windows (tmC)
  // and strips (tmS, when drift_kind is a strip kind)
  CUtensorMap tmC[8];
  CUtensorMap tmS[8];
  int drift_kind = DRIFT_WINDOW;
  uint32_t drift_spins = MBAR_SPIN_LIMIT;  // polls of each bounded wait of the drift
  vls_layout_desc layout{};                // what vls_get_layout reports
  // opt-in per-kernel event timing
  bool profiling = false;
  struct ProfRec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> prof;
  std::vector<cudaEvent_t> evpool;
  std::string err;
  std::vector<void *> allocs;
  // adjoint: checkpoints of the forward run (state before steps 0, K, 2K, ...),
  // the final state, and the FP64 adjoint arrays; freed by the next forward
  // run or by vls_destroy
  struct Ckpt {
    void *f = nullptr, *ch = nullptr;
    int64_t ndrift = 0, step = 0;
    double time = 0;
  };
  std::vector<Ckpt> adj_ck;  // the first adj_ncp are this run's
  Ckpt adj_final;
  int64_t adj_n = 0;
  int adj_K = 0, adj_ncp = 0;
  // second level: checkpoints every adj_inner steps inside a segment (0:
  // chosen from free device memory at the backward pass), kept between calls
  int adj_inner = 0, adj_last_inner = 0;
  // device bytes this handle holds (its allocations are freed by vls_destroy only)
  size_t dev_bytes = 0;
  std::vector<Ckpt> adj_sub;
  // backward-pass arrays (FP64) and the segment stash, kept between calls
  double *ab_lam = nullptr, *ab_Cb = nullptr, *ab_Gb = nullptr, *ab_A = nullptr,
         *ab_B = nullptr, *ab_ringb = nullptr, *ab_sbar = nullptr, *ab_beta = nullptr;
  bool ab_rc = false;
  std::vector<void *> ab_stash;
  double *ab_shifts = nullptr;  // shift of each stashed state (ab_nshift x N_r)
  int ab_nshift = 0;
  // inverse footpoint map of the drift's transpose (built for footpoint set
  // fp_gen; see launch_inv_fill), the chain cells and tail adjoints
  uint64_t fp_gen = 0, inv_gen = ~(uint64_t)0;
  uint32_t *inv_ends = nullptr, *inv_ent = nullptr, *inv_tot = nullptr;
  int64_t *inv_ebase = nullptr, *inv_chc = nullptr;
  double *inv_tv = nullptr;
  // FP32 handles: the entries' packed words and each step's values in entry
  // order
  uint2 *inv_geo = nullptr;
  double *inv_vperm = nullptr;
  bool adj_ready = false;
  // the last backward pass's dL/d(initial chain values), logical order, and
  // whether ab_lam still holds its dL/df0 (vls_adjoint_init_dot)
  std::vector<double> adj_dch0;
  bool adj_grad = false;
  // coordinates R, U, J, JV, the quadrature's row sums and the dot's block
  // sums for vls_adjoint_init_dot
  double *ip_xyz = nullptr, *ip_rows = nullptr, *ip_part = nullptr;
  std::vector<void *> adj_allocs;
};

static std::string g_create_error;

static int fail(vls_handle *h, int code, const std::string &msg) {
  if (h)
    h->err = msg;
  else
    g_create_error = msg;
  return code;
}

#define CK(h, call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess)                                                \
      return fail((h), VLS_ECUDA,                                         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

template <typename P>
static int dalloc(vls_handle *h, P **p, size_t bytes) {
  void *q = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, VLS_ENOMEM,
                "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                    cudaGetErrorString(e));
  }
  h->allocs.push_back(q);
  h->dev_bytes += bytes;
  *p = reinterpret_cast<P *>(q);
  return VLS_OK;
}

static int upload(vls_handle *h, void *dst, const void *src, size_t bytes) {
  CK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  return VLS_OK;
}

#define TRY(x)                 \
  do {                         \
    int s_ = (x);              \
    if (s_ != VLS_OK) return s_; \
  } while (0)

static Geometry geometry(const vls_handle *h) {
  Geometry g{};
  g.nr = h->co.nr;
  g.nu = h->co.nu;
  g.nj = h->co.nj;
  g.pc = h->pc;
  g.gp = h->gp;
  g.j0 = 0;
  g.nb = h->co.nj;
  g.U = h->dU_val;
  g.u0 = h->co.U.front();
  g.umax = h->co.U.back();
  g.su = h->co.sstart[1];
  g.hu = h->co.sstep_inv[1];
  return g;
}

static DirTables dir_tables(const HostDirTables &t, const double *rp,
                            const double *q) {
  DirTables d{};
  d.rp = rp;
  d.q = q;
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

static MomentTables moment_tables(const vls_handle *h) {
  MomentTables m{};
  m.bu = h->bu;
  m.bu32 = h->bu32;
  m.wj = h->wj;
  m.dR4 = h->dR4;
  m.Rcoef = h->Rcoef;
  return m;
}

static cudaEvent_t take_event(vls_handle *h) {
  if (!h->evpool.empty()) {
    cudaEvent_t e = h->evpool.back();
    h->evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Runs one launch; counts it and, with profiling on, brackets it with events.
template <typename F>
static cudaError_t timed(vls_handle *h, int kind, F &&launch, cudaStream_t st = nullptr) {
  if (!st) st = h->st;
  cudaEvent_t a = nullptr, b = nullptr;
  if (h->profiling) {
    a = take_event(h);
    b = take_event(h);
    cudaEventRecord(a, st);
  }
  const cudaError_t e = launch();
  h->launches++;
  if (h->profiling) {
    cudaEventRecord(b, st);
    h->prof.push_back({kind, a, b});
  }
  return e;
}

// ------------------------------------------------------------- footpoints
// FP32 packed word of one direction: index << 21 | fraction rounded to 21
// bits; a fraction that rounds up to 1 moves to the next node (same spline
// value, the B-spline is continuous there).
static uint32_t pack_coord(int32_t I, double F, int32_t maxI) {
  const double q = std::nearbyint(F * 2097152.0);
  int64_t qi = (int64_t)q;
  if (qi >= (int64_t)1 << 21) {
    if (I < maxI) {
      I += 1;
      qi = 0;
    } else {
      qi = ((int64_t)1 << 21) - 1;
    }
  }
  if (qi < 0) qi = 0;
  return ((uint32_t)I << 21) | (uint32_t)qi;
}
static const uint32_t FP_OUT = 0xFFFFFFFFu, FP_CHAIN = 0xFFFFFFFEu;

static uint2 encode_packed(const Coords &c, int32_t code, double rF, double uF) {
  uint2 w;
  if (code == -1) {
    w.x = FP_OUT;
    w.y = 0;
  } else if (code <= -2) {
    w.x = FP_CHAIN;
    w.y = (uint32_t)(-2 - (int64_t)code);
  } else {
    w.x = pack_coord(code & 0xffff, rF, c.nr - 1);
    w.y = pack_coord(code >> 16, uF, c.nu - 1);
  }
  return w;
}

// Encoding of one cell: -1 -> outside the box (value 0), <= -2 -> delayed
// kernel chain (-2 - chain id), else rI | uI << 16 (FP64 tables); the FP32
// tables pack the same information into two 32-bit words.
static int encode_and_upload_footpoints(vls_handle *h, bool build_chains) {
  const Coords &c = h->co;
  const bool linked = !h->solver.noLinking;
  const double dtd = linked ? h->solver.dt * 2 : h->solver.dt;
  const bool refl = h->solver.kernelType == VLS_KERNEL_REFLECTIVE;
  const size_t slice = (size_t)c.nr * c.nu;
  const int batch = std::max(1, (int)std::min<size_t>(c.nj, (16u << 20) / slice));
  std::vector<int32_t> idx(slice * batch);
  std::vector<double> fx(slice * batch), fy(slice * batch);
  std::vector<uint2> packed;
  if (h->prec != VLS_FP64) packed.resize(slice * batch);
  std::vector<SliceFootpoints> sfp(batch);
  std::vector<SliceChains> sch(batch);
  if (build_chains) {
    h->ch_cell_h.clear();
    h->ch_len_h.clear();
    h->ch_R_h.clear();
    h->ch_U_h.clear();
  }
  std::string bad;
  for (int j0 = 0; j0 < c.nj; j0 += batch) {
    const int nb = std::min(batch, c.nj - j0);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < nb; b++) {
      slice_footpoints(c, j0 + b, dtd, refl, sfp[b]);
      if (build_chains && !refl) slice_chains(c, j0 + b, dtd, sfp[b], sch[b]);
    }
    // chain ids of this batch continue the running count, in slice order
    int64_t chain_base = (int64_t)h->ch_cell_h.size();
    for (int b = 0; b < nb; b++) {
      const SliceFootpoints &fp = sfp[b];
      if (fp.halted >= 0 && bad.empty()) {
        const int64_t cell = (int64_t)(j0 + b) * (int64_t)slice + fp.halted;
        bad = "reflective kernel: the footpoint of cell " + std::to_string(cell) +
              " reaches the reflection radius a second time, where the reference "
              "terminates (vlasovSolver21.hxx:389-391); use kernelBufferSize 0 or "
              "the delayed kernel";
      }
      int64_t next_chain = chain_base;
      for (size_t i = 0; i < slice; i++) {
        const size_t o = (size_t)b * slice + i;
        int32_t code;
        if (fp.driftR[i] < c.kernelRadius) {
          code = refl ? -1 : (int32_t)(-2 - next_chain++);
        } else if (fp.out[i]) {
          code = -1;
        } else {
          const int32_t rI = fp.rI[i], uI = fp.uI[i];
          if (rI < 0 || rI > c.nr - 1 || uI < 0 || uI > c.nu - 1) {
            bad = "footpoint index outside the spline box at cell " +
                  std::to_string((size_t)(j0 + b) * slice + i);
            code = -1;
          } else {
            code = rI | (uI << 16);
          }
        }
        idx[o] = code;
        fx[o] = fp.rF[i];
        fy[o] = fp.uF[i];
      }
      if (build_chains && !refl) {
        const SliceChains &ch = sch[b];
        if ((int64_t)ch.cell.size() != next_chain - chain_base)
          bad = "chain bookkeeping mismatch";
        h->ch_cell_h.insert(h->ch_cell_h.end(), ch.cell.begin(), ch.cell.end());
        h->ch_len_h.insert(h->ch_len_h.end(), ch.len.begin(), ch.len.end());
        h->ch_R_h.insert(h->ch_R_h.end(), ch.R.begin(), ch.R.end());
        h->ch_U_h.insert(h->ch_U_h.end(), ch.U.begin(), ch.U.end());
      }
      chain_base = next_chain;
    }
    if (!bad.empty()) return fail(h, VLS_EINVAL, bad);
    const size_t off = (size_t)j0 * slice, n = (size_t)nb * slice;
    if (h->prec == VLS_FP64) {
      TRY(upload(h, h->idx + off, idx.data(), n * sizeof(int32_t)));
      TRY(upload(h, (double *)h->fx + off, fx.data(), n * sizeof(double)));
      TRY(upload(h, (double *)h->fy + off, fy.data(), n * sizeof(double)));
    } else {
      for (size_t i = 0; i < n; i++) packed[i] = encode_packed(c, idx[i], fx[i], fy[i]);
      TRY(upload(h, h->fp2 + off, packed.data(), n * sizeof(uint2)));
    }
  }
  h->fp_gen++;
  return VLS_OK;
}

// localSpline::evaluate(R, U) position decomposition of every chain tail
// (vlasovSolver21_spline.hxx:776-786, localSpline.hxx:477-488)
static int setup_chain_device(vls_handle *h) {
  const Coords &c = h->co;
  const int64_t nch = (int64_t)h->ch_cell_h.size();
  h->nch = nch;
  h->ch_start_h.resize(nch);
  int64_t acc = 0;
  for (int64_t k = 0; k < nch; k++) {
    h->ch_start_h[k] = acc;
    acc += h->ch_len_h[k];
  }
  h->nel = acc;
  h->chain_lo.assign(c.nj + 1, nch);
  for (int64_t k = nch - 1; k >= 0; k--)
    h->chain_lo[h->ch_cell_h[k] / ((int64_t)c.nr * c.nu)] = k;
  for (int j = c.nj - 1; j >= 0; j--) h->chain_lo[j] = std::min(h->chain_lo[j], h->chain_lo[j + 1]);
  std::vector<int32_t> tcode(2 * std::max<int64_t>(nch, 1), 0);
  std::vector<double> tx(std::max<int64_t>(nch, 1), 0), ty(std::max<int64_t>(nch, 1), 0);
  for (int64_t k = 0; k < nch; k++) {
    const int64_t e = h->ch_start_h[k] + h->ch_len_h[k] - 1;
    const double R = h->ch_R_h[e], U = h->ch_U_h[e];
    const int j = (int)(h->ch_cell_h[k] / ((int64_t)c.nr * c.nu));
    tcode[nch + k] = j;
    if ((U <= c.U.front()) || (U >= c.U.back())) {
      tcode[k] = -1;
      continue;
    }
    double xr = (rescale(R, c.rscale) - c.sstart[0]) * c.sstep_inv[0];
    double yu = (rescale(U, c.uscale) - c.sstart[1]) * c.sstep_inv[1];
    double ix, iy;
    xr = std::modf(xr, &ix);
    yu = std::modf(yu, &iy);
    if (ix < 0 || ix > c.nr - 1 || iy < 0 || iy > c.nu - 1)
      return fail(h, VLS_EINVAL,
                  "a delayed-kernel chain tail lies outside the spline box "
                  "(time step too large for this grid)");
    tcode[k] = (int32_t)ix | ((int32_t)iy << 16);
    tx[k] = xr;
    ty[k] = yu;
  }
  const size_t es = h->esize;
  TRY(dalloc(h, &h->ch_start, sizeof(int64_t) * std::max<int64_t>(nch, 1)));
  TRY(dalloc(h, &h->ch_len, sizeof(int32_t) * std::max<int64_t>(nch, 1)));
  TRY(dalloc(h, &h->ch_val, es * std::max<int64_t>(h->nel, 1)));
  TRY(dalloc(h, &h->t_idx, sizeof(int32_t) * tcode.size()));
  TRY(dalloc(h, &h->t_x, sizeof(double) * tx.size()));
  TRY(dalloc(h, &h->t_y, sizeof(double) * ty.size()));
  CK(h, cudaMemsetAsync(h->ch_val, 0, es * std::max<int64_t>(h->nel, 1), h->st));
  if (nch) {
    TRY(upload(h, h->ch_start, h->ch_start_h.data(), sizeof(int64_t) * nch));
    TRY(upload(h, h->ch_len, h->ch_len_h.data(), sizeof(int32_t) * nch));
  }
  TRY(upload(h, h->t_idx, tcode.data(), sizeof(int32_t) * tcode.size()));
  TRY(upload(h, h->t_x, tx.data(), sizeof(double) * tx.size()));
  TRY(upload(h, h->t_y, ty.data(), sizeof(double) * ty.size()));
  return VLS_OK;
}

// 3D tiled tensor maps of C ([N_J][N_u+3][pc], element T): boxes of 64
// columns x 40 rows x 1 slice for the drift windows, 48 columns x 64 rows x 1
// slice for the strips.  The encoder is the driver's cuTensorMapEncodeTiled,
// reached through the runtime (no libcuda link).  Returns false when it is
// unavailable or refuses a map (vls_create then fails: every drift kernel
// stages its coefficients by TMA).
static bool make_tensor_map(vls_handle *h) {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return false;
  }
  auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  const cuuint64_t es = h->esize;
  const size_t slot = (size_t)h->B * (h->co.nu + 3) * h->pc;  // elements per slot
  for (int s = 0; s < h->NS; s++) {
    const cuuint64_t dims[3] = {(cuuint64_t)h->pc, (cuuint64_t)h->co.nu + 3,
                                (cuuint64_t)h->B};
    const cuuint64_t strides[2] = {(cuuint64_t)h->pc * es,
                                   (cuuint64_t)h->pc * es * (cuuint64_t)(h->co.nu + 3)};
    const cuuint32_t box[3] = {64, 40, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    void *base = (char *)h->C + s * slot * es;
    const CUresult r = enc(&h->tmC[s],
                           es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                           3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (h->drift_kind != DRIFT_WINDOW) {
      const cuuint32_t sbox[3] = {48, 64, 1};
      if (enc(&h->tmS[s],
              es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
              base, dims, strides, sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    }
  }
  return true;
}

// ------------------------------------------------------------- life cycle
extern "C" int vls_version(int32_t *major, int32_t *minor) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  return VLS_OK;
}

extern "C" int vls_device_ok(int32_t device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return fail(nullptr, VLS_ECUDA, "no CUDA device " + std::to_string(device));
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess)
    return fail(nullptr, VLS_ECUDA, "cudaGetDeviceProperties failed");
  if (p.major < 10)
    return fail(nullptr, VLS_ECUDA,
                "device is sm_" + std::to_string(p.major * 10 + p.minor) +
                    "; this library is built for sm_100a");
  return VLS_OK;
}

static void free_all(vls_handle *h) {
  for (auto &r : h->prof) {
    h->evpool.push_back(r.a);
    h->evpool.push_back(r.b);
  }
  h->prof.clear();
  for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
  h->evpool.clear();
  for (void *p : h->allocs) cudaFree(p);
  h->allocs.clear();
  for (void *p : h->adj_allocs) cudaFree(p);
  h->adj_allocs.clear();
  h->adj_ck.clear();
  h->adj_sub.clear();
  h->adj_final = vls_handle::Ckpt();
  h->ab_lam = h->ab_Cb = h->ab_Gb = h->ab_A = h->ab_B = nullptr;
  h->ab_ringb = h->ab_sbar = h->ab_beta = nullptr;
  h->ab_stash.clear();
  h->ab_shifts = nullptr;
  h->ab_nshift = 0;
  h->inv_ends = h->inv_ent = h->inv_tot = nullptr;
  h->inv_ebase = h->inv_chc = nullptr;
  h->inv_tv = nullptr;
  h->inv_geo = nullptr;
  h->inv_vperm = nullptr;
  h->inv_gen = ~(uint64_t)0;
  h->dev_bytes = 0;
  for (int k = 0; k < 8; k++) {
    if (h->bst[k]) cudaStreamDestroy(h->bst[k]);
    if (h->ev_join[k]) cudaEventDestroy(h->ev_join[k]);
    h->bst[k] = nullptr;
    h->ev_join[k] = nullptr;
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  h->ev_fork = nullptr;
  if (h->st) cudaStreamDestroy(h->st);
  h->st = nullptr;
}

extern "C" int vls_create(const vls_grid_desc *grid,
                          const vls_solver_desc *solver, vls_handle **out) {
  return vls_create_layout(grid, solver, nullptr, out);
}

extern "C" int vls_create_layout(const vls_grid_desc *grid, const vls_solver_desc *solver,
                                 const vls_layout_desc *layout, vls_handle **out) {
  if (!grid || !solver || !out)
    return fail(nullptr, VLS_EINVAL, "vls_create: NULL argument");
  *out = nullptr;
  const vls_layout_desc lay = layout ? *layout : vls_layout_desc{};
  if (lay.prefilter < VLS_PREFILTER_AUTO || lay.prefilter > VLS_PREFILTER_SEGMENT ||
      lay.drift < VLS_DRIFT_AUTO || lay.drift > VLS_DRIFT_STRIP1 || lay.slices_per_batch < 0 ||
      lay.streams < 0 || lay.streams > 8)
    return fail(nullptr, VLS_EINVAL, "vls_create: invalid layout descriptor");
  if (solver->precision != VLS_FP64 && solver->precision != VLS_FP32_BULK &&
      solver->precision != VLS_FP32_ALL)
    return fail(nullptr, VLS_EINVAL, "unknown precision");
  if (solver->kernelType != VLS_KERNEL_DELAYED &&
      solver->kernelType != VLS_KERNEL_REFLECTIVE)
    return fail(nullptr, VLS_EINVAL, "unknown kernel type");
  if (!(solver->dt > 0)) return fail(nullptr, VLS_EINVAL, "solver.dt must be > 0");
  {
    int s = vls_device_ok(solver->device);
    if (s != VLS_OK) return s;
  }
  std::unique_ptr<vls_handle> h(new vls_handle());
  h->grid = *grid;
  h->solver = *solver;
  h->prec = solver->precision;
  h->esize = h->prec == VLS_FP64 ? 8 : 4;
  h->time = solver->T0;
  {
    std::string e;
    if (!make_coords(*grid, solver->kernelBufferSize, h->co, e))
      return fail(nullptr, VLS_EINVAL, e);
  }
  const Coords &c = h->co;
  if (c.nr > 2048 || c.nu > 2048)
    return fail(nullptr, VLS_EINVAL, "at most 2048 vertices along r and along v_r");
  h->cells = (size_t)c.nr * c.nu * c.nj;
  h->pc = ((c.nr + 3) + 3) / 4 * 4;
  {
    const int per16 = (int)(16 / h->esize);
    h->gp = (c.nr + per16 - 1) / per16 * per16;
  }
  h->tr = thomas_tables(c.nr, c.sstep_inv[0]);
  h->tu = thomas_tables(c.nu, c.sstep_inv[1]);
  {
    // prefilter kernels: register chunks where a line fits them, else the
    // shared-memory segment kernels (for every line with
    // VLS_PREFILTER_SEGMENT)
    const bool seg = lay.prefilter == VLS_PREFILTER_SEGMENT;
    const bool r64 = h->prec == VLS_FP64 || h->prec == VLS_FP32_BULK;
    if (!seg) {
      h->rcu_cfg = r64 ? rc_config<double>(h->tu, true) : rc_config<float>(h->tu, true);
      h->rcr_cfg = r64 ? rc_config<double>(h->tr, false) : rc_config<float>(h->tr, false);
    }
    h->rcu_d = rc_dir<double>(h->tu, h->rcu_cfg);
    h->rcr_d = rc_dir<double>(h->tr, h->rcr_cfg);
    h->rcu_f = rc_dir<float>(h->tu, h->rcu_cfg);
    h->rcr_f = rc_dir<float>(h->tr, h->rcr_cfg);
  }
  if (cudaSetDevice(solver->device) != cudaSuccess)
    return fail(nullptr, VLS_ECUDA, "cudaSetDevice failed");
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(nullptr, VLS_ECUDA, "cudaStreamCreate failed");

  vls_handle *hp = h.get();
  int s = VLS_OK;
  auto A = [&](int st) {
    if (s == VLS_OK) s = st;
  };
  const size_t es = h->esize, cells = h->cells;
  {
    // slice batching (slices_per_batch, streams); default: one batch of
    // every slice
    h->B = lay.slices_per_batch > 0 ? std::min(c.nj, lay.slices_per_batch) : c.nj;
    h->nbatch = (c.nj + h->B - 1) / h->B;
    h->NS = std::max(1, lay.streams);
    h->NS = std::min(h->NS, h->nbatch);
    for (int k = 0; k < h->NS; k++)
      if (cudaStreamCreateWithFlags(&h->bst[k], cudaStreamNonBlocking) != cudaSuccess)
        return fail(nullptr, VLS_ECUDA, "cudaStreamCreate failed");
    if (cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess)
      return fail(nullptr, VLS_ECUDA, "cudaEventCreate failed");
    for (int k = 0; k < h->NS; k++)
      if (cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming) != cudaSuccess)
        return fail(nullptr, VLS_ECUDA, "cudaEventCreate failed");
  }
  A(dalloc(hp, &h->f, es * cells));
  A(dalloc(hp, &h->G, es * (size_t)h->NS * h->B * (c.nu + 2) * h->gp));
  A(dalloc(hp, &h->C, es * (size_t)h->NS * h->B * (c.nu + 3) * h->pc));
  {
    const size_t fcells = cells + (size_t)FOOT_PAD_ROWS * c.nr + 32;
    if (h->prec == VLS_FP64) {
      A(dalloc(hp, &h->idx, sizeof(int32_t) * fcells));
      A(dalloc(hp, &h->fx, es * fcells));
      A(dalloc(hp, &h->fy, es * fcells));
      if (s == VLS_OK && (cudaMemset(h->idx, 0, sizeof(int32_t) * fcells) != cudaSuccess ||
          cudaMemset(h->fx, 0, es * fcells) != cudaSuccess ||
          cudaMemset(h->fy, 0, es * fcells) != cudaSuccess))
        return fail(nullptr, VLS_ECUDA, "cudaMemset of the footpoint tables failed");
    } else {
      A(dalloc(hp, &h->fp2, sizeof(uint2) * fcells));
      if (s == VLS_OK && cudaMemset(h->fp2, 0, sizeof(uint2) * fcells) != cudaSuccess)
        return fail(nullptr, VLS_ECUDA, "cudaMemset of the footpoint tables failed");
    }
  }
  A(dalloc(hp, &h->rp_r, sizeof(double) * h->tr.M));
  A(dalloc(hp, &h->q_r, sizeof(double) * h->tr.M));
  A(dalloc(hp, &h->rp_u, sizeof(double) * h->tu.M));
  A(dalloc(hp, &h->q_u, sizeof(double) * h->tu.M));
  A(dalloc(hp, &h->dU_val, sizeof(double) * c.nu));
  A(dalloc(hp, &h->dR_val, sizeof(double) * c.nr));
  A(dalloc(hp, &h->dJ_val, sizeof(double) * c.nj));
  A(dalloc(hp, &h->d_dR, sizeof(double) * c.nr));
  A(dalloc(hp, &h->d_dU, sizeof(double) * c.nu));
  A(dalloc(hp, &h->d_Ct1, sizeof(double) * c.nj));
  A(dalloc(hp, &h->bu, sizeof(double) * c.nu));
  A(dalloc(hp, &h->bu32, sizeof(float) * c.nu));
  A(dalloc(hp, &h->wj, sizeof(double) * c.nj));
  A(dalloc(hp, &h->dR4, sizeof(double) * c.nr));
  A(dalloc(hp, &h->Rcoef, sizeof(double) * c.nr));
  A(dalloc(hp, &h->partial, sizeof(double) * (size_t)c.nj * c.nr));
  A(dalloc(hp, &h->T2, sizeof(double) * c.nr));
  A(dalloc(hp, &h->bins, sizeof(double) * c.nr));
  A(dalloc(hp, &h->Mr, sizeof(double) * c.nr));
  A(dalloc(hp, &h->shift, sizeof(double) * c.nr));
  A(dalloc(hp, &h->mtot, sizeof(double) * 2));
  A(dalloc(hp, &h->count, sizeof(unsigned int) * 4));
  A(dalloc(hp, &h->flag, sizeof(unsigned int) * 4));
  h->stats_nblk = (size_t)((c.nu + 7) / 8) * c.nj;
  A(dalloc(hp, &h->stats_part, sizeof(double) * 8 * h->stats_nblk));
  h->staging_n = std::min<size_t>(cells, (size_t)16 << 20);
  if (h->prec != VLS_FP64) A(dalloc(hp, &h->staging, sizeof(double) * h->staging_n));
  if (s != VLS_OK) {
    g_create_error = hp->err;
    free_all(hp);
    return s;
  }
  auto fin = [&](int st) -> int {
    if (st != VLS_OK) {
      g_create_error = hp->err;
      free_all(hp);
    }
    return st;
  };
  if (cudaMemsetAsync(h->C, 0, es * (size_t)h->NS * h->B * (c.nu + 3) * h->pc, h->st) !=
          cudaSuccess ||
      cudaMemsetAsync(h->count, 0, sizeof(unsigned int) * 4, h->st) != cudaSuccess ||
      cudaMemsetAsync(h->flag, 0, sizeof(unsigned int) * 4, h->st) != cudaSuccess)
    return fin(fail(hp, VLS_ECUDA, "cudaMemsetAsync failed"));
  // drift kernel: whole-strip staging where it fits (see vls_layout_desc)
  h->drift_kind = h->esize == 4 ? drift_strip_width<float>(c.nu, lay.drift)
                                : drift_strip_width<double>(c.nu, lay.drift);
  h->drift_spins = lay.drift_wait_spins == 0  ? MBAR_SPIN_LIMIT
                   : lay.drift_wait_spins < 0 ? 0u
                                              : (uint32_t)lay.drift_wait_spins;
  if (!make_tensor_map(hp))
    return fin(fail(hp, VLS_ECUDA, "TMA tensor maps of the spline coefficients unavailable"));
  h->layout = lay;
  h->layout.prefilter =
      (h->rcu_cfg >= 0 || h->rcr_cfg >= 0) ? VLS_PREFILTER_REGISTER : VLS_PREFILTER_SEGMENT;
  h->layout.drift = h->drift_kind;
  h->layout.slices_per_batch = h->B;
  h->layout.streams = h->NS;
  h->layout.drift_wait_spins = (int32_t)std::min<uint32_t>(h->drift_spins, 0x7fffffffu);
  h->layout.u_chunk_rows = rc_chunk_rows(h->rcu_cfg);
  h->layout.r_chunk_rows = rc_chunk_rows(h->rcr_cfg);
  // tables
  std::vector<double> dR(c.nr), dU(c.nu), Ct1(c.nj), bu(c.nu), wj(c.nj), dR4(c.nr),
      Rcoef(c.nr);
  for (int r = 0; r < c.nr; r++) {
    dR[r] = (r >= c.nr - 1) ? 0 : (c.R[r + 1] - c.R[r]);  // get_dR
    dR4[r] = dR[r] * 0.25;
    // vlasovSolver21_spline.hxx:746: Mr[i] *= G/(R*R)*dt
    Rcoef[r] = h->solver.G / (c.R[r] * c.R[r]) * h->solver.dt;
  }
  for (int u = 0; u < c.nu; u++) dU[u] = (u >= c.nu - 1) ? 0 : (c.U[u + 1] - c.U[u]);
  for (int u = 0; u < c.nu; u++) bu[u] = dU[u] + (u > 0 ? dU[u - 1] : 0.0);
  for (int j = 0; j < c.nj; j++) {
    // get_dJ compares j with the u-vertex count (slice21Iterator.hxx:86)
    const double dJ = (j >= c.nu - 1) ? 0 : (c.JV[j + 1] - c.JV[j]);
    Ct1[j] = 8 * M_PI * M_PI * c.J[j] * dJ;
    wj[j] = Ct1[j];
  }
  int st2 = VLS_OK;
  auto U2 = [&](void *d, const void *src, size_t b) {
    if (st2 == VLS_OK) st2 = upload(hp, d, src, b);
  };
  U2(h->rp_r, h->tr.rp.data(), sizeof(double) * h->tr.M);
  U2(h->q_r, h->tr.q.data(), sizeof(double) * h->tr.M);
  U2(h->rp_u, h->tu.rp.data(), sizeof(double) * h->tu.M);
  U2(h->q_u, h->tu.q.data(), sizeof(double) * h->tu.M);
  U2(h->dU_val, c.U.data(), sizeof(double) * c.nu);
  U2(h->dR_val, c.R.data(), sizeof(double) * c.nr);
  U2(h->dJ_val, c.J.data(), sizeof(double) * c.nj);
  U2(h->d_dR, dR.data(), sizeof(double) * c.nr);
  U2(h->d_dU, dU.data(), sizeof(double) * c.nu);
  U2(h->d_Ct1, Ct1.data(), sizeof(double) * c.nj);
  U2(h->bu, bu.data(), sizeof(double) * c.nu);
  {
    const std::vector<float> b32(bu.begin(), bu.end());
    U2(h->bu32, b32.data(), sizeof(float) * c.nu);
  }
  U2(h->wj, wj.data(), sizeof(double) * c.nj);
  U2(h->dR4, dR4.data(), sizeof(double) * c.nr);
  U2(h->Rcoef, Rcoef.data(), sizeof(double) * c.nr);
  if (fin(st2) != VLS_OK) return st2;
  if (fin(encode_and_upload_footpoints(hp, true)) != VLS_OK) return VLS_EINVAL;
  {
    const int st3 = setup_chain_device(hp);
    if (fin(st3) != VLS_OK) return st3;
  }
  *out = h.release();
  return VLS_OK;
}

extern "C" int vls_get_layout(const vls_handle *h, vls_layout_desc *used) {
  if (!h || !used) return VLS_EINVAL;
  *used = h->layout;
  return VLS_OK;
}

extern "C" int vls_destroy(vls_handle *h) {
  if (!h) return VLS_OK;
  cudaSetDevice(h->solver.device);
  if (h->st) cudaStreamSynchronize(h->st);
  free_all(h);
  delete h;
  return VLS_OK;
}

extern "C" const char *vls_last_error(const vls_handle *h) {
  return h ? h->err.c_str() : g_create_error.c_str();
}

extern "C" int vls_dims(const vls_handle *h, int64_t *nr, int64_t *nu,
                        int64_t *nj) {
  if (!h) return VLS_EINVAL;
  if (nr) *nr = h->co.nr;
  if (nu) *nu = h->co.nu;
  if (nj) *nj = h->co.nj;
  return VLS_OK;
}

extern "C" int vls_coords(const vls_handle *h, double *R, double *U, double *J,
                          double *JV) {
  if (!h) return VLS_EINVAL;
  if (R) std::memcpy(R, h->co.R.data(), sizeof(double) * h->co.nr);
  if (U) std::memcpy(U, h->co.U.data(), sizeof(double) * h->co.nu);
  if (J) std::memcpy(J, h->co.J.data(), sizeof(double) * h->co.nj);
  if (JV) std::memcpy(JV, h->co.JV.data(), sizeof(double) * (h->co.nj + 1));
  return VLS_OK;
}

static int check_device_flags(vls_handle *h);

// ------------------------------------------------------------- f transfer
static int put_f(vls_handle *h, const double *host) {
  if (h->prec == VLS_FP64) {
    CK(h, cudaMemcpyAsync(h->f, host, sizeof(double) * h->cells,
                          cudaMemcpyHostToDevice, h->st));
  } else {
    for (size_t off = 0; off < h->cells; off += h->staging_n) {
      const size_t n = std::min(h->staging_n, h->cells - off);
      CK(h, cudaMemcpyAsync(h->staging, host + off, sizeof(double) * n,
                            cudaMemcpyHostToDevice, h->st));
      CK(h, timed(h, VLS_K_CONVERT, [&] {
           return launch_convert_in<float>(h->staging, (float *)h->f + off, n, h->st);
         }));
    }
  }
  // non-finite values in the uploaded grid: status word bit 0
  CK(h, h->prec == VLS_FP64
            ? launch_nonfinite<double>((const double *)h->f, h->cells, h->flag + 2, h->st)
            : launch_nonfinite<float>((const float *)h->f, h->cells, h->flag + 2, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  h->have_f = true;
  h->moments_valid = false;
  return check_device_flags(h);
}

static int take_f(vls_handle *h, double *host) {
  if (h->prec == VLS_FP64) {
    CK(h, cudaMemcpyAsync(host, h->f, sizeof(double) * h->cells,
                          cudaMemcpyDeviceToHost, h->st));
  } else {
    for (size_t off = 0; off < h->cells; off += h->staging_n) {
      const size_t n = std::min(h->staging_n, h->cells - off);
      CK(h, timed(h, VLS_K_CONVERT, [&] {
           return launch_convert_out<float>((const float *)h->f + off, h->staging, n,
                                            h->st);
         }));
      CK(h, cudaMemcpyAsync(host + off, h->staging, sizeof(double) * n,
                            cudaMemcpyDeviceToHost, h->st));
    }
  }
  CK(h, cudaStreamSynchronize(h->st));
  return check_device_flags(h);
}

extern "C" int vls_set_f(vls_handle *h, const double *host, size_t n) {
  if (!h || !host) return fail(h, VLS_EINVAL, "vls_set_f: NULL argument");
  if (n != h->cells) return fail(h, VLS_EINVAL, "vls_set_f: size mismatch");
  CK(h, cudaSetDevice(h->solver.device));
  return put_f(h, host);
}

extern "C" int vls_get_f(vls_handle *h, double *host, size_t n) {
  if (!h || !host) return fail(h, VLS_EINVAL, "vls_get_f: NULL argument");
  if (n != h->cells) return fail(h, VLS_EINVAL, "vls_get_f: size mismatch");
  if (!h->have_f) return fail(h, VLS_ESTATE, "vls_get_f: no grid data yet");
  CK(h, cudaSetDevice(h->solver.device));
  return take_f(h, host);
}

// ----------------------------------------------------------- init profile
extern "C" int vls_init_profile(vls_handle *h, const vls_init_desc *init,
                                double *mass_before) {
  if (!h || !init) return fail(h, VLS_EINVAL, "vls_init_profile: NULL argument");
  if (init->type < VLS_INIT_UDF || init->type > VLS_INIT_HERNQUIST)
    return fail(h, VLS_EINVAL, "unknown initial conditions type");
  CK(h, cudaSetDevice(h->solver.device));
  const Coords &c = h->co;
  Profile pr;
  pr.setup(*init, h->solver.G);
  std::vector<double> f(h->cells);
#pragma omp parallel for schedule(dynamic)
  for (int j = 0; j < c.nj; j++)
    for (int u = 0; u < c.nu; u++)
      for (int r = 0; r < c.nr; r++)
        f[((size_t)j * c.nu + u) * c.nr + r] = pr.value(c.R[r], c.U[u], c.J[j]);
  // quadrature21::integrate (quadrature21.hxx:56-85) in its one-thread order
  double mass = 0;
  for (int j = 0; j < c.nj; j++) {
    const double J = c.J[j];
    const double dJ = (j >= c.nu - 1) ? 0 : (c.JV[j + 1] - c.JV[j]);
    const double Ct1 = 8 * M_PI * M_PI * J * dJ;
    for (int u = 0; u < c.nu; u++) {
      const double dU = (u >= c.nu - 1) ? 0 : (c.U[u + 1] - c.U[u]);
      if (dU <= 0) continue;
      for (int r = 0; r < c.nr; r++) {
        const double dR = (r >= c.nr - 1) ? 0 : (c.R[r + 1] - c.R[r]);
        if (dR <= 0) continue;
        const double *fi = &f[((size_t)j * c.nu + u) * c.nr + r];
        const double avg = (fi[0] + fi[1] + fi[c.nr] + fi[c.nr + 1]) * 0.25;
        mass += Ct1 * dU * dR * avg;
      }
    }
  }
  if (mass_before) *mass_before = mass;
  // chain element values: init->valueAt at each element, tail 0
  // (vlasovSolver21.hxx:307-320)
  std::vector<double> vals(h->nel, 0.0);
  for (int64_t k = 0; k < h->nch; k++) {
    const int j = (int)(h->ch_cell_h[k] / ((int64_t)c.nr * c.nu));
    const int64_t s0 = h->ch_start_h[k];
    for (int32_t e = 0; e + 1 < h->ch_len_h[k]; e++)
      vals[s0 + e] = pr.value(h->ch_R_h[s0 + e], h->ch_U_h[s0 + e], c.J[j]);
  }
  // vlasovSolver21::renormalize(init->getMass(0), 0) (vlasovSolver21.hxx:468-524)
  if (init->M > 0) {
    const double fac = init->M / mass;
#pragma omp parallel for
    for (long long i = 0; i < (long long)h->cells; i++) f[i] *= fac;
    for (auto &v : vals) v *= fac;
  }
  TRY(put_f(h, f.data()));
  // the ring position restarts before the values are placed (they are given
  // in logical order, front first)
  h->ndrift = 0;
  TRY(vls_set_chain_values(h, vals.data(), h->nel));
  return VLS_OK;
}

// ----------------------------------------------------------------- chains
extern "C" int vls_get_chains(const vls_handle *hc, int64_t *n_chains,
                              int64_t *n_elems, int64_t *cell, int64_t *start,
                              int32_t *len, double *R, double *U, double *val) {
  vls_handle *h = const_cast<vls_handle *>(hc);
  if (!h) return VLS_EINVAL;
  if (n_chains) *n_chains = h->nch;
  if (n_elems) *n_elems = h->nel;
  if (cell) std::memcpy(cell, h->ch_cell_h.data(), sizeof(int64_t) * h->nch);
  if (start) std::memcpy(start, h->ch_start_h.data(), sizeof(int64_t) * h->nch);
  if (len) std::memcpy(len, h->ch_len_h.data(), sizeof(int32_t) * h->nch);
  if (R) std::memcpy(R, h->ch_R_h.data(), sizeof(double) * h->nel);
  if (U) std::memcpy(U, h->ch_U_h.data(), sizeof(double) * h->nel);
  if (val && h->nel) {
    // device ring buffers -> logical order (front first)
    CK(h, cudaSetDevice(h->solver.device));
    std::vector<double> phys(h->nel);
    if (h->prec == VLS_FP64) {
      CK(h, cudaMemcpyAsync(phys.data(), h->ch_val, sizeof(double) * h->nel,
                            cudaMemcpyDeviceToHost, h->st));
      CK(h, cudaStreamSynchronize(h->st));
    } else {
      std::vector<float> p32(h->nel);
      CK(h, cudaMemcpyAsync(p32.data(), h->ch_val, sizeof(float) * h->nel,
                            cudaMemcpyDeviceToHost, h->st));
      CK(h, cudaStreamSynchronize(h->st));
      for (int64_t i = 0; i < h->nel; i++) phys[i] = p32[i];
    }
    for (int64_t k = 0; k < h->nch; k++) {
      const int64_t s0 = h->ch_start_h[k];
      const int32_t L = h->ch_len_h[k];
      for (int32_t e = 0; e < L; e++) val[s0 + e] = phys[s0 + (h->ndrift + e) % L];
    }
  }
  return VLS_OK;
}

extern "C" int vls_set_chain_values(vls_handle *h, const double *val,
                                    int64_t n_elems) {
  if (!h) return VLS_EINVAL;
  if (n_elems != h->nel) return fail(h, VLS_EINVAL, "chain element count mismatch");
  if (!h->nel) return VLS_OK;
  CK(h, cudaSetDevice(h->solver.device));
  std::vector<double> phys(h->nel);
  for (int64_t k = 0; k < h->nch; k++) {
    const int64_t s0 = h->ch_start_h[k];
    const int32_t L = h->ch_len_h[k];
    for (int32_t e = 0; e < L; e++) phys[s0 + (h->ndrift + e) % L] = val[s0 + e];
  }
  if (h->prec == VLS_FP64) {
    TRY(upload(h, h->ch_val, phys.data(), sizeof(double) * h->nel));
  } else {
    std::vector<float> p32(h->nel);
    for (int64_t i = 0; i < h->nel; i++) p32[i] = (float)phys[i];
    TRY(upload(h, h->ch_val, p32.data(), sizeof(float) * h->nel));
  }
  // the values are loaded either way; a non-finite one is reported
  for (int64_t i = 0; i < h->nel; i++)
    if (!std::isfinite(val[i]))
      return fail(h, VLS_ENAN, "non-finite delayed-kernel chain value at element " +
                                   std::to_string(i));
  return VLS_OK;
}

// ------------------------------------------------------------- footpoints
extern "C" int vls_get_footpoints(const vls_handle *hc, int32_t *rI, double *rF,
                                  int32_t *uI, double *uF, uint8_t *out,
                                  double *driftR) {
  vls_handle *h = const_cast<vls_handle *>(hc);
  if (!h) return VLS_EINVAL;
  const Coords &c = h->co;
  const double dtd = h->solver.noLinking ? h->solver.dt : h->solver.dt * 2;
  const bool refl = h->solver.kernelType == VLS_KERNEL_REFLECTIVE;
  const size_t slice = (size_t)c.nr * c.nu;
#pragma omp parallel for schedule(dynamic)
  for (int j = 0; j < c.nj; j++) {
    SliceFootpoints fp;
    slice_footpoints(c, j, dtd, refl, fp);
    const size_t o = (size_t)j * slice;
    for (size_t i = 0; i < slice; i++) {
      if (rI) rI[o + i] = fp.rI[i];
      if (rF) rF[o + i] = fp.rF[i];
      if (uI) uI[o + i] = fp.uI[i];
      if (uF) uF[o + i] = fp.uF[i];
      if (out) out[o + i] = fp.out[i];
      if (driftR) driftR[o + i] = fp.driftR[i];
    }
  }
  return VLS_OK;
}

extern "C" int vls_set_footpoints(vls_handle *h, const int32_t *rI,
                                  const double *rF, const int32_t *uI,
                                  const double *uF, const uint8_t *out,
                                  const double *driftR) {
  if (!h || !rI || !rF || !uI || !uF || !out || !driftR)
    return fail(h, VLS_EINVAL, "vls_set_footpoints: NULL argument");
  CK(h, cudaSetDevice(h->solver.device));
  const Coords &c = h->co;
  // the chain layout stays the one built at creation: cells whose footpoint
  // falls inside the kernel radius must be the same cells
  std::vector<int32_t> idx(h->cells);
  int64_t next_chain = 0;
  for (size_t i = 0; i < h->cells; i++) {
    if (driftR[i] < c.kernelRadius) {
      if (h->solver.kernelType == VLS_KERNEL_REFLECTIVE) {
        idx[i] = -1;
        continue;
      }
      if (next_chain >= h->nch || h->ch_cell_h[next_chain] != (int64_t)i)
        return fail(h, VLS_EINVAL,
                    "vls_set_footpoints: kernel cells differ from the chain layout");
      idx[i] = (int32_t)(-2 - next_chain++);
    } else if (out[i]) {
      idx[i] = -1;
    } else {
      if (rI[i] < 0 || rI[i] > c.nr - 1 || uI[i] < 0 || uI[i] > c.nu - 1)
        return fail(h, VLS_EINVAL, "vls_set_footpoints: index outside the grid");
      idx[i] = rI[i] | (uI[i] << 16);
    }
  }
  if (h->prec == VLS_FP64) {
    TRY(upload(h, h->idx, idx.data(), sizeof(int32_t) * h->cells));
    TRY(upload(h, h->fx, rF, sizeof(double) * h->cells));
    TRY(upload(h, h->fy, uF, sizeof(double) * h->cells));
  } else {
    std::vector<uint2> p(h->cells);
    for (size_t i = 0; i < h->cells; i++) p[i] = encode_packed(c, idx[i], rF[i], uF[i]);
    TRY(upload(h, h->fp2, p.data(), sizeof(uint2) * h->cells));
  }
  h->fp_gen++;
  return VLS_OK;
}

// ------------------------------------------------------------------ step
template <typename R>
static const RcDir<R> &rcdir(const vls_handle *h, bool u);
template <>
const RcDir<double> &rcdir<double>(const vls_handle *h, bool u) {
  return u ? h->rcu_d : h->rcr_d;
}
template <>
const RcDir<float> &rcdir<float>(const vls_handle *h, bool u) {
  return u ? h->rcu_f : h->rcr_f;
}

// One split step: f_out = D P_r P_u Kick(P_u f_in).  f_in, f_out and the
// kick's shift are the handle's unless given (the adjoint's recomputation
// steps from one stored state into the next with the shift it stored); f_in
// and f_out may be the same buffer.
template <typename T, typename R>
static int drift_once(vls_handle *h, bool kick, const void *f_in = nullptr,
                      void *f_out = nullptr, const double *shift = nullptr) {
  const T *fin = (const T *)(f_in ? f_in : h->f);
  T *fout = (T *)(f_out ? f_out : h->f);
  const double *sft = shift ? shift : h->shift;
  const DirTables tu = dir_tables(h->tu, h->rp_u, h->q_u);
  const DirTables tr = dir_tables(h->tr, h->rp_r, h->q_r);
  const size_t gslot = (size_t)h->B * (h->co.nu + 2) * h->gp;
  const size_t cslot = (size_t)h->B * (h->co.nu + 3) * h->pc;
  CK(h, cudaEventRecord(h->ev_fork, h->st));
  for (int k = 0; k < h->NS; k++) CK(h, cudaStreamWaitEvent(h->bst[k], h->ev_fork, 0));
  for (int b = 0; b < h->nbatch; b++) {
    const int sl = b % h->NS;
    cudaStream_t bs = h->bst[sl];
    Geometry g = geometry(h);
    g.j0 = b * h->B;
    g.nb = std::min(h->B, h->co.nj - g.j0);
    T *G = (T *)h->G + sl * gslot;
    T *C = (T *)h->C + sl * cslot;
    CK(h, timed(
              h, kick ? VLS_K_UCOL_KICK : VLS_K_UCOL,
              [&] {
                if (h->rcu_cfg >= 0)
                  return launch_ucol_rc<T, R>(h->rcu_cfg, kick, fin, G, sft, g,
                                              rcdir<R>(h, true), bs);
                return launch_ucol<T, R>(kick, fin, G, sft, g, tu, bs);
              },
              bs));
    CK(h, timed(
              h, VLS_K_PRER,
              [&] {
                if (h->rcr_cfg >= 0)
                  return launch_prer_rc<T, R>(h->rcr_cfg, G, C, g, rcdir<R>(h, false),
                                              h->flag + 1, bs);
                return launch_prer<T, R>(G, C, g, tr, bs);
              },
              bs));
    const int64_t c_lo = h->chain_lo[g.j0], c_hi = h->chain_lo[g.j0 + g.nb];
    if (c_hi > c_lo) {
      CK(h, timed(
                h, VLS_K_TAILS,
                [&] {
                  return launch_chain_tails<T>(C, (T *)h->ch_val, h->ch_start, h->ch_len,
                                               h->t_idx, h->t_x, h->t_y, h->nch, c_lo,
                                               c_hi, h->ndrift, g, bs);
                },
                bs));
    }
    CK(h, timed(
              h, VLS_K_DRIFT,
              [&] {
                if (h->drift_kind != DRIFT_WINDOW)
                  return launch_drift_strip<T>(&h->tmS[sl], h->drift_kind, C, fout,
                                               h->idx, (const T *)h->fx, (const T *)h->fy,
                                               h->fp2, h->ch_start, h->ch_len,
                                               (const T *)h->ch_val, h->ndrift,
                                               moment_tables(h), h->partial, h->flag + 1,
                                               h->drift_spins, g, bs);
                return launch_drift_tma<T>(&h->tmC[sl], C, fout, h->idx,
                                           (const T *)h->fx, (const T *)h->fy, h->fp2,
                                           h->ch_start, h->ch_len, (const T *)h->ch_val,
                                           h->ndrift, moment_tables(h), h->partial,
                                           h->flag + 1, h->drift_spins, g, bs);
              },
              bs));
  }
  for (int k = 0; k < h->NS; k++) {
    CK(h, cudaEventRecord(h->ev_join[k], h->bst[k]));
    CK(h, cudaStreamWaitEvent(h->st, h->ev_join[k], 0));
  }
  h->ndrift++;
  h->moments_valid = true;
  return VLS_OK;
}

template <typename T>
static int ensure_moments(vls_handle *h) {
  if (h->moments_valid) return VLS_OK;
  const Geometry g = geometry(h);
  CK(h, timed(h, VLS_K_MOMENT, [&] {
       return launch_moment<T>((const T *)h->f, moment_tables(h), h->partial, g, h->st);
     }));
  h->moments_valid = true;
  return VLS_OK;
}

// shift_out: where the shift goes (the handle's unless given)
static int scan_once(vls_handle *h, double *shift_out = nullptr) {
  const Geometry g = geometry(h);
  CK(h, timed(h, VLS_K_SCAN, [&] {
       return launch_scan(h->partial, moment_tables(h), h->T2, h->bins, h->Mr,
                          shift_out ? shift_out : h->shift, h->mtot, h->count, h->flag + 2,
                          g, h->st);
     }));
  return VLS_OK;
}

template <typename T, typename R>
static int step_impl(vls_handle *h, int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    if (h->solver.noLinking) TRY((drift_once<T, R>(h, false)));
    TRY(ensure_moments<T>(h));
    TRY(scan_once(h));
    TRY((drift_once<T, R>(h, true)));
    h->time += h->solver.dt;
    h->step++;
  }
  return VLS_OK;
}

extern "C" int vls_step(vls_handle *h, int32_t nsteps) {
  if (!h) return VLS_EINVAL;
  if (nsteps < 0) return fail(h, VLS_EINVAL, "nsteps < 0");
  if (!h->have_f) return fail(h, VLS_ESTATE, "vls_step before the grid was set");
  CK(h, cudaSetDevice(h->solver.device));
  switch (h->prec) {
    case VLS_FP64:
      return step_impl<double, double>(h, nsteps);
    case VLS_FP32_BULK:
      return step_impl<float, double>(h, nsteps);
    default:
      return step_impl<float, float>(h, nsteps);
  }
}

// One linked step from the state f_in, whose shift scan_once has just
// computed into `shift`, to f_out (the adjoint's recomputation).
static int step_between(vls_handle *h, const void *f_in, void *f_out, const double *shift) {
  int rc;
  switch (h->prec) {
    case VLS_FP64:
      rc = drift_once<double, double>(h, true, f_in, f_out, shift);
      break;
    case VLS_FP32_BULK:
      rc = drift_once<float, double>(h, true, f_in, f_out, shift);
      break;
    default:
      rc = drift_once<float, float>(h, true, f_in, f_out, shift);
  }
  if (rc != VLS_OK) return rc;
  h->time += h->solver.dt;
  h->step++;
  return VLS_OK;
}

// device-side status words, cleared once reported:
// flag[1] bit 0/1 = a bounded mbarrier wait of the drift timed out (the step
// then read global memory instead; results stay valid but the hardware path
// misbehaved); bit 2/3 = the r-solve's bulk row staging timed out (that
// step's results are not valid);
// flag[2] bit 0 = a non-finite value in a grid uploaded from the host; bit 1
// = the enclosed-mass scan of a step found a non-finite total mass (a NaN or
// an infinity in f at the start of that step)
static int check_device_flags(vls_handle *h) {
  unsigned int fl[4] = {0, 0, 0, 0};
  CK(h, cudaMemcpyAsync(fl, h->flag, sizeof(fl), cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  if (fl[1] || fl[2]) {
    CK(h, cudaMemsetAsync(h->flag, 0, sizeof(fl), h->st));
    CK(h, cudaStreamSynchronize(h->st));
  }
  if (fl[1])
    return fail(h, VLS_ECUDA,
                (fl[1] & 12u) ? "a bounded device wait timed out in the r-solve kernel"
                              : "a bounded device wait timed out in the drift kernel");
  if (fl[2])
    return fail(h, VLS_ENAN,
                (fl[2] & 1u) ? "non-finite value in the grid loaded from the host"
                             : "non-finite value in the grid: the total mass of a step "
                               "is not finite");
  return VLS_OK;
}

extern "C" int vls_sync(vls_handle *h) {
  if (!h) return VLS_EINVAL;
  CK(h, cudaSetDevice(h->solver.device));
  CK(h, cudaStreamSynchronize(h->st));
  CK(h, cudaGetLastError());
  return check_device_flags(h);
}

extern "C" int vls_kernel_launches(const vls_handle *h, int64_t *n) {
  if (!h || !n) return VLS_EINVAL;
  *n = h->launches;
  return VLS_OK;
}

extern "C" int vls_stream(const vls_handle *h, void **stream) {
  if (!h || !stream) return VLS_EINVAL;
  *stream = (void *)h->st;
  return VLS_OK;
}

extern "C" int vls_set_profiling(vls_handle *h, int32_t on) {
  if (!h) return VLS_EINVAL;
  h->profiling = on != 0;
  return VLS_OK;
}

extern "C" int vls_profile_read(vls_handle *h, double *ms, int64_t *count,
                                int32_t nk) {
  if (!h) return VLS_EINVAL;
  CK(h, cudaSetDevice(h->solver.device));
  CK(h, cudaStreamSynchronize(h->st));
  for (int k = 0; k < nk; k++) {
    if (ms) ms[k] = 0;
    if (count) count[k] = 0;
  }
  for (auto &r : h->prof) {
    float t = 0;
    CK(h, cudaEventElapsedTime(&t, r.a, r.b));
    if (r.kind < nk) {
      if (ms) ms[r.kind] += t;
      if (count) count[r.kind]++;
    }
    h->evpool.push_back(r.a);
    h->evpool.push_back(r.b);
  }
  h->prof.clear();
  return VLS_OK;
}

// --------------------------------------------------------------- moments
template <typename T>
static int moments_impl(vls_handle *h) {
  TRY(ensure_moments<T>(h));
  return scan_once(h);
}

extern "C" int vls_moments(vls_handle *h, double *bins, double *Mr, double *mtot) {
  if (!h) return VLS_EINVAL;
  if (!h->have_f) return fail(h, VLS_ESTATE, "vls_moments before the grid was set");
  CK(h, cudaSetDevice(h->solver.device));
  TRY(h->prec == VLS_FP64 ? moments_impl<double>(h) : moments_impl<float>(h));
  const int nr = h->co.nr;
  if (bins)
    CK(h, cudaMemcpyAsync(bins, h->bins, sizeof(double) * nr, cudaMemcpyDeviceToHost,
                          h->st));
  if (Mr)
    CK(h, cudaMemcpyAsync(Mr, h->Mr, sizeof(double) * nr, cudaMemcpyDeviceToHost, h->st));
  if (mtot)
    CK(h, cudaMemcpyAsync(mtot, h->mtot, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  return VLS_OK;
}

extern "C" int vls_last_mass(vls_handle *h, double *mtot) {
  if (!h || !mtot) return VLS_EINVAL;
  CK(h, cudaSetDevice(h->solver.device));
  CK(h, cudaMemcpyAsync(mtot, h->mtot, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  return VLS_OK;
}

extern "C" int vls_last_mass_async(vls_handle *h, double *mtot) {
  if (!h || !mtot) return VLS_EINVAL;
  CK(h, cudaSetDevice(h->solver.device));
  CK(h, cudaMemcpyAsync(mtot, h->mtot, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  return VLS_OK;
}

// ------------------------------------------------------------------ stats
static void two_sum_acc(double &s, double &c, double x) {
  const double t = s + x;
  const double bb = t - s;
  c += (s - (t - bb)) + (x - bb);
  s = t;
}

template <typename T>
static int stats_impl(vls_handle *h, vls_stats_out *o) {
  const Coords &c = h->co;
  TRY(moments_impl<T>(h));
  std::vector<double> bins(c.nr);
  CK(h, cudaMemcpyAsync(bins.data(), h->bins, sizeof(double) * c.nr,
                        cudaMemcpyDeviceToHost, h->st));
  CK(h, timed(h, VLS_K_STATS, [&] {
       return launch_stats<T>((const T *)h->f, h->dR_val, h->dU_val, h->dJ_val,
                              h->d_dR, h->d_dU, h->d_Ct1, h->stats_part, nullptr,
                              geometry(h), h->st);
     }));
  std::vector<double> part(8 * h->stats_nblk);
  CK(h, cudaMemcpyAsync(part.data(), h->stats_part, sizeof(double) * part.size(),
                        cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  double q[4];
  for (int k = 0; k < 4; k++) {
    double s = 0, cc = 0;
    for (size_t b = 0; b < h->stats_nblk; b++) {
      two_sum_acc(s, cc, part[b * 8 + 2 * k]);
      two_sum_acc(s, cc, part[b * 8 + 2 * k + 1]);
    }
    q[k] = s + cc;
  }
  // vlasovSolver21::potentialEnergy (vlasovSolver21.hxx:627-642); the last
  // shell (mass 0) is skipped instead of reading past R_Val
  double M = 0, Ep = 0;
  for (int i = 1; i < c.nr + 1; i++) {
    const double Mi = bins[i - 1];
    if (i < c.nr) {
      const double r = 0.5 * (c.R[i - 1] + c.R[i]);
      Ep -= (Mi * h->solver.G * M) / r;
    }
    M += Mi;
  }
  o->time = h->time;
  o->step = h->step;
  o->Mass = M;
  o->Ek = q[0];
  o->Ep = Ep;
  o->E = q[0] + Ep;
  o->S = q[1];
  o->L1 = q[2];
  o->L2 = q[3];
  return VLS_OK;
}

extern "C" int vls_stats(vls_handle *h, vls_stats_out *out) {
  if (!h || !out) return fail(h, VLS_EINVAL, "vls_stats: NULL argument");
  if (!h->have_f) return fail(h, VLS_ESTATE, "vls_stats before the grid was set");
  CK(h, cudaSetDevice(h->solver.device));
  return h->prec == VLS_FP64 ? stats_impl<double>(h, out) : stats_impl<float>(h, out);
}

extern "C" int vls_get_time(const vls_handle *h, double *time, int64_t *step) {
  if (!h) return VLS_EINVAL;
  if (time) *time = h->time;
  if (step) *step = h->step;
  return VLS_OK;
}

extern "C" int vls_set_time(vls_handle *h, double time, int64_t step) {
  if (!h) return VLS_EINVAL;
  h->time = time;
  h->step = step;
  return VLS_OK;
}

// ---------------------------------------------------------------- NDfield
// Save_NDfield (NDfield.hxx:308-363) of NDfieldFromData (vlasovSolver21.hxx:717-773)
namespace {
const int ND_MAX_DIMS = 20;
const int ND_DOUBLE_T = 1 << 9;
}  // namespace

extern "C" int vls_write_ndfield(vls_handle *h, const char *path) {
  if (!h || !path) return fail(h, VLS_EINVAL, "vls_write_ndfield: NULL argument");
  if (!h->have_f) return fail(h, VLS_ESTATE, "no grid data");
  std::vector<double> f(h->cells);
  TRY(take_f(h, f.data()));
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return fail(h, VLS_EIO, std::string("cannot open ") + path);
  const vls_grid_desc &g = h->grid;
  int dims[3] = {g.Pres + 1, g.Ures[0] + 1, g.Ures[1]};
  double x0[3] = {g.Pmin, g.Umin[0], g.Umin[1]};
  double delta[3] = {g.Pmax - g.Pmin, g.Umax[0] - g.Umin[0], g.Umax[1] - g.Umin[1]};
  char comment[80];
  std::memset(comment, 0, sizeof(comment));
  // (Rscale, VERTEX=1, Uscale, VERTEX=1, Jscale, CELL=0)
  std::snprintf(comment, sizeof(comment), "%d %d %d %d %d %d", g.Pscale, 1,
                g.Uscale[0], 1, g.Uscale[1], 0);
  char tag[16];
  std::memset(tag, 0, sizeof(tag));
  std::strcpy(tag, "NDFIELD");
  char dummy[160];
  std::memset(dummy, 0, sizeof(dummy));
  int i = 16;
  bool ok = true;
  auto W = [&](const void *p, size_t sz, size_t n) {
    ok = ok && std::fwrite(p, sz, n, fp) == n;
  };
  W(&i, sizeof(int), 1);
  W(tag, 1, 16);
  W(&i, sizeof(int), 1);
  i = (int)(sizeof(int) * (ND_MAX_DIMS + 3) + sizeof(double) * (2 * ND_MAX_DIMS) +
            (160 + 80) * sizeof(char));
  W(&i, sizeof(int), 1);
  W(comment, 1, 80);
  const int ndims = 3;
  W(&ndims, sizeof(int), 1);
  W(dims, sizeof(int), 3);
  W(dummy, sizeof(int), ND_MAX_DIMS - 3);
  const int fdims_index = 0, dtype = ND_DOUBLE_T;
  W(&fdims_index, sizeof(int), 1);
  W(&dtype, sizeof(int), 1);
  W(x0, sizeof(double), 3);
  W(dummy, sizeof(double), ND_MAX_DIMS - 3);
  W(delta, sizeof(double), 3);
  W(dummy, sizeof(double), ND_MAX_DIMS - 3);
  W(dummy, 1, 160);
  W(&i, sizeof(int), 1);
  // record marker is an int: nval*8 wraps above 2 GiB exactly as the
  // reference's does (NDfield.hxx:355)
  const int marker = (int)(uint32_t)(h->cells * sizeof(double));
  W(&marker, sizeof(int), 1);
  W(f.data(), sizeof(double), h->cells);
  W(&marker, sizeof(int), 1);
  if (std::fclose(fp) != 0) ok = false;
  if (!ok) return fail(h, VLS_EIO, std::string("write failed: ") + path);
  return VLS_OK;
}

extern "C" int vls_read_ndfield(vls_handle *h, const char *path) {
  if (!h || !path) return fail(h, VLS_EINVAL, "vls_read_ndfield: NULL argument");
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return fail(h, VLS_EIO, std::string("cannot open ") + path);
  std::unique_ptr<FILE, int (*)(FILE *)> guard(fp, std::fclose);
  int m0, m1, hs;
  char tag[16];
  if (std::fread(&m0, 4, 1, fp) != 1 || std::fread(tag, 1, 16, fp) != 16 ||
      std::fread(&m1, 4, 1, fp) != 1 || m0 != 16 || m1 != 16 ||
      std::strncmp(tag, "NDFIELD", 7) != 0)
    return fail(h, VLS_EIO, "not an NDfield file (bad tag record)");
  if (std::fread(&hs, 4, 1, fp) != 1 || hs != 652)
    return fail(h, VLS_EIO, "unsupported NDfield header size");
  char comment[80];
  int ndims, dims[ND_MAX_DIMS], fdi, dtype;
  if (std::fread(comment, 1, 80, fp) != 80 || std::fread(&ndims, 4, 1, fp) != 1 ||
      std::fread(dims, 4, ND_MAX_DIMS, fp) != (size_t)ND_MAX_DIMS ||
      std::fread(&fdi, 4, 1, fp) != 1 || std::fread(&dtype, 4, 1, fp) != 1)
    return fail(h, VLS_EIO, "truncated NDfield header");
  if (ndims != 3 || dims[0] != h->co.nr || dims[1] != h->co.nu || dims[2] != h->co.nj)
    return fail(h, VLS_EIO, "NDfield dimensions do not match the grid");
  if (dtype != ND_DOUBLE_T) return fail(h, VLS_EIO, "NDfield datatype is not DOUBLE");
  if (std::fseek(fp, 4 + 16 + 4 + 4 + 652 + 4, SEEK_SET) != 0)
    return fail(h, VLS_EIO, "seek failed");
  int marker;
  if (std::fread(&marker, 4, 1, fp) != 1 ||
      marker != (int)(uint32_t)(h->cells * sizeof(double)))
    return fail(h, VLS_EIO, "NDfield data record size mismatch");
  std::vector<double> f(h->cells);
  if (std::fread(f.data(), sizeof(double), h->cells, fp) != h->cells)
    return fail(h, VLS_EIO, "truncated NDfield data");
  CK(h, cudaSetDevice(h->solver.device));
  return put_f(h, f.data());
}

// ------------------------------------------------------------------ adjoint
// Reverse-mode derivative of N linked steps (vls_adjoint.cu holds the
// transposed kernels).  vls_adjoint_forward runs the steps and keeps a copy
// of the state every K steps; vls_adjoint_backward walks the segments
// backwards, recomputes each segment's states from its checkpoint, and
// applies the transposed step to the adjoint field from the last step to the
// first.  Memory: ceil(N/K) + 1 checkpoints and K states of f, plus six FP64
// arrays of about one grid each.
// Device buffers of the adjoint stay with the handle between runs (every
// forward/backward pair of an optimisation loop would otherwise allocate and
// free ~10 grids); vls_destroy frees them.
static void adj_release(vls_handle *h) {
  h->adj_ready = false;
  h->adj_grad = false;
}

template <typename P>
static int adj_alloc(vls_handle *h, P **p, size_t bytes) {
  void *q = nullptr;
  if (bytes == 0) bytes = 16;
  const cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, VLS_ECUDA,
                "adjoint: cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                    cudaGetErrorString(e));
  }
  h->adj_allocs.push_back(q);
  h->dev_bytes += bytes;
  *p = reinterpret_cast<P *>(q);
  return VLS_OK;
}

static int ckpt_save(vls_handle *h, vls_handle::Ckpt &c) {
  const size_t fb = h->esize * h->cells, cb = h->esize * (size_t)h->nel;
  if (!c.f) {
    TRY(adj_alloc(h, &c.f, fb));
    TRY(adj_alloc(h, &c.ch, cb));
  }
  CK(h, cudaMemcpyAsync(c.f, h->f, fb, cudaMemcpyDeviceToDevice, h->st));
  if (cb) CK(h, cudaMemcpyAsync(c.ch, h->ch_val, cb, cudaMemcpyDeviceToDevice, h->st));
  c.ndrift = h->ndrift;
  c.time = h->time;
  c.step = h->step;
  return VLS_OK;
}

static int ckpt_load(vls_handle *h, const vls_handle::Ckpt &c) {
  const size_t fb = h->esize * h->cells, cb = h->esize * (size_t)h->nel;
  CK(h, cudaMemcpyAsync(h->f, c.f, fb, cudaMemcpyDeviceToDevice, h->st));
  if (cb) CK(h, cudaMemcpyAsync(h->ch_val, c.ch, cb, cudaMemcpyDeviceToDevice, h->st));
  h->ndrift = c.ndrift;
  h->time = c.time;
  h->step = c.step;
  h->moments_valid = false;
  return VLS_OK;
}

extern "C" int vls_adjoint_forward(vls_handle *h, int32_t nsteps, int32_t checkpoint_every) {
  if (!h) return VLS_EINVAL;
  if (nsteps < 1 || checkpoint_every < 1)
    return fail(h, VLS_EINVAL, "adjoint: nsteps and checkpoint_every must be >= 1");
  if (h->solver.noLinking)
    return fail(h, VLS_EINVAL, "adjoint: only the linked step (noLinking = false) is supported");
  if (!h->have_f) return fail(h, VLS_ESTATE, "adjoint: the grid was not set");
  CK(h, cudaSetDevice(h->solver.device));
  CK(h, cudaStreamSynchronize(h->st));
  adj_release(h);
  const int ncp = (nsteps + checkpoint_every - 1) / checkpoint_every;
  if ((int)h->adj_ck.size() < ncp) h->adj_ck.resize(ncp);  // new entries allocate on first save
  for (int s = 0; s < nsteps; ++s) {
    if (s % checkpoint_every == 0) TRY(ckpt_save(h, h->adj_ck[s / checkpoint_every]));
    TRY(vls_step(h, 1));
  }
  TRY(ckpt_save(h, h->adj_final));
  h->adj_n = nsteps;
  h->adj_K = checkpoint_every;
  h->adj_ncp = ncp;
  h->adj_ready = true;
  return VLS_OK;
}

namespace {
struct AdjBufs {
  double *lam, *Cb, *Gb, *A, *B, *ringb, *sbar, *beta;
  std::vector<void *> stash;
  std::vector<int64_t> ndrift;
  // chunked line kernels (else one thread per line through A and B)
  bool rc = false;
  // lam still lacks the moment term in beta[N_r..2 N_r): the next step's
  // readers of lam (chain fronts and the gather) add it, or the end does
  bool pending = false;
  bool perm = true;  // FP32 handles: the gather over entry-ordered values
  // shift of each stashed state (N_r per state), saved by the recomputation
  double *shifts = nullptr;
  RcDir<double> rcu{}, rcr{};
};
}  // namespace

// The inverse footpoint map of the current footpoints for the drift's
// transpose (launch_inv_fill), built once per footpoint set: count, scan,
// place, order.
// FP32 handles whose adjoint field (8 B per cell) does not fit in L2 read
// the drift transpose's entries in entry order, after a permutation pass
// each step; below that the cell-ordered reads hit L2 and the pass costs
// more than it saves (FP32 per transposed step: 257 x 257 x 128 0.155 ms
// cell-ordered against 0.184; 513 x 513 x 256 1.035 against 0.978; 1025 x
// 1025 x 64 1.015 against 0.933).  FP64 handles read their 16 B of
// fractions through the cell index at every size.
template <typename T>
static bool adj_entry_ordered(vls_handle *h) {
  if (sizeof(T) != 4) return false;
  int l2 = 0;
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->solver.device) != cudaSuccess)
    l2 = 0;
  return h->cells * sizeof(double) > (size_t)l2;
}

template <typename T>
static int ensure_inv(vls_handle *h) {
  if (h->inv_gen == h->fp_gen) return VLS_OK;
  const Geometry g = geometry(h);
  const int64_t nch = h->nch;
  if (!h->inv_ends) {
    TRY(adj_alloc(h, &h->inv_ends, h->cells * sizeof(uint32_t)));
    TRY(adj_alloc(h, &h->inv_ent, (h->cells + (size_t)nch) * sizeof(uint32_t)));
    TRY(adj_alloc(h, &h->inv_tot, (size_t)g.nj * sizeof(uint32_t)));
    TRY(adj_alloc(h, &h->inv_ebase, (size_t)(g.nj + 1) * sizeof(int64_t)));
    TRY(adj_alloc(h, &h->inv_chc, (size_t)std::max<int64_t>(nch, 1) * sizeof(int64_t)));
    TRY(adj_alloc(h, &h->inv_tv, (size_t)std::max<int64_t>(nch, 1) * sizeof(double)));
    if (adj_entry_ordered<T>(h)) {
      const size_t ne = h->cells + (size_t)nch;
      TRY(adj_alloc(h, &h->inv_geo, ne * sizeof(uint2)));
      TRY(adj_alloc(h, &h->inv_vperm, ne * sizeof(double)));
    }
  }
  if (nch) TRY(upload(h, h->inv_chc, h->ch_cell_h.data(), sizeof(int64_t) * nch));
  CK(h, cudaMemsetAsync(h->inv_ends, 0, h->cells * sizeof(uint32_t), h->st));
  CK(h, launch_inv_fill<T>(h->idx, h->fp2, h->t_idx, nch, h->inv_ends, nullptr,
                           nullptr, g, h->st));
  CK(h, launch_inv_scan(h->inv_ends, h->inv_tot, g, h->st));
  std::vector<uint32_t> tot((size_t)g.nj);
  CK(h, cudaMemcpyAsync(tot.data(), h->inv_tot, sizeof(uint32_t) * g.nj, cudaMemcpyDeviceToHost,
                        h->st));
  CK(h, cudaStreamSynchronize(h->st));
  std::vector<int64_t> eb((size_t)g.nj + 1, 0);
  for (int j = 0; j < g.nj; ++j) eb[j + 1] = eb[j] + tot[j];
  if ((size_t)eb[g.nj] > h->cells + (size_t)nch)
    return fail(h, VLS_ECUDA, "adjoint: inverse footpoint map larger than its cells");
  TRY(upload(h, h->inv_ebase, eb.data(), sizeof(int64_t) * eb.size()));
  CK(h, launch_inv_fill<T>(h->idx, h->fp2, h->t_idx, nch, h->inv_ends, h->inv_ent,
                           h->inv_ebase, g, h->st));
  CK(h, launch_inv_sort(h->inv_ends, h->inv_ent, h->inv_ebase, g, h->st));
  if (h->inv_geo) {
    CK(h, launch_inv_geo(h->inv_ent, h->inv_ebase, h->fp2, h->inv_geo, g, h->st));
    h->launches++;
  }
  h->launches += 4;
  h->inv_gen = h->fp_gen;
  return VLS_OK;
}

template <typename T>
// the transposed step n: state f_n, its drift count and its shift s(f_n)
static int adj_step(vls_handle *h, AdjBufs &b, const void *fn, int64_t ndrift,
                    const double *shift) {
  const Geometry g = geometry(h);
  const MomentTables mt = moment_tables(h);
  const DirTables tu = dir_tables(h->tu, h->rp_u, h->q_u);
  const DirTables tr = dir_tables(h->tr, h->rp_r, h->q_r);
  {
    // lam of this step is lam + the moment term of the step after it, when
    // that was left pending
    const double *mB = b.pending ? b.beta + g.nr : nullptr;
    if (h->nch > 0)
      CK(h, timed(h, VLS_K_ADJ_TAILS, [&] {
        return launch_chain_adj(b.lam, mB, mt, b.ringb, h->inv_tv, h->inv_chc, h->ch_start,
                                h->ch_len, h->nch, ndrift, g, h->st);
      }));
    if (b.perm) {
      CK(h, timed(h, VLS_K_ADJ_DRIFT, [&] {
        return launch_inv_perm(h->inv_ent, h->inv_ebase, b.lam, mB, mt, h->inv_tv, h->inv_vperm,
                               g, h->st);
      }));
      CK(h, timed(h, VLS_K_ADJ_DRIFT, [&] {
        return launch_drift_adj_gather_perm(h->inv_vperm, h->inv_geo, b.Cb, h->inv_ends,
                                            h->inv_ebase, h->t_idx, h->t_x, h->t_y, g, h->st);
      }));
    } else
    CK(h, timed(h, VLS_K_ADJ_DRIFT, [&] {
      return launch_drift_adj_gather<T>(b.lam, mB, mt, h->inv_tv, b.Cb, h->inv_ends,
                                        h->inv_ent, h->inv_ebase, (const T *)h->fx,
                                        (const T *)h->fy, h->fp2, h->t_x, h->t_y, g,
                                        h->st);
    }));
  }
  CK(h, timed(h, VLS_K_ADJ_PRER, [&] {
    return b.rc ? launch_prer_adj_rc(b.Cb, b.Gb, g, b.rcr, h->st)
                : launch_prer_adj(b.Cb, b.Gb, g, tr, h->st);
  }));
  CK(h, timed(h, VLS_K_ADJ_UCOL, [&] {
    return b.rc ? launch_ucol_adj_rc<T>((const T *)fn, b.Gb, b.lam, b.sbar, shift, g, b.rcu,
                                        h->st)
                : launch_ucol_adj<T>((const T *)fn, b.Gb, b.A, b.B, b.lam, b.sbar, shift, g, tu,
                                     h->st);
  }));
  // count[1]: the shift transpose's blocks (count[0] is the scan's)
  CK(h, timed(h, VLS_K_ADJ_MOMENT, [&] {
    return launch_shift_adj(b.sbar, b.beta, h->count + 1, mt, g, h->st);
  }));
  b.pending = true;  // added by the next step's readers of lam, or at the end
  return VLS_OK;
}

template <typename T>
static int adjoint_backward_impl(vls_handle *h, const double *dbins, double *df0,
                                 double *dchain0) {
  const Geometry g = geometry(h);
  const MomentTables mt = moment_tables(h);
  const size_t cells = h->cells;
  const size_t gn = (size_t)g.nj * (g.nu + 2) * g.nr;
  AdjBufs b{};
  {
    // chunked transposed line solves where the forward prefilter uses
    // register chunks and the lines fit them; the entry-ordered gather for
    // FP32 handles whose adjoint field does not fit in L2, the cell-ordered
    // one otherwise
    b.rc = rc_adj_supported(h->tu, h->tr) && h->layout.prefilter != VLS_PREFILTER_SEGMENT;
    b.rcu = rc_dir<double>(h->tu, 2);
    b.rcr = rc_dir<double>(h->tr, 2);
    b.perm = adj_entry_ordered<T>(h);
  }
  TRY(ensure_inv<T>(h));
  if (!h->ab_lam || (h->ab_rc != b.rc && !b.rc)) {
    if (!h->ab_lam) {
      TRY(adj_alloc(h, &h->ab_lam, cells * sizeof(double)));
      TRY(adj_alloc(h, &h->ab_Cb, (size_t)g.nj * (g.nu + 3) * g.pc * sizeof(double)));
      TRY(adj_alloc(h, &h->ab_Gb, gn * sizeof(double)));
      TRY(adj_alloc(h, &h->ab_ringb, (size_t)std::max<int64_t>(h->nel, 1) * sizeof(double)));
      TRY(adj_alloc(h, &h->ab_sbar, (size_t)g.nj * g.nr * sizeof(double)));
      TRY(adj_alloc(h, &h->ab_beta, (size_t)2 * g.nr * sizeof(double)));
    }
    // scratch of the one-thread-per-line kernels
    TRY(adj_alloc(h, &h->ab_A, (b.rc ? 1 : gn) * sizeof(double)));
    TRY(adj_alloc(h, &h->ab_B, (b.rc ? 1 : gn) * sizeof(double)));
    h->ab_rc = b.rc;
  }
  b.lam = h->ab_lam;
  b.Cb = h->ab_Cb;
  b.Gb = h->ab_Gb;
  b.A = h->ab_A;
  b.B = h->ab_B;
  b.ringb = h->ab_ringb;
  b.sbar = h->ab_sbar;
  b.beta = h->ab_beta;
  const int K = h->adj_K;
  // states stashed per pass: the whole segment (K), or with a second level of
  // checkpoints every K2 steps, K2 states plus ceil(K / K2) checkpoints
  int K2 = h->adj_inner > 0 ? std::min(h->adj_inner, K) : K;
  if (h->adj_inner <= 0) {
    size_t fr = 0, tot = 0;
    CK(h, cudaMemGetInfo(&fr, &tot));
    const size_t state = h->esize * cells, ckb = state + h->esize * (size_t)h->nel;
    const size_t have = h->ab_stash.size() * state + h->adj_sub.size() * ckb;
    const size_t margin = std::max<size_t>(tot / 50, (size_t)1 << 30);
    const size_t room = (fr > margin ? fr - margin : 0) + have;
    if ((size_t)K * state > room) {
      // two levels cost one more forward run whatever the spacing, so take
      // the spacing with the fewest stored states, K2 + ceil(K / K2) (about
      // 2 sqrt(K)); the larger spacing on a tie
      K2 = 1;
      for (int k = 1; k < K; ++k)
        if (k + (K + k - 1) / k <= K2 + (K + K2 - 1) / K2) K2 = k;
      if ((size_t)K2 * state + (size_t)((K + K2 - 1) / K2) * ckb > room)
        return fail(h, VLS_ENOMEM,
                    "adjoint: the states of one segment do not fit in device memory");
    }
  }
  const bool two_level = K2 < K;
  while ((int)h->ab_stash.size() < K2) {
    void *q = nullptr;
    TRY(adj_alloc(h, &q, h->esize * cells));
    h->ab_stash.push_back(q);
  }
  if (two_level && (int)h->adj_sub.size() < (K + K2 - 1) / K2)
    h->adj_sub.resize((K + K2 - 1) / K2);  // entries allocate on first save
  b.stash.assign(h->ab_stash.begin(), h->ab_stash.begin() + K2);
  b.ndrift.assign(K2, 0);
  if (h->ab_nshift < K2) {
    TRY(adj_alloc(h, &h->ab_shifts, (size_t)K2 * g.nr * sizeof(double)));
    h->ab_nshift = K2;
  }
  b.shifts = h->ab_shifts;
  // seed: the derivative of the loss with respect to the final radial bins
  TRY(upload(h, b.beta, dbins, (size_t)g.nr * sizeof(double)));
  CK(h, cudaMemsetAsync(b.lam, 0, cells * sizeof(double), h->st));
  CK(h, cudaMemsetAsync(b.ringb, 0, (size_t)std::max<int64_t>(h->nel, 1) * sizeof(double), h->st));
  CK(h, launch_moment_adj(b.lam, b.beta, mt, g, h->st));
  // from the state at step a (in h->f): stash the states of steps a .. e-1,
  // each step reading its state from the stash and writing the next one
  // there, then apply the transposed steps e-1 .. a.  h->f keeps the state
  // of step a, and the moments (valid after each step) are those of the
  // last state stashed.
  auto pass = [&](int64_t a, int64_t e) -> int {
    CK(h, cudaMemcpyAsync(b.stash[0], h->f, h->esize * cells, cudaMemcpyDeviceToDevice, h->st));
    for (int64_t n = a; n < e; ++n) {
      b.ndrift[n - a] = h->ndrift;
      // the shift of step n, as the step computes it from f_n, kept for the
      // transposed step
      double *sn = b.shifts + (size_t)(n - a) * g.nr;
      TRY(ensure_moments<T>(h));
      TRY(scan_once(h, sn));
      if (n + 1 < e) TRY(step_between(h, b.stash[n - a], b.stash[n + 1 - a], sn));
    }
    for (int64_t n = e - 1; n >= a; --n)
      TRY(adj_step<T>(h, b, b.stash[n - a], b.ndrift[n - a], b.shifts + (size_t)(n - a) * g.nr));
    return VLS_OK;
  };
  const int ncp = h->adj_ncp;
  for (int seg = ncp - 1; seg >= 0; --seg) {
    const int64_t n0 = (int64_t)seg * K;
    const int64_t n1 = std::min<int64_t>(n0 + K, h->adj_n);
    TRY(ckpt_load(h, h->adj_ck[seg]));
    if (!two_level || n1 - n0 <= K2) {
      TRY(pass(n0, n1));
      continue;
    }
    // second level: run through the segment keeping a state every K2 steps,
    // then take its sub-segments from the last
    const int nsub = (int)((n1 - n0 + K2 - 1) / K2);
    for (int s = 0; s < nsub; ++s) {
      TRY(ckpt_save(h, h->adj_sub[s]));
      if (s + 1 < nsub) TRY(vls_step(h, K2));
    }
    for (int s = nsub - 1; s >= 0; --s) {
      TRY(ckpt_load(h, h->adj_sub[s]));
      const int64_t a = n0 + (int64_t)s * K2;
      TRY(pass(a, std::min<int64_t>(a + K2, n1)));
    }
  }
  h->adj_last_inner = two_level ? K2 : 0;
  if (b.pending) CK(h, launch_moment_adj(b.lam, b.beta, mt, g, h->st));
  // results: the derivative with respect to the initial grid and the initial
  // chain values (logical ring order at the first step)
  CK(h, cudaMemcpyAsync(df0, b.lam, cells * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  std::vector<double> rb((size_t)h->nel);
  if (h->nel)
    CK(h, cudaMemcpyAsync(rb.data(), b.ringb, rb.size() * sizeof(double),
                          cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  h->adj_dch0.assign((size_t)h->nel, 0.0);
  {
    const int64_t nd0 = h->adj_ck[0].ndrift;
    for (int64_t c = 0; c < h->nch; ++c) {
      const int64_t s0 = h->ch_start_h[c];
      const int32_t L = h->ch_len_h[c];
      for (int32_t e = 0; e < L; e++) h->adj_dch0[s0 + e] = rb[s0 + (nd0 + e) % L];
    }
  }
  if (dchain0 && h->nel) std::memcpy(dchain0, h->adj_dch0.data(), sizeof(double) * h->nel);
  h->adj_grad = true;
  // back to the final state of the forward run
  TRY(ckpt_load(h, h->adj_final));
  CK(h, cudaGetLastError());
  return VLS_OK;
}

// <dL/df0, f(plus) - f(minus)> and <dL/dc0, c(plus) - c(minus)> for the last
// backward pass's dL/df0 (still in ab_lam) and dL/dc0: f and c the
// renormalised initial grid and chain values of two parameter sets, the grid
// evaluated on the device (vls_profile.cu) into the backward's scratch
// arrays, its mass by the reference's quadrature with the rows summed in
// (j, u) order, the chain values on the host as vls_init_profile makes them
extern "C" int vls_adjoint_init_dot(vls_handle *h, const vls_init_desc *plus,
                                    const vls_init_desc *minus, double *dgrid, double *dchain) {
  if (!h) return VLS_EINVAL;
  if (!plus || !minus || !dgrid || !dchain)
    return fail(h, VLS_EINVAL, "vls_adjoint_init_dot: NULL argument");
  for (const vls_init_desc *d : {plus, minus})
    if (d->type < VLS_INIT_UDF || d->type > VLS_INIT_HERNQUIST)
      return fail(h, VLS_EINVAL, "unknown initial conditions type");
  if (!h->adj_grad)
    return fail(h, VLS_ESTATE, "vls_adjoint_init_dot before vls_adjoint_backward");
  CK(h, cudaSetDevice(h->solver.device));
  const Coords &c = h->co;
  const size_t cells = h->cells, nrow = (size_t)c.nu * c.nj;
  const int nb = profile_dot_blocks();
  if (!h->ip_xyz) {
    std::vector<double> xyz;
    xyz.insert(xyz.end(), c.R.begin(), c.R.end());
    xyz.insert(xyz.end(), c.U.begin(), c.U.end());
    xyz.insert(xyz.end(), c.J.begin(), c.J.end());
    xyz.insert(xyz.end(), c.JV.begin(), c.JV.end());
    TRY(adj_alloc(h, &h->ip_xyz, xyz.size() * sizeof(double)));
    TRY(adj_alloc(h, &h->ip_rows, nrow * sizeof(double)));
    TRY(adj_alloc(h, &h->ip_part, (size_t)nb * sizeof(double)));
    TRY(upload(h, h->ip_xyz, xyz.data(), xyz.size() * sizeof(double)));
  }
  double *fgrid[2] = {h->ab_Gb, h->ab_Cb};  // each holds at least one grid
  double fac[2];
  std::vector<double> vals[2];
  std::vector<double> rows(nrow);
  for (int s = 0; s < 2; ++s) {
    const vls_init_desc &d = s ? *minus : *plus;
    Profile pr;
    pr.setup(d, h->solver.G);
    ProfileConsts pc;
    pc.type = pr.d.type;
    pc.R0 = pr.d.R0;
    pc.smoothingRadius = pr.d.smoothingRadius;
    pc.gap0 = pr.d.gap[0];
    pc.gap1 = pr.d.gap[1];
    pc.n = pr.d.n;
    pc.M = pr.d.M;
    pc.Ra = pr.d.Ra;
    pc.G = pr.G;
    pc.C0 = pr.C0;
    pc.C1 = pr.C1;
    pc.C2 = pr.C2;
    pc.Vg = pr.Vg;
    CK(h, launch_profile_grid(pc, h->ip_xyz, fgrid[s], c.nr, c.nu, c.nj, h->st));
    CK(h, launch_profile_rows(fgrid[s], h->ip_xyz, h->ip_rows, c.nr, c.nu, c.nj, h->st));
    CK(h, cudaMemcpyAsync(rows.data(), h->ip_rows, nrow * sizeof(double),
                          cudaMemcpyDeviceToHost, h->st));
    CK(h, cudaStreamSynchronize(h->st));
    double mass = 0.0;
    for (size_t i = 0; i < nrow; ++i) mass += rows[i];
    fac[s] = d.M > 0 ? d.M / mass : 1.0;
    vals[s].assign((size_t)h->nel, 0.0);
    for (int64_t k = 0; k < h->nch; k++) {
      const int j = (int)(h->ch_cell_h[k] / ((int64_t)c.nr * c.nu));
      const int64_t s0 = h->ch_start_h[k];
      for (int32_t e = 0; e + 1 < h->ch_len_h[k]; e++)
        vals[s][s0 + e] = pr.value(h->ch_R_h[s0 + e], h->ch_U_h[s0 + e], c.J[j]) * fac[s];
    }
  }
  std::vector<double> part((size_t)nb);
  CK(h, launch_profile_dot(h->ab_lam, fgrid[0], fgrid[1], fac[0], fac[1], cells, h->ip_part,
                           h->st));
  CK(h, cudaMemcpyAsync(part.data(), h->ip_part, (size_t)nb * sizeof(double),
                        cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  double dg = 0.0;
  for (int b = 0; b < nb; ++b) dg += part[b];
  double dc = 0.0;
  for (int64_t i = 0; i < h->nel; ++i) dc += h->adj_dch0[i] * (vals[0][i] - vals[1][i]);
  *dgrid = dg;
  *dchain = dc;
  return VLS_OK;
}

extern "C" int vls_device_bytes(vls_handle *h, size_t *bytes) {
  if (!h || !bytes) return VLS_EINVAL;
  *bytes = h->dev_bytes;
  return VLS_OK;
}

extern "C" int vls_adjoint_set_inner(vls_handle *h, int32_t inner_every) {
  if (!h) return VLS_EINVAL;
  if (inner_every < 0) return fail(h, VLS_EINVAL, "adjoint: inner_every must be >= 0");
  h->adj_inner = inner_every;
  return VLS_OK;
}

extern "C" int vls_adjoint_inner_used(vls_handle *h, int32_t *inner_every) {
  if (!h || !inner_every) return VLS_EINVAL;
  *inner_every = h->adj_last_inner;
  return VLS_OK;
}

extern "C" int vls_adjoint_backward(vls_handle *h, const double *dbins, int64_t nbins,
                                    double *df0, size_t ncells, double *dchain0,
                                    int64_t nelems) {
  if (!h || !dbins || !df0) return VLS_EINVAL;
  if (!h->adj_ready) return fail(h, VLS_ESTATE, "adjoint: run vls_adjoint_forward first");
  if (nbins != h->co.nr || ncells != h->cells || (dchain0 && nelems != h->nel))
    return fail(h, VLS_EINVAL, "adjoint: buffer sizes do not match the grid");
  for (int64_t r = 0; r < nbins; r++)
    if (!std::isfinite(dbins[r]))
      return fail(h, VLS_ENAN, "adjoint: non-finite dL/dbins at bin " + std::to_string(r));
  CK(h, cudaSetDevice(h->solver.device));
  const int rc = h->esize == 8 ? adjoint_backward_impl<double>(h, dbins, df0, dchain0)
                               : adjoint_backward_impl<float>(h, dbins, df0, dchain0);
  if (rc != VLS_OK) return rc;
  return check_device_flags(h);
}

// ------------------------------------------------------------------ restart
// .vls restart files in the reference's layout (vlasovSolver::write,
// vlasovSolver.hxx:272-287 and the chain it calls): endianness word, tagged
// sections (int length + characters) with 2048-byte spares, the FP64 grid
// [j][u][r], and the delayed-kernel chains per J slice in ascending cell
// order (its std::map order), each as length + (R, U, nVal = 1, value) per
// element, front first.  gridBase::paramT::write writes Pmax with the count of
// U and Umin with the count of P (grid_base.hxx:129-130), so the six doubles
// are Pmin, Pmax, Umin[0], Umin[0], Umax[0], Umax[1]; Umin[1] (the J minimum)
// is not in the file.
namespace {
const char *const TAG_SOLVER = "VLASOV_SOLVER v0.13";
const char *const TAG_GH = "GRID_HANDLER v0.11";
const char *const TAG_GB = "GRID_BASE v0.12";
const char *const TAG_G21 = "GRID_21 v0.11";
const char *const TAG_S21 = "VLASOV_SOLVER21 v0.12";
const char *const TAG_KERNEL = "KERNEL_CELLS v0.10";
const char *const TAG_SPLINE = "VLASOV_SOLVER21_SPLINE v0.11";
constexpr size_t SPARE = 256 * 8;
constexpr size_t PARAM_SPARE = SPARE - sizeof(int32_t) * (3 + 3) - sizeof(int64_t);

struct Out {
  std::vector<char> b;
  template <typename V>
  void put(V v) {
    const char *p = reinterpret_cast<const char *>(&v);
    b.insert(b.end(), p, p + sizeof(V));
  }
  void tag(const char *s) {
    const int32_t n = (int32_t)std::strlen(s);
    put(n);
    b.insert(b.end(), s, s + n);
  }
  void zeros(size_t n) { b.insert(b.end(), n, 0); }
  void param(const vls_grid_desc &g) {
    put(g.Pmin);
    put(g.Pmax);
    put(g.Umin[0]);
    put(g.Umin[0]);
    put(g.Umax[0]);
    put(g.Umax[1]);
    put(g.Pres);
    put(g.Ures[0]);
    put(g.Ures[1]);
    put(g.Pscale);
    put(g.Uscale[0]);
    put(g.Uscale[1]);
    for (int i = 0; i < 6; ++i) put((int32_t)0);  // margins: P low/high, U low/high
    put((int32_t)1);                               // nFields
    put((int32_t)0);                               // haveParentGrid
    put((int32_t)1);                               // parent_P_DIMS
    put((int32_t)2);                               // parent_U_DIMS
    put((int32_t)0);                               // parent_which
    put((int32_t)1);
    put((int32_t)2);
    put((int64_t)0);  // minStorageSize
    zeros(PARAM_SPARE);
  }
};

struct In {
  const std::vector<char> &b;
  size_t o = 0;
  bool swap = false, bad = false;
  std::string why;
  explicit In(const std::vector<char> &v) : b(v) {}
  template <typename V>
  V get() {
    V v{};
    if (o + sizeof(V) > b.size()) {
      if (!bad) why = "file too short";
      bad = true;
      return v;
    }
    std::memcpy(&v, b.data() + o, sizeof(V));
    o += sizeof(V);
    if (swap) {
      char *p = reinterpret_cast<char *>(&v);
      std::reverse(p, p + sizeof(V));
    }
    return v;
  }
  void tag(const char *s) {
    const int32_t n = get<int32_t>();
    const size_t len = std::strlen(s);
    if (bad) return;
    if ((size_t)n != len || o + len > b.size() || std::memcmp(b.data() + o, s, len) != 0) {
      bad = true;
      why = std::string("tag '") + s + "' not found";
      return;
    }
    o += len;
  }
  void skip(size_t n) {
    if (o + n > b.size()) {
      if (!bad) why = "file too short";
      bad = true;
      return;
    }
    o += n;
  }
  void param(vls_grid_desc &g) {
    g.Pmin = get<double>();
    g.Pmax = get<double>();
    get<double>();  // Umin[0] (written through Pmax's count)
    g.Umin[0] = get<double>();
    g.Umax[0] = get<double>();
    g.Umax[1] = get<double>();
    g.Umin[1] = 0.0;  // not in the file
    g.Pres = get<int32_t>();
    g.Ures[0] = get<int32_t>();
    g.Ures[1] = get<int32_t>();
    g.Pscale = get<int32_t>();
    g.Uscale[0] = get<int32_t>();
    g.Uscale[1] = get<int32_t>();
    for (int i = 0; i < 6; ++i) get<int32_t>();
    const int32_t nfields = get<int32_t>();
    if (!bad && nfields != 1) {
      bad = true;
      why = "only one field (species) is supported";
    }
    skip(sizeof(int32_t) * 6 + sizeof(int64_t) + PARAM_SPARE);
  }
};

struct RestartHead {
  vls_grid_desc grid{};
  vls_solver_desc solver{};
  int64_t every[3] = {0, 0, 0};  // snapshotEvery, restartEvery, statsEvery
  double time = 0;
  int64_t step = 0;
  size_t f_offset = 0;  // byte offset of the FP64 grid
};

bool read_file(const char *path, std::vector<char> &b, std::string &why) {
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    why = std::string("cannot open ") + path;
    return false;
  }
  std::fseek(f, 0, SEEK_END);
  const long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  b.resize(n > 0 ? (size_t)n : 0);
  const size_t got = b.empty() ? 0 : std::fread(b.data(), 1, b.size(), f);
  std::fclose(f);
  if (got != b.size()) {
    why = std::string("cannot read ") + path;
    return false;
  }
  return true;
}

// parses up to the grid data; `in` is left at the grid's first value
bool parse_head(In &in, RestartHead &h) {
  const int32_t e = in.get<int32_t>();
  if (e != 1) {
    in.swap = true;
    int32_t s = e;
    char *p = reinterpret_cast<char *>(&s);
    std::reverse(p, p + 4);
    if (s != 1) {
      in.bad = true;
      in.why = "not a restart file (endianness word)";
      return false;
    }
  }
  in.tag(TAG_SOLVER);
  h.solver.G = in.get<double>();
  h.solver.T0 = in.get<double>();
  h.solver.Tmax = in.get<double>();
  h.solver.dt = in.get<double>();
  const int32_t nsp = in.get<int32_t>();
  for (int k = 0; k < 3; ++k) h.every[k] = in.get<int64_t>();
  h.time = in.get<double>();
  const double dt2 = in.get<double>();
  (void)dt2;  // deltaTime (equal to solverParam.dt in the reference's runs)
  h.step = in.get<int64_t>();
  h.solver.noLinking = in.get<int32_t>();
  if (!in.bad && nsp != 1) {
    in.bad = true;
    in.why = "only one species is supported";
  }
  in.tag(TAG_GH);
  in.get<int32_t>();  // endianness word of the grid handler
  const int32_t pd = in.get<int32_t>(), ud = in.get<int32_t>(), jd = in.get<int32_t>();
  const int64_t dsz = in.get<int64_t>(), ngrids = in.get<int64_t>();
  in.get<int64_t>();  // rank
  if (!in.bad && (pd != 1 || ud != 2 || jd != 1 || dsz != 8 || ngrids != 1)) {
    in.bad = true;
    in.why = "not a single FP64 (r, u, J) grid";
  }
  vls_grid_desc full{};
  in.param(full);
  in.tag(TAG_GB);
  in.param(h.grid);
  h.f_offset = in.o;
  return !in.bad;
}

bool same_grid(const vls_grid_desc &a, const vls_grid_desc &b) {
  return a.Pmin == b.Pmin && a.Pmax == b.Pmax && a.Pres == b.Pres && a.Pscale == b.Pscale &&
         a.Umin[0] == b.Umin[0] && a.Umax[0] == b.Umax[0] && a.Umax[1] == b.Umax[1] &&
         a.Ures[0] == b.Ures[0] && a.Ures[1] == b.Ures[1] && a.Uscale[0] == b.Uscale[0] &&
         a.Uscale[1] == b.Uscale[1];
}
}  // namespace

extern "C" int vls_write_restart(vls_handle *h, const char *path, int64_t snapshot_every,
                                 int64_t restart_every, int64_t stats_every) {
  if (!h || !path) return VLS_EINVAL;
  if (!h->have_f) return fail(h, VLS_ESTATE, "vls_write_restart before the grid was set");
  CK(h, cudaSetDevice(h->solver.device));
  std::vector<double> f(h->cells);
  TRY(take_f(h, f.data()));
  int64_t nch = 0, nel = 0;
  TRY(vls_get_chains(h, &nch, &nel, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr));
  std::vector<double> val((size_t)nel);
  if (nel)
    TRY(vls_get_chains(h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                       val.data()));
  Out o;
  o.b.reserve(h->cells * 8 + 32768);
  o.put((int32_t)1);
  o.tag(TAG_SOLVER);
  o.put(h->solver.G);
  o.put(h->solver.T0);
  o.put(h->solver.Tmax);
  o.put(h->solver.dt);
  o.put((int32_t)1);
  o.put(snapshot_every);
  o.put(restart_every);
  o.put(stats_every);
  o.put(h->time);
  o.put(h->solver.dt);
  o.put((int64_t)h->step);
  o.put((int32_t)(h->solver.noLinking ? 1 : 0));
  o.tag(TAG_GH);
  o.put((int32_t)1);
  o.put((int32_t)1);
  o.put((int32_t)2);
  o.put((int32_t)1);
  o.put((int64_t)sizeof(double));
  o.put((int64_t)1);  // nGrids
  o.put((int64_t)0);  // rank
  o.param(h->grid);
  o.tag(TAG_GB);
  o.param(h->grid);
  {
    const char *p = reinterpret_cast<const char *>(f.data());
    o.b.insert(o.b.end(), p, p + h->cells * sizeof(double));
  }
  o.tag(TAG_G21);
  o.zeros(SPARE);
  o.zeros(SPARE);  // grid handler
  o.zeros(SPARE);  // vlasovSolver
  o.tag(TAG_S21);
  o.put((int32_t)h->solver.kernelType);
  o.put(0.0);  // kernelMass (always 0, vlasovSolver21.hxx:535)
  o.put((int32_t)h->solver.kernelBufferSize);
  o.zeros(SPARE);
  if (h->solver.kernelType == VLS_KERNEL_DELAYED) {
    o.tag(TAG_KERNEL);
    const int64_t nr = h->co.nr, nu = h->co.nu, nj = h->co.nj;
    o.put(nj);
    int64_t c = 0;
    for (int64_t j = 0; j < nj; ++j) {
      int64_t c1 = c;
      while (c1 < nch && h->ch_cell_h[c1] / (nr * nu) == j) ++c1;
      o.put(c1 - c);
      for (; c < c1; ++c) {
        o.put(h->ch_cell_h[c]);
        const int64_t L = h->ch_len_h[c], s0 = h->ch_start_h[c];
        o.put(L);
        for (int64_t e = 0; e < L; ++e) {
          o.put(h->ch_R_h[s0 + e]);
          o.put(h->ch_U_h[s0 + e]);
          o.put((int32_t)1);
          o.put(val[s0 + e]);
        }
      }
    }
  }
  o.tag(TAG_SPLINE);
  o.zeros(SPARE);
  FILE *fo = std::fopen(path, "wb");
  if (!fo) return fail(h, VLS_EIO, std::string("cannot open ") + path + " for writing");
  const size_t w = std::fwrite(o.b.data(), 1, o.b.size(), fo);
  const int cl = std::fclose(fo);
  if (w != o.b.size() || cl != 0) return fail(h, VLS_EIO, std::string("cannot write ") + path);
  return VLS_OK;
}

extern "C" int vls_restart_info(const char *path, vls_grid_desc *grid, vls_solver_desc *solver,
                                int64_t *every, double *time, int64_t *step) {
  std::vector<char> b;
  std::string why;
  if (!path || !read_file(path, b, why)) return fail(nullptr, VLS_EIO, why);
  In in(b);
  RestartHead hd;
  if (!parse_head(in, hd)) return fail(nullptr, VLS_EIO, "restart file: " + in.why);
  // the kernel section follows the grid data and three spares
  in.skip(sizeof(double) * (size_t)(hd.grid.Pres + 1) * (hd.grid.Ures[0] + 1) * hd.grid.Ures[1]);
  in.tag(TAG_G21);
  in.skip(3 * SPARE);
  in.tag(TAG_S21);
  hd.solver.kernelType = in.get<int32_t>();
  in.get<double>();
  hd.solver.kernelBufferSize = in.get<int32_t>();
  if (in.bad) return fail(nullptr, VLS_EIO, "restart file: " + in.why);
  hd.solver.precision = VLS_FP64;
  hd.solver.device = 0;
  if (grid) *grid = hd.grid;
  if (solver) *solver = hd.solver;
  if (every)
    for (int k = 0; k < 3; ++k) every[k] = hd.every[k];
  if (time) *time = hd.time;
  if (step) *step = hd.step;
  return VLS_OK;
}

extern "C" int vls_read_restart(vls_handle *h, const char *path) {
  if (!h || !path) return VLS_EINVAL;
  CK(h, cudaSetDevice(h->solver.device));
  std::vector<char> b;
  std::string why;
  if (!read_file(path, b, why)) return fail(h, VLS_EIO, why);
  In in(b);
  RestartHead hd;
  if (!parse_head(in, hd)) return fail(h, VLS_EIO, "restart file: " + in.why);
  if (!same_grid(hd.grid, h->grid))
    return fail(h, VLS_EINVAL, "restart file: its grid differs from the handle's");
  if (hd.solver.dt != h->solver.dt || hd.solver.G != h->solver.G ||
      (hd.solver.noLinking != 0) != (h->solver.noLinking != 0))
    return fail(h, VLS_EINVAL, "restart file: dt, G or noLinking differ from the handle's");
  std::vector<double> f(h->cells);
  for (size_t i = 0; i < h->cells; ++i) f[i] = in.get<double>();
  in.tag(TAG_G21);
  in.skip(3 * SPARE);
  in.tag(TAG_S21);
  const int32_t kt = in.get<int32_t>();
  in.get<double>();
  const int32_t kbs = in.get<int32_t>();
  in.skip(SPARE);
  if (in.bad) return fail(h, VLS_EIO, "restart file: " + in.why);
  if (kt != h->solver.kernelType || kbs != h->solver.kernelBufferSize)
    return fail(h, VLS_EINVAL, "restart file: kernel type or buffer size differ");
  std::vector<double> val((size_t)h->nel);
  if (kt == VLS_KERNEL_DELAYED) {
    in.tag(TAG_KERNEL);
    const int64_t nr = h->co.nr, nu = h->co.nu;
    const int64_t ns = in.get<int64_t>();
    int64_t c = 0;
    for (int64_t j = 0; j < ns && !in.bad; ++j) {
      const int64_t cnt = in.get<int64_t>();
      for (int64_t k = 0; k < cnt && !in.bad; ++k, ++c) {
        const int64_t key = in.get<int64_t>(), L = in.get<int64_t>();
        if (c >= h->nch || key != h->ch_cell_h[c] || key / (nr * nu) != j ||
            L != h->ch_len_h[c])
          return fail(h, VLS_EINVAL, "restart file: its delayed-kernel chains differ");
        const int64_t s0 = h->ch_start_h[c];
        for (int64_t e = 0; e < L; ++e) {
          in.get<double>();  // R, U: the chain geometry, fixed by the grid and dt
          in.get<double>();
          const int32_t nv = in.get<int32_t>();
          if (nv != 1) return fail(h, VLS_EINVAL, "restart file: chains with several values");
          val[s0 + e] = in.get<double>();
        }
      }
    }
    if (c != h->nch) return fail(h, VLS_EINVAL, "restart file: its delayed-kernel chains differ");
  }
  in.tag(TAG_SPLINE);
  if (in.bad) return fail(h, VLS_EIO, "restart file: " + in.why);
  TRY(put_f(h, f.data()));
  h->ndrift = 0;
  if (h->nel) TRY(vls_set_chain_values(h, val.data(), h->nel));
  h->time = hd.time;
  h->step = hd.step;
  h->moments_valid = false;
  return VLS_OK;
}
