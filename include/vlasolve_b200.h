/*
 * vlasolve_b200.h -- C-ABI of the B200 (sm_100a) split semi-Lagrangian step
 * for the spherically symmetric (r, v_r, J) Vlasov-Poisson system.
 *
 * One handle owns one phase-space grid f(r, u=v_r, J) resident in the HBM of
 * one GPU, the time-invariant footpoint tables of the drift, the delayed-kernel
 * ring buffers and all scratch.  Every entry point returns an int status
 * (VLS_OK = 0); a failed call leaves a message in vls_last_error().  No entry
 * point aborts the process.  Calls on one handle are not re-entrant; distinct
 * handles may be driven from distinct host threads.
 *
 * Layout of every host-side grid array: [j][u][r] with r fastest
 * (slice21Iterator.hxx:63 of the reference), FP64.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the reference project's src/).  The reference has no C-ABI: the boundary
 * is its C++ class surface (vlasovSolver21_spline / localSpline<2>), which the
 * C++ adapter in include/vlasolve_b200.hpp mirrors on top of these calls.
 */
#ifndef VLASOLVE_B200_H
#define VLASOLVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (the reference exits instead, e.g. localSpline.hxx:320-324,
   typeSelect.hxx:29-38, vlasovSolver21.hxx:296-298) */
enum {
  VLS_OK = 0,
  VLS_EINVAL = 1, /* invalid argument or configuration */
  VLS_ECUDA = 2,  /* CUDA runtime error, or the CUDA path is unavailable */
  VLS_ENAN = 3,   /* non-finite value detected: in a grid loaded from the
                     host (vls_set_f, vls_read_ndfield, vls_read_restart; the
                     grid is loaded all the same), in chain values
                     (vls_set_chain_values), in an adjoint seed, or by a
                     step's enclosed-mass scan (reported by the next call that
                     waits for the device, e.g. vls_sync) */
  VLS_EIO = 4,    /* file format / I/O error */
  VLS_ENOMEM = 5, /* device or host allocation failed */
  VLS_ESTATE = 6  /* call out of order (e.g. step before initialisation) */
};

/* scale::scaleTypeV, scale.hxx:17-19 */
enum { VLS_SCALE_LINEAR = 0, VLS_SCALE_LOG = 1, VLS_SCALE_QUADRATIC = 2 };
/* vlasovSolver21::kernelTypeV, vlasovSolver21.hxx:66-68 */
enum { VLS_KERNEL_DELAYED = 0, VLS_KERNEL_REFLECTIVE = 1 };
/* initGenAll registry, initGen_all.hxx:132-138 ("UDF", "PLDF", "Plummer",
   "Hernquist") */
enum { VLS_INIT_UDF = 0, VLS_INIT_PLDF = 1, VLS_INIT_PLUMMER = 2,
       VLS_INIT_HERNQUIST = 3 };
/* arithmetic/storage of the step.  FP64: every value FP64.  FP32_BULK: f,
   spline coefficients and the gathers in FP32; prefilter recursions, footpoint
   indexing, moments, enclosed-mass scan and statistics in FP64.  FP32_ALL:
   as FP32_BULK but the prefilter recursions also run in FP32 (indexing,
   moments, scan and statistics stay FP64).  In both FP32 modes the drift
   footpoint fractions are stored with 21 bits (rounded). */
enum { VLS_FP64 = 0, VLS_FP32_BULK = 1, VLS_FP32_ALL = 2 };

/* gridBase::paramT, grid_base.hxx:58-82, i.e. the grid.* options
   (grid_handler.hxx:224-238): r is index P, u and J are U[0] and U[1].
   N_r = Pres+1 and N_u = Ures[0]+1 vertices, N_J = Ures[1] cells. */
typedef struct {
  double Pmin, Pmax;
  int32_t Pres, Pscale;
  double Umin[2], Umax[2];
  int32_t Ures[2], Uscale[2];
} vls_grid_desc;

/* solverParam (solverParam.hxx:6-14) plus the solver.* options of
   vlasovSolver21 (vlasovSolver21.hxx:537-539) and vlasovSolver.hxx:78 */
typedef struct {
  double G, T0, Tmax, dt;
  int32_t noLinking;        /* solver.noLinking */
  int32_t kernelType;       /* solver.kernelType: VLS_KERNEL_* */
  int32_t kernelBufferSize; /* solver.kernelBufferSize */
  int32_t precision;        /* VLS_FP64 or VLS_FP32_BULK */
  int32_t device;           /* CUDA device ordinal */
} vls_solver_desc;

/* init.* options of the four profiles (initGen_UniformDensitySphere.hxx:49-62,
   initGen_PowerLawDensitySphere.hxx:50-61, initGen_Plummer.hxx:45-48,
   initGen_Hernquist.hxx:41-48).  R0_given = 0 lets PLDF take R0 = 1/eta. */
typedef struct {
  int32_t type; /* VLS_INIT_* */
  double M, R0, alpha, smoothingRadius, gap[2], eta, n, Ra;
  int32_t R0_given;
} vls_init_desc;

/* statistics row of vlasovSolver21::statistics, vlasovSolver21.hxx:644-690 */
typedef struct {
  double time;
  int64_t step;
  double Mass, E, Ek, Ep, S, L1, L2;
} vls_stats_out;

typedef struct vls_handle vls_handle;

/* Build number of this library and whether a usable sm_100 device exists.
   Replaces nothing in the reference (its binary has no device). */
int vls_version(int32_t *major, int32_t *minor);
int vls_device_ok(int32_t device);

/* vlasovSolver21::setup + vlasovSolver21_spline::setup
   (vlasovSolver21.hxx:411-446, :533-548; vlasovSolver21_spline.hxx:296-374):
   coordinate tables, spline constants, kernel radius, host-tabulated drift
   footpoints (generateDisplacement :102-204, decomposeDisplacement
   vlasovSolver21_spline.hxx:76-117) and the delayed-kernel chain layout
   (setupBoundaryConditions vlasovSolver21.hxx:265-326).  Allocates every
   device buffer of the handle. */
int vls_create(const vls_grid_desc *grid, const vls_solver_desc *solver,
               vls_handle **out);
/* Kernel layouts of a handle (no counterpart in the reference, whose step has
   one CPU code path).  A zero-initialised descriptor, or NULL, selects the
   defaults, which vls_create uses; the other values serve tests and
   measurements and never change the arithmetic beyond FP rounding order.
     prefilter         VLS_PREFILTER_AUTO: register-resident chunked solves
                       where a line fits them, else shared-memory segments;
                       VLS_PREFILTER_SEGMENT: segments for every line.
     drift             VLS_DRIFT_AUTO: FP32 storage stages each block's whole
                       coefficient strip (two blocks per SM where they fit,
                       else one block of 32 warps), FP64 storage and strips
                       too tall for one block take staged 64 x 40 windows;
                       VLS_DRIFT_WINDOW / _STRIP2 / _STRIP1 ask for one of
                       those (a strip that does not fit falls back to windows).
     slices_per_batch  J slices per batch of the prefilter and drift scratch
                       (0: all slices in one batch); the G and C scratch
                       holds streams x slices_per_batch slices.
     streams           batches run on this many streams, each with its own
                       scratch slot (0 or 1: one stream).
     drift_wait_spins  polls of each bounded wait of the drift for its staged
                       coefficients (0: the default, about 2^20; < 0: none,
                       every such wait gives up at once, which sends every
                       cell to the gather from global memory and makes
                       vls_sync report VLS_ECUDA: a test of the timeout path).
   vls_get_layout reports what a handle uses: prefilter REGISTER or SEGMENT
   and the chunk length of each direction (0 for segments), the drift kind,
   the batch size and stream count, and the wait limit. */
enum { VLS_PREFILTER_AUTO = 0, VLS_PREFILTER_REGISTER = 1, VLS_PREFILTER_SEGMENT = 2 };
enum { VLS_DRIFT_AUTO = 0, VLS_DRIFT_WINDOW = 1, VLS_DRIFT_STRIP2 = 2, VLS_DRIFT_STRIP1 = 3 };
typedef struct {
  int32_t prefilter;
  int32_t drift;
  int32_t slices_per_batch;
  int32_t streams;
  int32_t drift_wait_spins;
  int32_t u_chunk_rows; /* reported by vls_get_layout; ignored on input */
  int32_t r_chunk_rows; /* reported by vls_get_layout; ignored on input */
} vls_layout_desc;
int vls_create_layout(const vls_grid_desc *grid, const vls_solver_desc *solver,
                      const vls_layout_desc *layout, vls_handle **out);
int vls_get_layout(const vls_handle *h, vls_layout_desc *used);
/* ~vlasovSolver21_spline: frees the handle and all its device memory */
int vls_destroy(vls_handle *h);
/* message of the last failed call on h (or of the last vls_create failure
   when h is NULL) */
const char *vls_last_error(const vls_handle *h);

/* grid_21.hxx:150-158 getValCoord21_* sizes */
int vls_dims(const vls_handle *h, int64_t *nr, int64_t *nu, int64_t *nj);
/* grid_21.hxx:150-158: R_Val (N_r), U_Val (N_u), J_Val (N_J), J_V (N_J+1) */
int vls_coords(const vls_handle *h, double *R, double *U, double *J,
               double *JV);
/* initGen_*::generate + vlasovSolver21::renormalize(init->getMass(0), 0)
   (vlasovSolver.hxx:83-96, vlasovSolver21.hxx:468-524): samples the profile
   at every node, fills the chain values with init->valueAt and rescales both
   so that the quadrature mass equals M.  Returns the pre-normalisation mass
   in *mass_before (may be NULL). */
int vls_init_profile(vls_handle *h, const vls_init_desc *init,
                     double *mass_before);

/* grid data access (gridBase::getDataPtr): FP64 host array of n = N_r*N_u*N_J
   values in [j][u][r] order */
int vls_set_f(vls_handle *h, const double *host, size_t n);
int vls_get_f(vls_handle *h, double *host, size_t n);

/* footpoint tables as decomposeDisplacement produces them
   (vlasovSolver21_spline.hxx:69-72, :88-100) and disp_driftOut
   (vlasovSolver21.hxx:94, :140-143); each array has N_r*N_u*N_J entries.
   Any pointer may be NULL.  vls_set_footpoints replaces the tables (driftR is
   only used for the kernel-radius test). */
int vls_get_footpoints(const vls_handle *h, int32_t *rI, double *rF,
                       int32_t *uI, double *uF, uint8_t *out, double *driftR);
int vls_set_footpoints(vls_handle *h, const int32_t *rI, const double *rF,
                       const int32_t *uI, const double *uF, const uint8_t *out,
                       const double *driftR);

/* delayed-kernel chains (sphericalKernel.hxx:21-24, cellChain.hxx:85-86) in
   compressed-row form, in build order: per chain its cell index, first element
   and length; per element R, U and value, logical front first (the last
   element of a chain is its tail).  *n_chains / *n_elems report sizes when
   the arrays are NULL. */
int vls_get_chains(const vls_handle *h, int64_t *n_chains, int64_t *n_elems,
                   int64_t *cell, int64_t *start, int32_t *len, double *R,
                   double *U, double *val);
int vls_set_chain_values(vls_handle *h, const double *val, int64_t n_elems);

/* vlasovSolver::run body / vlasovSolver21_spline::makeOneStep
   (vlasovSolver.hxx:158-180, vlasovSolver21_spline.hxx:680-801): nsteps
   linked (or noLinking) steps on the device; time += dt and step += 1 per
   step.  Asynchronous with respect to the host except for errors of the
   launch itself; the handle's stream orders all later calls. */
int vls_step(vls_handle *h, int32_t nsteps);
/* wait for all work on the handle's stream; reports device-side errors */
int vls_sync(vls_handle *h);
/* number of kernels this handle has launched so far (diagnostic; the
   reference has no device) */
int vls_kernel_launches(const vls_handle *h, int64_t *n);
/* the cudaStream_t every launch of this handle goes to (for CUDA-event
   timing by the caller); the reference has no device */
int vls_stream(const vls_handle *h, void **stream);
/* per-kernel device timing: with profiling on, every launch is bracketed by
   CUDA events on the handle's stream.  vls_profile_read synchronises, returns
   the summed milliseconds and launch counts of each kernel kind
   (VLS_K_* below, nk entries) and clears the record.  Diagnostic only. */
enum { VLS_K_UCOL_KICK = 0, VLS_K_UCOL = 1, VLS_K_PRER = 2, VLS_K_TAILS = 3,
       VLS_K_DRIFT = 4, VLS_K_SCAN = 5, VLS_K_MOMENT = 6, VLS_K_STATS = 7,
       VLS_K_CONVERT = 8,
       /* adjoint step: drift transpose, chain fronts and tails, r-solve and
          u-solves + kick transposed, the step's shift (moment + scan), the
          moment and shift transposed */
       VLS_K_ADJ_DRIFT = 9, VLS_K_ADJ_TAILS = 10, VLS_K_ADJ_PRER = 11,
       VLS_K_ADJ_UCOL = 12, VLS_K_ADJ_SHIFT = 13, VLS_K_ADJ_MOMENT = 14,
       VLS_K_COUNT = 15 };
int vls_set_profiling(vls_handle *h, int32_t on);
int vls_profile_read(vls_handle *h, double *ms, int64_t *count, int32_t nk);

/* quadrature21::integrate1D_acc on the current f (vlasovSolver21_spline.hxx:736,
   quadrature21.hxx:43-52, grid_handler.hxx:387-407): radial bins (N_r),
   enclosed mass strictly inside R_r (N_r) and the total mass.  Any pointer may
   be NULL. */
int vls_moments(vls_handle *h, double *bins, double *Mr, double *mtot);
/* mass of the most recent step's moment (the value the reference prints as
   " (M=...)" each step, vlasovSolver21_spline.hxx:744) */
int vls_last_mass(vls_handle *h, double *mtot);
/* the same read without waiting: the copy of the most recent step's mass
   into *mtot is queued on the handle's stream, and *mtot holds it once a
   synchronising call (vls_sync, vls_get_f, ...) has returned.  With mtot in
   page-locked host memory the call returns at once, so a loop that reads
   every step's mass does not stall the device between steps. */
int vls_last_mass_async(vls_handle *h, double *mtot);

/* vlasovSolver21::statistics (vlasovSolver21.hxx:627-690) on the current f:
   FP64 device reductions with compensated summation. */
int vls_stats(vls_handle *h, vls_stats_out *out);

/* time / step counters of vlasovSolver (vlasovSolver.hxx:202-204) */
int vls_get_time(const vls_handle *h, double *time, int64_t *step);
int vls_set_time(vls_handle *h, double time, int64_t step);

/* NDfield snapshot of f (vlasovSolver21::snapshot / NDfieldFromData,
   vlasovSolver21.hxx:585-598, :717-773; Save_NDfield NDfield.hxx:308-363) */
int vls_write_ndfield(vls_handle *h, const char *path);
/* reads the payload of an NDfield written by the reference or by
   vls_write_ndfield into f (dims and datatype are checked) */
int vls_read_ndfield(vls_handle *h, const char *path);

/* .vls restart files in the reference's layout (vlasovSolver::write and the
   sections it calls: vlasovSolver.hxx:272-287, grid_handler.hxx:325-347,
   grid_base.hxx:123-153 and :492-497, grid_21.hxx:85-91,
   vlasovSolver21.hxx:568-583, sphericalKernel.hxx:88-106,
   vlasovSolver21_spline.hxx:437-444), so that the reference's -reload reads
   ours and vls_read_restart reads the reference's.  The grid is written in
   FP64 whatever the precision.  snapshot_every, restart_every and
   stats_every are the solverParam fields the file carries.
   vls_restart_info reads a file's grid and solver parameters (so a caller can
   create a matching handle first; the J minimum is not stored in the file
   and is returned as 0), the three intervals, the time and the step count.
   vls_read_restart loads the grid, the chain values, the time and the step
   count into a handle whose grid, dt, G, noLinking, kernel type and kernel
   buffer size match the file's. */
int vls_write_restart(vls_handle *h, const char *path, int64_t snapshot_every,
                      int64_t restart_every, int64_t stats_every);
int vls_restart_info(const char *path, vls_grid_desc *grid, vls_solver_desc *solver,
                     int64_t *every, double *time, int64_t *step);
int vls_read_restart(vls_handle *h, const char *path);

/* Adjoint of the linked step (the reference has no derivative code).
   vls_adjoint_forward runs nsteps steps from the current state (as vls_step)
   and keeps a device copy of the state every checkpoint_every steps.
   vls_adjoint_backward then takes dL/dbins of a loss L of the final radial
   bins (nbins = N_r, the bins vls_moments returns for the final grid) and
   returns dL/df of the initial grid (df0, N_r*N_u*N_J doubles, [j][u][r]) and
   of the initial delayed-kernel chain values (dchain0, n_elems doubles in
   vls_get_chains order; may be NULL).  The backward pass recomputes each
   segment of checkpoint_every steps from its checkpoint and applies the
   transposed step: drift and chain-tail gathers as scatter-adds, the
   natural-BC prefilter transposed, the kick's gather transposed plus its
   derivative with respect to the shift, and the transposed enclosed-mass
   scan and moment.  The derivative is of the step as computed in the
   handle's precision, evaluated in FP64.  Afterwards the handle holds the
   final state again; vls_adjoint_backward may be called again with another
   seed.  Linked step only (noLinking = 0). */
int vls_adjoint_forward(vls_handle *h, int32_t nsteps, int32_t checkpoint_every);
int vls_adjoint_backward(vls_handle *h, const double *dbins, int64_t nbins, double *df0,
                         size_t ncells, double *dchain0, int64_t nelems);

/* Second level of checkpoints for the adjoint (no counterpart in the
   reference).  The backward pass recomputes a segment of checkpoint_every
   steps and keeps each of its states on the device; when those states do not
   fit (a 1025 x 1025 x 512 FP32 grid is 2.15 GB per state, 215 GB for a
   segment of 100 steps), it first runs through the segment keeping a
   checkpoint every inner_every steps and then recomputes and transposes one
   sub-segment of inner_every steps at a time: device memory of inner_every
   states plus ceil(checkpoint_every / inner_every) checkpoints, at the cost
   of one more forward run.  inner_every = 0 (the default) chooses it at each
   backward pass from the free device memory: one level when the segment's
   states fit, else the spacing that stores the fewest states (about
   sqrt(checkpoint_every): the extra forward run costs the same for every
   spacing).  vls_adjoint_inner_used
   returns the spacing the last backward pass used (0: one level).  The
   gradient does not depend on the choice: the recomputed states are the
   same. */
int vls_adjoint_set_inner(vls_handle *h, int32_t inner_every);
/* Device memory the handle holds, in bytes: grid, coefficients, footpoint
   tables, chains, moments and, once used, the adjoint's checkpoints, stash
   and FP64 arrays (no counterpart in the reference).  A handle frees its
   memory only in vls_destroy, so this is also its peak. */
int vls_device_bytes(vls_handle *h, size_t *bytes);
int vls_adjoint_inner_used(vls_handle *h, int32_t *inner_every);
/* For derivatives with respect to init.* parameters by central differences
   (no counterpart in the reference): with the dL/df0 and dL/dc0 of the last
   vls_adjoint_backward, *dgrid = <dL/df0, f(plus) - f(minus)> and *dchain =
   <dL/dc0, c(plus) - c(minus)>, f and c the initial grid and chain values
   vls_init_profile makes for the two parameter sets (renormalised to their
   M).  The grids are evaluated on the device with its FP64 math functions,
   so they differ from vls_init_profile's host grid in the last bits; the
   handle's state is not touched.  VLS_ESTATE before a backward pass. */
int vls_adjoint_init_dot(vls_handle *h, const vls_init_desc *plus,
                         const vls_init_desc *minus, double *dgrid, double *dchain);

/* ---------------------------------------------------------------------------
   Spline level.  localSpline<2, double> (localSpline.hxx:60-503) is the
   reference's 2D cubic B-spline: init(initT), assign(data), build(),
   evaluateC, evaluateNxPy, evaluate, pos2Coord.  A vls_spline2d is a batch of
   nslices such splines on one GPU, built by the step's prefilter kernels and
   evaluated at batches of points; positions are decomposed into (index,
   fraction) on the host in FP64 (pos2Coord), so indices are the reference's
   bit for bit.  Only the natural boundary condition (the one the step's
   splines use) is built; other boundary types return VLS_EINVAL.  Points
   whose indices lie outside [0, dim) return VLS_EINVAL (the reference reads
   outside its buffer there). */
/* localSpline::boundaryTypeV, localSpline.hxx:34 */
enum { VLS_BC_PERIODIC = 0, VLS_BC_FLAT = 1, VLS_BC_NATURAL = 2, VLS_BC_SUPRA_NATURAL = 3,
       VLS_BC_NOT_A_KNOT = 4, VLS_BC_LOCAL = 5 };
/* localSpline::initT (localSpline.hxx:39-46), dimension 0 fastest in the data;
   vlType: 1 = values at vertices (VERTEX), 0 = at cell centres (CELL);
   precision VLS_FP64 or VLS_FP32_BULK (FP32 storage, FP64 solves) */
typedef struct {
  double start[2], stop[2];
  int32_t N[2];
  int32_t scaleType[2];
  int32_t vlType[2];
  int32_t bCond[2][2];
  int32_t precision;
  int32_t device;
} vls_spline2d_desc;
typedef struct vls_spline2d vls_spline2d;
/* localSpline::init: value counts dim0, dim1 from genScale, start / step_inv
   in rescaled coordinates (vls_spline2d_scale), device buffers of nslices */
int vls_spline2d_create(const vls_spline2d_desc *desc, int64_t nslices, vls_spline2d **out);
int vls_spline2d_destroy(vls_spline2d *s);
int vls_spline2d_dims(const vls_spline2d *s, int32_t *dim0, int32_t *dim1, int64_t *nslices);
int vls_spline2d_scale(const vls_spline2d *s, double *start, double *step_inv);
/* localSpline::assign (localSpline.hxx:205-246): host FP64 values
   [slice][dim1][dim0] of every slice */
int vls_spline2d_assign(vls_spline2d *s, const double *data, int64_t nslices);
/* localSpline::build / create_2D (localSpline.hxx:248-260, :1238-1258) */
int vls_spline2d_build(vls_spline2d *s);
/* the padded coefficients of one slice as localSpline's buffer holds them
   (localSpline.hxx:222): (dim0+2) x (dim1+2) FP64, dim0 fastest */
int vls_spline2d_coefficients(vls_spline2d *s, int64_t slice, double *coef);
/* localSpline::pos2Coord (localSpline.hxx:352-358) of n positions along dir */
int vls_spline2d_pos2coord(const vls_spline2d *s, int32_t dir, int64_t n, const double *p,
                           int32_t *I, double *F);
/* localSpline::evaluateC(int, double, int, double) (localSpline.hxx:381-398),
   evaluateNxPy (:423-441) and evaluate(double, double) (:477-488) at n points;
   slice (n entries) may be NULL for slice 0 */
int vls_spline2d_evaluate_c(vls_spline2d *s, int64_t n, const int64_t *slice, const int32_t *Nx,
                            const double *x, const int32_t *Ny, const double *y, double *v);
int vls_spline2d_evaluate_nxpy(vls_spline2d *s, int64_t n, const int64_t *slice,
                               const int32_t *Nx, const double *yy, double *v);
int vls_spline2d_evaluate(vls_spline2d *s, int64_t n, const int64_t *slice, const double *xx,
                          const double *yy, double *v);
/* message of the last failed call on s (or of the last create failure when
   s is NULL, per host thread) */
const char *vls_spline2d_last_error(const vls_spline2d *s);

/* interpolSpline<double> (interpol_spline.hxx:9-189), the reference's
   einspline-backed interface (third-party einspline, not vendored, compiled
   out by the reference's build).  Boundary codes are einspline's bc_code
   values the reference passes through (:23-27); natural ends (NATURAL, or
   DERIV2 with value 0) are built, others return VLS_EINVAL.  Grids in
   rescaled coordinates, the last node nudged by 1e-10 of a cell as createInit
   does. */
enum { VLS_EBC_PERIODIC = 0, VLS_EBC_DERIV1 = 1, VLS_EBC_DERIV2 = 2, VLS_EBC_FLAT = 3,
       VLS_EBC_NATURAL = 4, VLS_EBC_ANTIPERIODIC = 5 };
/* interpolSpline::initT (:33-39) */
typedef struct {
  double xstart, xend, ystart, yend;
  int32_t nx, ny;
  int32_t xbc[2], ybc[2];
  double xbcv[2], ybcv[2];
  int32_t xscaleType, yscaleType;
  int32_t rescaleNeeded, useLog;
} vls_interp_init;
typedef struct vls_interp vls_interp;
/* interpolSpline::createInit (:49-91) */
int vls_interp_create_init(double xstart, double xstop, int32_t Nx, double ystart,
                           double ystop, int32_t Ny, int32_t xbctL, int32_t xbctR,
                           int32_t ybctL, int32_t ybctR, int32_t xscaleType,
                           int32_t yscaleType, int32_t vltype, int32_t useLog, double xbcvL,
                           double xbcvR, double ybcvL, double ybcvR, vls_interp_init *out);
/* interpolSpline::create (:93-110): data ny x nx, x fastest */
int vls_interp_create(const vls_interp_init *ini, const double *data, int32_t device,
                      vls_interp **out);
/* interpolSpline::evaluate (:112-183) at n points: v; g (2 per point: dv/dy,
   dv/dx) and h (4 per point: yy, yx, xy, xx) when not NULL, in rescaled
   coordinates; points are clamped to the grid */
int vls_interp_evaluate(vls_interp *s, int64_t n, const double *x, const double *y, double *v,
                        double *g, double *h);
/* interpolSpline::destroy (:185-189) */
int vls_interp_destroy(vls_interp *s);
const char *vls_interp_last_error(const vls_interp *s);

/* Radial moment of a grid that already lives in device memory, without any
   allocation (no counterpart in the reference, whose grid is host memory).
   For callers that own all device memory and must not let a library call
   cudaMalloc (an application with its own memory pool or a fixed budget
   reserved at start-up): the grid f_dev ([j][u][r], double for VLS_FP64,
   float otherwise) and the outputs bins_dev, Mr_dev (N_r doubles each) and
   mtot_dev (one double) are the caller's device buffers; the coordinates R
   (N_r), U (N_u), J (N_J), JV (N_J+1) are host arrays, as vls_coords returns
   them.  Results are those of vls_moments for the same grid.  Work is queued
   on `stream` (a cudaStream_t, NULL for the legacy default stream) of
   `device`.  Working space is a fixed 512 KiB device array inside the
   library: grids above 2048 r vertices, 2048 u vertices or 2048 J cells are
   rejected with VLS_EINVAL.  That array is shared by every call, so calls that
   overlap on the GPU race and must be serialised by the caller; the first
   call on a device looks up the array's device address with that device
   current, so it should come before any stream capture on that device (after
   cudaDeviceReset the next call looks it up again).  Every call copies R, U,
   J and JV from host memory with cudaMemcpyAsync on `stream`.  Errors are
   reported by vls_noalloc_last_error(), which returns the message of the
   calling host thread's last failed call. */
int vls_radial_mass_noalloc(const void *f_dev, int32_t precision, int64_t nr,
                            int64_t nu, int64_t nj, const double *R,
                            const double *U, const double *J, const double *JV,
                            double *bins_dev, double *Mr_dev, double *mtot_dev,
                            void *stream, int32_t device);
const char *vls_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
