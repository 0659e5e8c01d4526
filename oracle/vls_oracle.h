/*
 * vls_oracle.h -- CPU oracle for the vlasolve spherical (r, v_r, J) split
 * semi-Lagrangian step.  TEST INFRASTRUCTURE ONLY: this library is the
 * checker that the CUDA path is compared against.  Nothing in the product
 * (the vlasolve_b200 package, its C-ABI library or bench.py's timed GPU arm)
 * links or calls it.
 *
 * It restates, in plain C and in the reference's own operation order (FP64,
 * no FMA contraction, one thread), the reference functions below.  Each
 * function in vls_oracle.c cites the reference file:line it follows.
 *
 * Parity pin: the oracle is checked bit-for-bit against outputs of the
 * reference binary itself (built from the reference sources by
 * oracle/build_ref.sh, run with -threads_per_node 1); the golden vectors are
 * committed under tests/golden/ together with the script that made them.
 */
#ifndef VLS_ORACLE_H
#define VLS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* scale types, scale.hxx:18 */
enum { VLO_LINEAR = 0, VLO_LOG = 1, VLO_QUAD = 2 };
/* initial-condition profiles, initGen_all.hxx:132-138 (type strings) */
enum { VLO_UDF = 0, VLO_PLDF = 1, VLO_PLUMMER = 2, VLO_HERNQUIST = 3 };
/* kernel types, vlasovSolver21.hxx:66-68 */
enum { VLO_DELAYED = 0, VLO_REFLECTIVE = 1 };

typedef struct {
  /* grid.* (grid_handler.hxx:224-238): r, then u and J */
  double Pmin, Pmax;
  int Pres, Pscale;
  double Umin[2], Umax[2];
  int Ures[2], Uscale[2];
  /* solver.* (vlasovSolver.hxx:68-78, vlasovSolver21.hxx:537-539) */
  double G, dt;
  int noLinking, kernelType, kernelBufferSize;
  /* init.* */
  int initType;
  double M, R0, alpha, smoothingRadius, gap0, gap1; /* UDF, PLDF */
  double eta, n;                                   /* PLDF */
  double Ra;                                       /* Hernquist */
  int R0_given;                                    /* PLDF: R0 defaults to 1/eta */
} vlo_params;

typedef struct vlo_ctx vlo_ctx;

vlo_ctx *vlo_create(const vlo_params *p);
void vlo_destroy(vlo_ctx *c);

/* dims: N_r, N_u, N_J (cells = N_r*N_u*N_J) */
void vlo_dims(const vlo_ctx *c, long *nr, long *nu, long *nj);
/* coordinate tables: R_Val (N_r), U_Val (N_u), J_Val (N_J), J_V (N_J+1) */
void vlo_coords(const vlo_ctx *c, double *R, double *U, double *J, double *JV);
/* spline scale constants: start/step_inv in rescaled coordinates, dir 0 = r, 1 = u */
void vlo_spline_consts(const vlo_ctx *c, double *start, double *step_inv);
double vlo_kernel_radius(const vlo_ctx *c);

/* f access, layout [j][u][r] */
void vlo_get_f(const vlo_ctx *c, double *out);
void vlo_set_f(vlo_ctx *c, const double *in);

/* footpoint tables (after setup): driftR, driftU, out flag, and the
   decomposed (int, frac) pairs of decomposeDisplacement */
void vlo_get_footpoints(const vlo_ctx *c, double *driftR, double *driftU,
                        uint8_t *out, int32_t *rI, double *rF, int32_t *uI,
                        double *uF);

/* delayed-kernel chains, in build order (slice j, then cell index).
   n_chains / n_elems query; then cell index, start offset and length per
   chain and R, U, val per element (the last element of a chain is its tail) */
void vlo_chain_counts(const vlo_ctx *c, long *n_chains, long *n_elems);
void vlo_get_chains(const vlo_ctx *c, int64_t *cell, int64_t *start,
                    int32_t *len, double *R, double *U, double *val);
void vlo_set_chain_vals(vlo_ctx *c, const double *val);

/* one or more linked (or noLinking) steps */
void vlo_step(vlo_ctx *c, int nsteps);

/* radial moment bins (integrate1D, N_r), enclosed mass Mr (accumulate, N_r)
   and the total, for the current f */
double vlo_moments(const vlo_ctx *c, double *bins, double *Mr);

/* statistics row: M, E, Ek, Ep, S, L1, L2 (vlasovSolver21.hxx:644-690) */
void vlo_stats(const vlo_ctx *c, double *out7);

/* building blocks, exposed for kernel-level tests */
/* 2D natural-BC cubic B-spline prefilter of one slice: f (nu x nr, r fastest)
   -> padded coefficients ((nu+2) x (nr+2)) */
void vlo_prefilter2d(long nr, long nu, double hi_r, double hi_u,
                     const double *f, double *coef);
/* evaluateC (localSpline.hxx:381-398) and evaluateNxPy's sum (:423-441) on
   padded coefficients of row pitch s1 = nr + 2; Ny for the latter is the
   integer part pos2Coord returns */
double vlo_evaluate_c(const double *coef, long s1, int Nx, double x, int Ny, double y);
double vlo_evaluate_nxpy(const double *coef, long s1, int Nx, int Ny, double y);
/* kick of the whole grid with per-r shift (already multiplied by G/R^2 dt) */
void vlo_kick(vlo_ctx *c, const double *shift);
/* drift of the whole grid (tails refreshed, chains rolled) */
void vlo_drift(vlo_ctx *c);

#ifdef __cplusplus
}
#endif
#endif
