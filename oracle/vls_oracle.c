/*
 * vls_oracle.c -- CPU oracle (FP64, one thread, reference operation order)
 * for the vlasolve spherical split semi-Lagrangian step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is
 * compared against; the product never links it.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the reference project's src/).  Compile with -ffp-contract=off so no
 * FMA is formed: the reference is built for x86-64 without FMA, and the
 * oracle must round every product and sum exactly as it does.
 */
#include "vls_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct vlo_ctx {
  vlo_params p;
  long nr, nu, nj;
  double *R, *U, *J;  /* value coordinates R_Val, U_Val, J_Val */
  double *JV;         /* J vertices J_V (N_J+1) */
  /* spline constants, localSpline.hxx:60-93 */
  double sstart[2], sstep_inv[2];
  double kernelRadius;
  long halted_cell; /* first cell where the reference would halt, or -1 */
  /* init-profile constants */
  double rho0, sig0, C0, C1, C2, sigR2, sigO2, Vg;
  /* state */
  double *f;
  double *coef; /* one padded slice ((nu+2) x (nr+2)) */
  double *tmpA; /* Thomas work array, 4*(max(nr,nu)+2) */
  /* footpoints */
  double *driftR, *driftU;
  uint8_t *driftOut;
  int32_t *rI, *uI;
  double *rF, *uF;
  /* chains */
  long nch, nel, cap_ch, cap_el;
  int64_t *ch_cell, *ch_start;
  int32_t *ch_len;
  int64_t *cell2ch; /* -1 if the cell has no chain */
  double *el_R, *el_U, *el_val;
};

/* ---------------------------------------------------------------- scales */

/* scale::genScale, scale.hxx:114-151 (vertex=1 -> VERTEX, 0 -> CELL).
   Returns a malloc'd array of N+1 (vertex) or N (cell) values. */
static double *gen_scale(double start, double stop, long N, int sct,
                         int vertex, long *size_out) {
  double *s = (double *)malloc(sizeof(double) * (N + 1));
  long i;
  if (sct == VLO_LINEAR) {
    double dx = (stop - start) / (N);
    for (i = 0; i < N + 1; i++) s[i] = start + dx * (double)i;
  } else if (sct == VLO_LOG) {
    double sg = (start < 0) ? -1 : 1;
    long n2;
    double *l = gen_scale(log(fabs(start)), log(fabs(stop)), N, VLO_LINEAR, 1,
                          &n2);
    for (i = 0; i < N + 1; i++) s[i] = sg * exp(l[i]);
    free(l);
  } else {
    int pp = sct;
    long n2;
    double *l = gen_scale(pow(start, 1. / pp), pow(stop, 1. / pp), N,
                          VLO_LINEAR, 1, &n2);
    for (i = 0; i < N + 1; i++) s[i] = pow(l[i], (double)pp);
    free(l);
  }
  if (!vertex) {
    for (i = 0; i < N; i++) s[i] = (s[i] + s[i + 1]) * 0.5;
    *size_out = N;
  } else {
    s[0] = start;
    s[N] = stop;
    *size_out = N + 1;
  }
  return s;
}

/* scale::rescale, scale.hxx:175-189 */
static double rescale(double x, int sct) {
  if (sct == VLO_LOG) return log(x);
  if (sct == VLO_LINEAR) return x;
  return pow(x, 1. / sct);
}

/* ------------------------------------------------------- initial profiles */

/* UniformDensitySphere::setupParameters, initGen_UniformDensitySphere.hxx:65-74
   PowerLawDensitySphere::setupParameters, initGen_PowerLawDensitySphere.hxx:63-82
   Hernquist::setupParameters, initGen_Hernquist.hxx:48 */
static void setup_profile(vlo_ctx *c) {
  const vlo_params *p = &c->p;
  if (p->initType == VLO_UDF) {
    c->rho0 = (3 * p->M) / (4 * M_PI * pow(p->R0, 3));
    c->sig0 = sqrt((p->alpha) / (5 * p->R0));
    c->C1 = c->rho0 * pow(2 * M_PI * c->sig0 * c->sig0, -1.5);
    c->C2 = 2 * c->sig0 * c->sig0;
  } else if (p->initType == VLO_PLDF) {
    double R0 = p->R0_given ? p->R0 : 1. / p->eta;
    c->rho0 = ((3.0 - p->n) * p->M) / (4 * M_PI * pow(R0, 3.0 - p->n));
    c->sigO2 = (3.0 - p->n) / (5.0 - 2 * p->n) * (p->M * p->eta) /
               (R0 * (p->alpha * 0.5 + 1));
    c->sigR2 = c->sigO2 * 0.5 * p->alpha;
    c->C0 = c->rho0 / (sqrt(2 * c->sigR2 * M_PI * M_PI * M_PI) * c->sigO2);
    c->C1 = 1.0 / (2 * c->sigR2);
    c->C2 = 1.0 / (c->sigO2);
  } else if (p->initType == VLO_HERNQUIST) {
    c->Vg = sqrt((p->G * p->M) / (p->R0));
  }
}

static double pldf_R0(const vlo_ctx *c) {
  return c->p.R0_given ? c->p.R0 : 1. / c->p.eta;
}

/* computeF / valueAt of each profile:
   UDF initGen_UniformDensitySphere.hxx:158-173,
   PLDF initGen_PowerLawDensitySphere.hxx:181-189,
   Plummer initGen_Plummer.hxx:89-92,126-137,
   Hernquist initGen_Hernquist.hxx:97-99,133-161 */
static double profile_value(const vlo_ctx *c, double r, double u, double j) {
  const vlo_params *p = &c->p;
  switch (p->initType) {
    case VLO_UDF: {
      double sm = 0.5 * (1. + erf((p->R0 - r) / p->smoothingRadius));
      double res = sm * c->C1 * exp(-(u * u + (j * j) / (r * r)) / c->C2);
      if (p->gap1 > 0) {
        double sm0 = 0.5 * (1. + erf((p->gap0 - r) / 0.15));
        double sm1 = 0.5 * (1. + erf(-(p->gap1 - r) / 0.15));
        res *= (sm0 + sm1);
      }
      if (res < 1.E-200) res = 1.E-200;
      return res;
    }
    case VLO_PLDF: {
      double sm = 0.5 * (1. + erf((pldf_R0(c) - r) / p->smoothingRadius));
      double res = sm * c->C0 *
                   exp(-u * u * c->C1 - ((j * j) / (r * r)) * c->C2) *
                   pow(r, -p->n);
      if (res < 1.E-200) res = 1.E-200;
      return res;
    }
    case VLO_PLUMMER: {
      double phi = -(p->G * p->M) / sqrt(r * r + p->R0 * p->R0);
      double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      if (eps >= 0) return 0;
      return pow(-2. * eps, 3.5) * (3. / (M_PI * M_PI * M_PI * 7.));
    }
    case VLO_HERNQUIST: {
      double phi = -(p->G * p->M) / (p->R0 + r);
      double eps = phi + (u * u + (j * j) / (r * r)) * 0.5;
      double q, q2, A1, A2, result;
      if (p->Ra > 0) eps = eps + (j * j) / (2 * p->Ra * p->Ra);
      if (eps >= 0) return 0;
      q = sqrt(-(p->R0) / (p->G * p->M) * eps);
      q2 = q * q;
      A1 = (p->M) / (8. * sqrt(2.) * pow(M_PI * p->R0 * c->Vg, 3.)) *
           pow(1. - q2, -2.5);
      A2 = 3 * asin(q) + q * sqrt(1. - q2) * (1. - 2 * q2) *
                             (8 * q2 * q2 - 8 * q2 - 3);
      result = A1 * A2;
      if (p->Ra > 0) {
        A1 = (p->M) / (sqrt(2) * pow(M_PI * p->R0 * c->Vg, 3)) *
             pow(p->R0 / p->Ra, 2);
        A2 = q * (1. - 2 * q2);
        result += A1 * A2;
      }
      return result;
    }
  }
  return 0;
}

/* ------------------------------------------------------------- footpoints */

/* vlasovSolver21::advanceParticleDrift, vlasovSolver21.hxx:328-408 */
static void advance_particle_drift(double R, double U, double J, double dt,
                                   double R0, double *outR, double *outU,
                                   int *halted) {
  double H0, newU, newR, tlim, tR0, sgn, deltaT;
  if (halted) *halted = 0;
  H0 = 0.5 * (U * U + (J * J) / (R * R));
  sgn = (U <= 0) ? -1 : 1;
  deltaT = dt;
  newR = R;
  newU = U;
  if (sgn < 0) {
    tlim = 10 * dt;
    tR0 = 10 * dt;
  } else {
    tlim = sqrt(2 * R * R * H0 - J * J) / (2 * H0);
    if (R0 > 0) {
      double A, B, C, D;
      A = 2 * H0;
      B = -2 * sgn * sqrt(2 * R * R * H0 - J * J);
      C = (R * R - R0 * R0);
      D = B * B - 4 * A * C;
      if (D < 0)
        tR0 = 10 * dt;
      else
        tR0 = (-B - sqrt(D)) / (2 * A);
      if (tR0 < 0) {
        tR0 = (-B + sqrt(D)) / (2 * A);
        if (tR0 < 0) tR0 = 10 * dt;
      }
    } else
      tR0 = 10 * dt;
  }
  if ((tR0 < deltaT) && (tR0 < tlim)) {
    newR = sqrt(pow(fabs(newR * newU) - 2 * sgn * H0 * tR0, 2) + J * J) *
           pow(2 * H0, -0.5);
    newU = (2 * H0 - (J * J) / (newR * newR));
    newU = -sqrt(newU);
    sgn = -1;
    H0 = 0.5 * (newU * newU + (J * J) / (newR * newR));
    deltaT -= tR0;
    tlim = 10 * dt;
    tR0 = 10 * dt;
  }
  if (tlim < deltaT) {
    newR = sqrt(pow(fabs(newR * newU) - 2 * sgn * H0 * tlim, 2) + J * J) *
           pow(2 * H0, -0.5);
    newU = 0;
    H0 = 0.5 * (J * J) / (newR * newR);
    sgn = -1;
    deltaT -= tlim;
    tR0 -= tlim;
    tlim = 10 * dt;
    /* the reference prints and exits the process on tR0<deltaT here
       (:389-391).  Reached with a reflection radius R0 > 0 only, by cells
       inside R0 (reflective kernel, kernelBufferSize > 0); *halted reports
       it and vlo_create then fails, as the reference run ends there */
    if (tR0 < deltaT && halted) *halted = 1;
  }
  newR = sqrt(pow(fabs(newR * newU) - 2 * sgn * H0 * deltaT, 2) + J * J) *
         pow(2 * H0, -0.5);
  newU = (2 * H0 - (J * J) / (newR * newR));
  if (newU <= 0)
    newU = 0;
  else
    newU = sgn * sqrt(newU);
  *outR = newR;
  *outU = newU;
}

/* localSpline::pos2Coord, localSpline.hxx:352-358 */
static void pos2coord(const vlo_ctx *c, double p, int dir, int32_t *I,
                      double *F) {
  double ip, x;
  int sct = dir == 0 ? c->p.Pscale : c->p.Uscale[0];
  p = rescale(p, sct);
  x = (p - c->sstart[dir]) * c->sstep_inv[dir];
  x = modf(x, &ip);
  /* (int) of a non-finite or huge value is undefined in C; such cells are
     never evaluated (they are out of the box), so store a sentinel */
  if (!(ip > -2.0e9 && ip < 2.0e9))
    *I = INT32_MIN;
  else
    *I = (int32_t)ip;
  *F = x;
}

/* vlasovSolver21::generateDisplacement, vlasovSolver21.hxx:102-143, and
   vlasovSolver21_spline::decomposeDisplacement, vlasovSolver21_spline.hxx:76-100 */
static void generate_displacement(vlo_ctx *c, double dt, int reflective) {
  const double dth = 0.5 * dt;
  const double R0 = reflective ? c->kernelRadius : -1;
  long j, u, r;
  for (j = 0; j < c->nj; j++) {
    double J = c->J[j];
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        long i = (j * c->nu + u) * c->nr + r;
        double dR, dU;
        int halted = 0;
        advance_particle_drift(c->R[r], c->U[u], J, dth, R0, &dR, &dU, &halted);
        if (halted && c->halted_cell < 0) c->halted_cell = i;
        c->driftR[i] = dR;
        c->driftU[i] = dU;
        c->driftOut[i] = ((dR >= c->R[c->nr - 1]) || (dR <= c->R[0]) ||
                          (dU >= c->U[c->nu - 1]) || (dU <= c->U[0]))
                             ? 1
                             : 0;
      }
  }
  for (long i = 0; i < c->nr * c->nu * c->nj; i++) {
    pos2coord(c, c->driftR[i], 0, &c->rI[i], &c->rF[i]);
    pos2coord(c, c->driftU[i], 1, &c->uI[i], &c->uF[i]);
  }
}

/* ----------------------------------------------------------------- chains */

static void chain_push(vlo_ctx *c, double R, double U, double v) {
  if (c->nel == c->cap_el) {
    c->cap_el = c->cap_el ? 2 * c->cap_el : 1024;
    c->el_R = (double *)realloc(c->el_R, sizeof(double) * c->cap_el);
    c->el_U = (double *)realloc(c->el_U, sizeof(double) * c->cap_el);
    c->el_val = (double *)realloc(c->el_val, sizeof(double) * c->cap_el);
  }
  c->el_R[c->nel] = R;
  c->el_U[c->nel] = U;
  c->el_val[c->nel] = v;
  c->nel++;
  c->ch_len[c->nch - 1]++;
}

/* vlasovSolver21::setupBoundaryConditions, vlasovSolver21.hxx:265-326
   (sphericalKernel::newChain sphericalKernel.hxx:67-80, cellChain::push
   cellChain.hxx:26-29, the tail dummyCell21(R,U,1) dummyCell21_vect.hxx:35-39) */
static int setup_chains(vlo_ctx *c, double dt) {
  const double dth = 0.5 * dt;
  long j, u, r;
  if (c->p.kernelType != VLO_DELAYED) return 0;
  for (j = 0; j < c->nj; j++) {
    double J = c->J[j];
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        long i = (j * c->nu + u) * c->nr + r;
        double nR, nU, deltaT;
        if (!(c->driftR[i] < c->kernelRadius)) continue;
        if (c->nch == c->cap_ch) {
          c->cap_ch = c->cap_ch ? 2 * c->cap_ch : 256;
          c->ch_cell =
              (int64_t *)realloc(c->ch_cell, sizeof(int64_t) * c->cap_ch);
          c->ch_start =
              (int64_t *)realloc(c->ch_start, sizeof(int64_t) * c->cap_ch);
          c->ch_len = (int32_t *)realloc(c->ch_len, sizeof(int32_t) * c->cap_ch);
        }
        c->ch_cell[c->nch] = i;
        c->ch_start[c->nch] = c->nel;
        c->ch_len[c->nch] = 0;
        c->cell2ch[i] = c->nch;
        c->nch++;
        deltaT = dth;
        advance_particle_drift(c->R[r], c->U[u], J, deltaT, -1, &nR, &nU, NULL);
        while (nR < c->kernelRadius) {
          chain_push(c, nR, nU, profile_value(c, nR, nU, J));
          deltaT += dth;
          advance_particle_drift(c->R[r], c->U[u], J, deltaT, -1, &nR, &nU, NULL);
        }
        chain_push(c, nR, nU, 0.0);
      }
  }
  return 0;
}

/* ------------------------------------------------------ spline prefilter */

/* localSpline::create_1D for NATURAL boundaries at both ends,
   localSpline.hxx:953-1182 (rows :976-981, :1002-1008, :1019-1024; forward
   elimination :1045-1059 and :1104-1112; last row :1143-1153; back
   substitution :1155-1172).  tab[k*delta], k=0..M-1, M = dim+2; the interior
   k=1..M-2 holds the data on entry and every k holds a coefficient on exit. */
static void create_1d(double *A, double *tab, long dim, double hi,
                      long delta) {
  const long M = dim + 2;
  double *a = A;
  double *t = &tab[delta];
  long row;
  {
    double hi2 = hi * hi;
    a[0] = hi2;
    a[1] = -2.0 * hi2;
    a[2] = hi2;
    a[3] = 0;
  }
  a += 4;
  for (long i = 1; i < M - 1; i++, t += delta, a += 4) {
    a[0] = 1.0 / 6.0;
    a[1] = 4.0 / 6.0;
    a[2] = 1.0 / 6.0;
    a[3] = *t;
  }
  a = &A[(M - 1) * 4];
  {
    double hi2 = hi * hi;
    a[0] = hi2;
    a[1] = -2.0 * hi2;
    a[2] = hi2;
    a[3] = 0;
  }
  A[4 * (0) + 1] /= A[4 * (0) + 0];
  A[4 * (0) + 2] /= A[4 * (0) + 0];
  A[4 * (0) + 3] /= A[4 * (0) + 0];
  A[4 * (0) + 0] = 1.0;
  A[4 * (1) + 1] -= A[4 * (1) + 0] * A[4 * (0) + 1];
  A[4 * (1) + 2] -= A[4 * (1) + 0] * A[4 * (0) + 2];
  A[4 * (1) + 3] -= A[4 * (1) + 0] * A[4 * (0) + 3];
  A[4 * (1) + 0] = 0.0;
  A[4 * (1) + 2] /= A[4 * (1) + 1];
  A[4 * (1) + 3] /= A[4 * (1) + 1];
  A[4 * (1) + 1] = 1.0;
  row = 2;
  a = &A[4 * (row - 1) + 0];
  for (; row < M - 1; row++, a += 4) {
    a[4 + 1] -= a[4 + 0] * a[2];
    a[4 + 3] -= a[4 + 0] * a[3];
    a[4 + 2] /= a[4 + 1];
    a[4 + 3] /= a[4 + 1];
    a[4 + 0] = 0.0;
    a[4 + 1] = 1.0;
  }
  A[4 * (M - 1) + 1] -= A[4 * (M - 1) + 0] * A[4 * (M - 3) + 2];
  A[4 * (M - 1) + 3] -= A[4 * (M - 1) + 0] * A[4 * (M - 3) + 3];
  A[4 * (M - 1) + 2] -= A[4 * (M - 1) + 1] * A[4 * (M - 2) + 2];
  A[4 * (M - 1) + 3] -= A[4 * (M - 1) + 1] * A[4 * (M - 2) + 3];
  A[4 * (M - 1) + 3] /= A[4 * (M - 1) + 2];
  A[4 * (M - 1) + 2] = 1.0;

  t = &tab[delta * (M - 1)];
  *t = A[4 * (M - 1) + 3];
  t -= delta;
  for (row = M - 2; row > 0; row--, t -= delta)
    (*t) = A[4 * (row) + 3] - A[4 * (row) + 2] * t[delta];
  (*t) = A[4 * (0) + 3] - A[4 * (0) + 1] * t[delta] - A[4 * (0) + 2] * t[2 * delta];
}

/* localSpline::assign (localSpline.hxx:210-246) + create_2D
   (localSpline.hxx:1238-1258): r-solves on the interior u-rows, then u-solves
   on every r-column including both ghost columns. */
static void build_2d(double *A, double *coef, const double *f, long nr,
                     long nu, double hi_r, double hi_u) {
  const long s1 = nr + 2;
  long u, r;
  for (u = 0; u < nu; u++)
    for (r = 0; r < nr; r++) coef[(u + 1) * s1 + (r + 1)] = f[u * nr + r];
  for (u = 0; u < nu; u++) create_1d(A, &coef[(u + 1) * s1], nr, hi_r, 1);
  for (r = -1; r <= nr; r++) create_1d(A, &coef[r + 1], nu, hi_u, s1);
}

void vlo_prefilter2d(long nr, long nu, double hi_r, double hi_u,
                     const double *f, double *coef) {
  long m = (nr > nu ? nr : nu) + 2;
  double *A = (double *)malloc(sizeof(double) * 4 * m);
  memset(coef, 0, sizeof(double) * (nr + 2) * (nu + 2));
  build_2d(A, coef, f, nr, nu, hi_r, hi_u);
  free(A);
}

static inline double BV2(double x) { return x * x * x; }
static inline double BV1(double x) {
  return 1.0 + 3.0 * x + 3.0 * x * x - 3.0 * x * x * x;
}

/* localSpline::evaluateC(int,double,int,double), localSpline.hxx:381-398 */
static double evaluate_c(const double *d, long s1, int Nx, double x, int Ny,
                         double y) {
  long ref0, ref1, ref2, ref3;
  double b2xI, b1xI, b2x, b1x, result;
  Nx++;
  Ny++;
  ref0 = Nx + (Ny - 1) * s1;
  ref1 = Nx + Ny * s1;
  ref2 = Nx + (Ny + 1) * s1;
  ref3 = Nx + (Ny + 2) * s1;
  b2xI = BV2(1. - x);
  b1xI = BV1(1. - x);
  b2x = BV2(x);
  b1x = BV1(x);
  result = 1.0 / 36.0;
  result *=
      BV2(1. - y) * (d[ref0 - 1] * b2xI + d[ref0] * b1xI + d[ref0 + 1] * b1x + d[ref0 + 2] * b2x) +
      BV1(1. - y) * (d[ref1 - 1] * b2xI + d[ref1] * b1xI + d[ref1 + 1] * b1x + d[ref1 + 2] * b2x) +
      BV1(y) * (d[ref2 - 1] * b2xI + d[ref2] * b1xI + d[ref2 + 1] * b1x + d[ref2 + 2] * b2x) +
      BV2(y) * (d[ref3 - 1] * b2xI + d[ref3] * b1xI + d[ref3 + 1] * b1x + d[ref3 + 2] * b2x);
  return result;
}

/* localSpline::evaluateNxPy, localSpline.hxx:423-441 (u is a linear scale) */
static double evaluate_nxpy(const vlo_ctx *c, const double *d, long s1,
                            int Nx, double yy) {
  double y, ip, result;
  int Ny;
  long ref0, ref1, ref2, ref3;
  Nx++;
  yy = rescale(yy, c->p.Uscale[0]);
  y = (yy - c->sstart[1]) * c->sstep_inv[1];
  y = modf(y, &ip);
  Ny = 1 + (int)ip;
  ref0 = Nx + (Ny - 1) * s1;
  ref1 = Nx + Ny * s1;
  ref2 = Nx + (Ny + 1) * s1;
  ref3 = Nx + (Ny + 2) * s1;
  result = 1.0 / 36.0;
  result *= BV2(1. - y) * (d[ref0 - 1] + d[ref0] * 4 + d[ref0 + 1]) +
            BV1(1. - y) * (d[ref1 - 1] + d[ref1] * 4 + d[ref1 + 1]) +
            BV1(y) * (d[ref2 - 1] + d[ref2] * 4 + d[ref2 + 1]) +
            BV2(y) * (d[ref3 - 1] + d[ref3] * 4 + d[ref3 + 1]);
  return result;
}

/* the two gathers on a padded coefficient slice of row pitch s1 (exposed
   for the spline-level tests): evaluateC at (Nx, x, Ny, y), and evaluateNxPy's
   sum at node Nx and (Ny, y) already decomposed by pos2Coord (Ny = the integer
   part, before localSpline's "1 +") */
double vlo_evaluate_c(const double *coef, long s1, int Nx, double x, int Ny, double y) {
  return evaluate_c(coef, s1, Nx, x, Ny, y);
}
double vlo_evaluate_nxpy(const double *d, long s1, int Nx, int Ny0, double y) {
  long ref0, ref1, ref2, ref3;
  int Ny = 1 + Ny0;
  double result;
  Nx++;
  ref0 = Nx + (Ny - 1) * s1;
  ref1 = Nx + Ny * s1;
  ref2 = Nx + (Ny + 1) * s1;
  ref3 = Nx + (Ny + 2) * s1;
  result = 1.0 / 36.0;
  result *= BV2(1. - y) * (d[ref0 - 1] + d[ref0] * 4 + d[ref0 + 1]) +
            BV1(1. - y) * (d[ref1 - 1] + d[ref1] * 4 + d[ref1 + 1]) +
            BV1(y) * (d[ref2 - 1] + d[ref2] * 4 + d[ref2 + 1]) +
            BV2(y) * (d[ref3 - 1] + d[ref3] * 4 + d[ref3 + 1]);
  return result;
}

/* localSpline::evaluate(double,double), localSpline.hxx:477-488 */
static double evaluate_xy(const vlo_ctx *c, const double *d, long s1,
                          double xx, double yy) {
  double x, y, ix, iy;
  xx = rescale(xx, c->p.Pscale);
  yy = rescale(yy, c->p.Uscale[0]);
  x = (xx - c->sstart[0]) * c->sstep_inv[0];
  y = (yy - c->sstart[1]) * c->sstep_inv[1];
  x = modf(x, &ix);
  y = modf(y, &iy);
  /* the reference reads out of the padded array when a tail lies beyond
     r_max; clamp the read so the oracle stays defined (never hit by the
     configurations in use) */
  if (ix < 0 || ix > c->nr - 2 || iy < 0 || iy > c->nu - 2) {
    fprintf(stderr, "vls_oracle: chain tail outside the spline box\n");
    return 0;
  }
  return evaluate_c(d, s1, (int)ix, x, (int)iy, y);
}

/* ------------------------------------------------------------- quadrature */

/* slice21Iterator::get_dR/get_dU/get_dJ, slice21Iterator.hxx:84-86 (get_dJ
   compares j against the u-vertex count, as the reference does) */
static double get_dR(const vlo_ctx *c, long r) {
  return (r >= c->nr - 1) ? 0 : (c->R[r + 1] - c->R[r]);
}
static double get_dU(const vlo_ctx *c, long u) {
  return (u >= c->nu - 1) ? 0 : (c->U[u + 1] - c->U[u]);
}
static double get_dJ(const vlo_ctx *c, long j) {
  return (j >= c->nu - 1) ? 0 : (c->JV[j + 1] - c->JV[j]);
}

enum { IG_F = 0, IG_EK, IG_S, IG_L1, IG_L2 };

/* integrand21 functors, integrand21.hxx:66-145, on the 4-corner average
   slice21Iterator::get_avg, slice21Iterator.hxx:90-94 */
static double integrand(int which, double r, double u, double j,
                        const double *fi, long nr) {
  double avg = (fi[0] + fi[1] + fi[nr] + fi[nr + 1]) * 0.25;
  switch (which) {
    case IG_F:
      return avg;
    case IG_EK:
      return 0.5 * avg * (u * u + j * j / (r * r));
    case IG_S:
      return (avg <= 0) ? 0 : -avg * log(avg);
    case IG_L1:
      return fabs(avg);
    case IG_L2:
      return avg * avg;
  }
  return 0;
}

/* quadrature21::integrate, quadrature21.hxx:56-85 (one thread) */
static double integrate(const vlo_ctx *c, const double *f, int which) {
  double res = 0;
  long j, u, r;
  for (j = 0; j < c->nj; j++) {
    double J = c->J[j];
    double dJ = get_dJ(c, j);
    double Ct1 = 8 * M_PI * M_PI * J * dJ;
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        double dU = get_dU(c, u), dR;
        if (dU <= 0) continue;
        dR = get_dR(c, r);
        if (dR <= 0) continue;
        res += Ct1 * dU * dR *
               integrand(which, c->R[r] + 0.5 * dR, c->U[u] + 0.5 * dU, J,
                         &f[(j * c->nu + u) * c->nr + r], c->nr);
      }
  }
  return res;
}

/* quadrature21::integrate1D along r, quadrature21.hxx:87-142 (one thread) */
static void integrate1d_r(const vlo_ctx *c, const double *f, double *bins) {
  long j, u, r;
  for (r = 0; r < c->nr; r++) bins[r] = 0;
  for (j = 0; j < c->nj; j++) {
    double J = c->J[j];
    double dJ = get_dJ(c, j);
    double Ct1 = 8 * M_PI * M_PI * J * dJ;
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        double dU = get_dU(c, u), dR, tmp;
        if (dU <= 0) continue;
        dR = get_dR(c, r);
        if (dR <= 0) continue;
        tmp = Ct1 * dU * dR *
              integrand(IG_F, c->R[r] + 0.5 * dR, c->U[u] + 0.5 * dU, J,
                        &f[(j * c->nu + u) * c->nr + r], c->nr);
        bins[r] += tmp;
      }
  }
}

/* gridHandler::accumulate with addSpare=1, grid_handler.hxx:350-407:
   Mr[r] = sum of bins strictly below r; returns the total */
static double accumulate(const vlo_ctx *c, const double *bins, double *Mr) {
  double run = 0;
  long r;
  for (r = 0; r < c->nr; r++) {
    Mr[r] = run;
    run = run + bins[r];
  }
  return run;
}

double vlo_moments(const vlo_ctx *c, double *bins, double *Mr) {
  integrate1d_r(c, c->f, bins);
  return accumulate(c, bins, Mr);
}

/* ------------------------------------------------------------------- step */

static void kick(vlo_ctx *c, const double *shift) {
  const long s1 = c->nr + 2;
  long j, u, r;
  for (j = 0; j < c->nj; j++) {
    double *fj = &c->f[j * c->nu * c->nr];
    build_2d(c->tmpA, c->coef, fj, c->nr, c->nu, c->sstep_inv[0],
             c->sstep_inv[1]);
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        double newU = c->U[u] + shift[r];
        double *it = &fj[u * c->nr + r];
        if ((newU <= c->U[0]) || (newU >= c->U[c->nu - 1]))
          *it = 0;
        else
          *it = evaluate_nxpy(c, c->coef, s1, (int)r, newU);
      }
  }
}

void vlo_kick(vlo_ctx *c, const double *shift) { kick(c, shift); }

/* cellChain::readRoll + roll, cellChain.hxx:49-63: return the front value and
   rotate the values by one towards the front */
static double chain_read_roll(vlo_ctx *c, long ch) {
  double *v = &c->el_val[c->ch_start[ch]];
  long L = c->ch_len[ch];
  double front = v[0];
  for (long k = 0; k < L - 1; k++) v[k] = v[k + 1];
  v[L - 1] = front;
  return front;
}

/* drift half of vlasovSolver21_spline::makeOneStep, vlasovSolver21_spline.hxx:769-798 */
static void drift(vlo_ctx *c) {
  const long s1 = c->nr + 2;
  long j, u, r, ch;
  long ch0 = 0;
  for (j = 0; j < c->nj; j++) {
    double *fj = &c->f[j * c->nu * c->nr];
    build_2d(c->tmpA, c->coef, fj, c->nr, c->nu, c->sstep_inv[0],
             c->sstep_inv[1]);
    if (c->p.kernelType == VLO_DELAYED) {
      /* chains of this slice are contiguous in build order */
      for (ch = ch0; ch < c->nch && c->ch_cell[ch] < (j + 1) * c->nu * c->nr;
           ch++) {
        long t = c->ch_start[ch] + c->ch_len[ch] - 1;
        if ((c->el_U[t] <= c->U[0]) || (c->el_U[t] >= c->U[c->nu - 1]))
          c->el_val[t] = 0;
        else
          c->el_val[t] = evaluate_xy(c, c->coef, s1, c->el_R[t], c->el_U[t]);
      }
    }
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++) {
        long i = (j * c->nu + u) * c->nr + r;
        if (c->driftR[i] < c->kernelRadius) {
          if (c->cell2ch[i] >= 0)
            fj[u * c->nr + r] = chain_read_roll(c, c->cell2ch[i]);
          else
            fj[u * c->nr + r] = 0; /* reflective kernel: no chain exists */
        } else if (c->driftOut[i])
          fj[u * c->nr + r] = 0;
        else
          fj[u * c->nr + r] = evaluate_c(c->coef, s1, c->rI[i], c->rF[i],
                                         c->uI[i], c->uF[i]);
      }
    while (ch0 < c->nch && c->ch_cell[ch0] < (j + 1) * c->nu * c->nr) ch0++;
  }
}

void vlo_drift(vlo_ctx *c) { drift(c); }

/* vlasovSolver21_spline::makeOneStep, vlasovSolver21_spline.hxx:680-801 */
void vlo_step(vlo_ctx *c, int nsteps) {
  double *bins = (double *)malloc(sizeof(double) * c->nr);
  double *Mr = (double *)malloc(sizeof(double) * c->nr);
  for (int s = 0; s < nsteps; s++) {
    if (c->p.noLinking) drift(c);
    integrate1d_r(c, c->f, bins);
    accumulate(c, bins, Mr);
    for (long i = 0; i < c->nr; i++)
      Mr[i] *= c->p.G / (c->R[i] * c->R[i]) * c->p.dt;
    kick(c, Mr);
    drift(c);
  }
  free(bins);
  free(Mr);
}

/* ------------------------------------------------------------- statistics */

/* vlasovSolver21::potentialEnergy (vlasovSolver21.hxx:627-642) and
   statistics (:644-690).  The reference reads one element past R_Val for the
   last shell, whose mass is always 0; that term is taken as 0. */
void vlo_stats(const vlo_ctx *c, double *out7) {
  double *bins = (double *)malloc(sizeof(double) * c->nr);
  double M = 0, Ep = 0;
  integrate1d_r(c, c->f, bins);
  for (long i = 1; i < c->nr + 1; i++) {
    double Mi = bins[i - 1];
    if (i < c->nr) {
      double r = 0.5 * (c->R[i - 1] + c->R[i]);
      Ep -= (Mi * c->p.G * M) / r;
    }
    M += Mi;
  }
  free(bins);
  {
    double Ek = integrate(c, c->f, IG_EK);
    double E = Ek + Ep;
    double S = integrate(c, c->f, IG_S);
    double L1 = integrate(c, c->f, IG_L1);
    double L2 = integrate(c, c->f, IG_L2);
    out7[0] = M;
    out7[1] = E;
    out7[2] = Ek;
    out7[3] = Ep;
    out7[4] = S;
    out7[5] = L1;
    out7[6] = L2;
  }
}

/* ------------------------------------------------------------------ setup */

/* vlasovSolver::init (vlasovSolver.hxx:61-102): grid generation
   (grid_base.hxx:258-300), initial conditions (initGen_*::generate),
   vlasovSolver21::setup (vlasovSolver21.hxx:411-446, :533-548),
   vlasovSolver21_spline::setup (vlasovSolver21_spline.hxx:296-374) and
   renormalize (vlasovSolver21.hxx:468-524). */
vlo_ctx *vlo_create(const vlo_params *p) {
  vlo_ctx *c = (vlo_ctx *)calloc(1, sizeof(vlo_ctx));
  long n, ncell, i, j, u, r;
  double *scl;
  c->p = *p;
  c->R = gen_scale(p->Pmin, p->Pmax, p->Pres, p->Pscale, 1, &c->nr);
  c->U = gen_scale(p->Umin[0], p->Umax[0], p->Ures[0], p->Uscale[0], 1, &c->nu);
  c->J = gen_scale(p->Umin[1], p->Umax[1], p->Ures[1], p->Uscale[1], 0, &c->nj);
  c->JV = gen_scale(p->Umin[1], p->Umax[1], p->Ures[1], p->Uscale[1], 1, &n);
  /* localSpline::init, localSpline.hxx:60-93 */
  scl = gen_scale(c->R[0], c->R[c->nr - 1], c->nr - 1, p->Pscale, 1, &n);
  c->sstart[0] = rescale(scl[0], p->Pscale);
  {
    double stop = rescale(scl[n - 1], p->Pscale);
    double step = (stop - c->sstart[0]) / (n - 1);
    c->sstep_inv[0] = 1. / step;
  }
  free(scl);
  scl = gen_scale(c->U[0], c->U[c->nu - 1], c->nu - 1, p->Uscale[0], 1, &n);
  c->sstart[1] = rescale(scl[0], p->Uscale[0]);
  {
    double stop = rescale(scl[n - 1], p->Uscale[0]);
    double step = (stop - c->sstart[1]) / (n - 1);
    c->sstep_inv[1] = 1. / step;
  }
  free(scl);
  /* vlasovSolver21::setup, vlasovSolver21.hxx:436-438 */
  c->kernelRadius = c->R[p->kernelBufferSize];

  ncell = c->nr * c->nu * c->nj;
  c->f = (double *)malloc(sizeof(double) * ncell);
  c->coef = (double *)calloc((c->nr + 2) * (c->nu + 2), sizeof(double));
  c->tmpA = (double *)malloc(sizeof(double) * 4 *
                             ((c->nr > c->nu ? c->nr : c->nu) + 2));
  c->driftR = (double *)malloc(sizeof(double) * ncell);
  c->driftU = (double *)malloc(sizeof(double) * ncell);
  c->driftOut = (uint8_t *)malloc(ncell);
  c->rI = (int32_t *)malloc(sizeof(int32_t) * ncell);
  c->uI = (int32_t *)malloc(sizeof(int32_t) * ncell);
  c->rF = (double *)malloc(sizeof(double) * ncell);
  c->uF = (double *)malloc(sizeof(double) * ncell);
  c->cell2ch = (int64_t *)malloc(sizeof(int64_t) * ncell);
  for (i = 0; i < ncell; i++) c->cell2ch[i] = -1;

  setup_profile(c);
  for (j = 0; j < c->nj; j++)
    for (u = 0; u < c->nu; u++)
      for (r = 0; r < c->nr; r++)
        c->f[(j * c->nu + u) * c->nr + r] =
            profile_value(c, c->R[r], c->U[u], c->J[j]);

  {
    double dtd = p->noLinking ? p->dt : p->dt * 2;
    c->halted_cell = -1;
    generate_displacement(c, dtd, p->kernelType == VLO_REFLECTIVE);
    if (c->halted_cell >= 0) {
      /* the reference terminates in generateDisplacement for this set-up */
      vlo_destroy(c);
      return NULL;
    }
    setup_chains(c, dtd);
  }
  /* renormalize(init->getMass(0), 0) */
  {
    double mass = integrate(c, c->f, IG_F) + 0; /* kernelMass = 0 */
    double fac = p->M / mass;
    if (p->M > 0) {
      for (i = 0; i < ncell; i++) c->f[i] *= fac;
      for (i = 0; i < c->nel; i++) c->el_val[i] *= fac;
    }
  }
  return c;
}

void vlo_destroy(vlo_ctx *c) {
  if (!c) return;
  free(c->R); free(c->U); free(c->J); free(c->JV);
  free(c->f); free(c->coef); free(c->tmpA);
  free(c->driftR); free(c->driftU); free(c->driftOut);
  free(c->rI); free(c->uI); free(c->rF); free(c->uF);
  free(c->cell2ch);
  free(c->ch_cell); free(c->ch_start); free(c->ch_len);
  free(c->el_R); free(c->el_U); free(c->el_val);
  free(c);
}

void vlo_dims(const vlo_ctx *c, long *nr, long *nu, long *nj) {
  *nr = c->nr;
  *nu = c->nu;
  *nj = c->nj;
}

void vlo_coords(const vlo_ctx *c, double *R, double *U, double *J,
                double *JV) {
  if (R) memcpy(R, c->R, sizeof(double) * c->nr);
  if (U) memcpy(U, c->U, sizeof(double) * c->nu);
  if (J) memcpy(J, c->J, sizeof(double) * c->nj);
  if (JV) memcpy(JV, c->JV, sizeof(double) * (c->nj + 1));
}

void vlo_spline_consts(const vlo_ctx *c, double *start, double *step_inv) {
  start[0] = c->sstart[0];
  start[1] = c->sstart[1];
  step_inv[0] = c->sstep_inv[0];
  step_inv[1] = c->sstep_inv[1];
}

double vlo_kernel_radius(const vlo_ctx *c) { return c->kernelRadius; }

void vlo_get_f(const vlo_ctx *c, double *out) {
  memcpy(out, c->f, sizeof(double) * c->nr * c->nu * c->nj);
}

void vlo_set_f(vlo_ctx *c, const double *in) {
  memcpy(c->f, in, sizeof(double) * c->nr * c->nu * c->nj);
}

void vlo_get_footpoints(const vlo_ctx *c, double *driftR, double *driftU,
                        uint8_t *out, int32_t *rI, double *rF, int32_t *uI,
                        double *uF) {
  long n = c->nr * c->nu * c->nj;
  if (driftR) memcpy(driftR, c->driftR, sizeof(double) * n);
  if (driftU) memcpy(driftU, c->driftU, sizeof(double) * n);
  if (out) memcpy(out, c->driftOut, n);
  if (rI) memcpy(rI, c->rI, sizeof(int32_t) * n);
  if (rF) memcpy(rF, c->rF, sizeof(double) * n);
  if (uI) memcpy(uI, c->uI, sizeof(int32_t) * n);
  if (uF) memcpy(uF, c->uF, sizeof(double) * n);
}

void vlo_chain_counts(const vlo_ctx *c, long *n_chains, long *n_elems) {
  *n_chains = c->nch;
  *n_elems = c->nel;
}

void vlo_get_chains(const vlo_ctx *c, int64_t *cell, int64_t *start,
                    int32_t *len, double *R, double *U, double *val) {
  if (cell) memcpy(cell, c->ch_cell, sizeof(int64_t) * c->nch);
  if (start) memcpy(start, c->ch_start, sizeof(int64_t) * c->nch);
  if (len) memcpy(len, c->ch_len, sizeof(int32_t) * c->nch);
  if (R) memcpy(R, c->el_R, sizeof(double) * c->nel);
  if (U) memcpy(U, c->el_U, sizeof(double) * c->nel);
  if (val) memcpy(val, c->el_val, sizeof(double) * c->nel);
}

void vlo_set_chain_vals(vlo_ctx *c, const double *val) {
  memcpy(c->el_val, val, sizeof(double) * c->nel);
}
