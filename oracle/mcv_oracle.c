/*
 * mcv_oracle.c -- FP64 CPU restatement of MCV_SW's explicit time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed
 * CPU baseline.  Only the test suite, the smoke check and the benchmark's CPU
 * baseline leg load it.  The GPU product never links or calls it.
 *
 * Parity status: unpinned by reference-run fixtures.  The reference ships no
 * tests or golden vectors and cannot be compiled in this image (Fortran 90, no
 * Fortran compiler).  The restatement is instead pinned by analytic known
 * answers (polynomial exactness of the reconstruction and ghost interpolation,
 * total cube area, steady-state convergence of Williamson case 2).
 *
 * The restatement follows the reference function for function and keeps its
 * evaluation order (Fortran evaluates a+b+c as (a+b)+c; x**2 and x**2. are
 * products x*x; x**3. and x**4. are pow() calls, as GCC lowers them without
 * -ffast-math).  It is compiled without FMA contraction so the arithmetic is
 * the reference's own (gfortran -O3 -fdefault-real-8 on x86-64).
 *
 * Reference files restated here (paths inside the MCV_SW project):
 *   src/constants_mod.F90, src/parameters_mod.F90, src/projection_mod.F90,
 *   src/mesh_mod.F90, src/ghost_mod.f90, src/stat_mod.F90, src/tend_mod.F90,
 *   src/spatial_operators_mod.F90, src/time_scheme_mod.F90, src/diag_mod.F90,
 *   src/test_case_mod.F90.
 *
 * Array layout is the reference's: Fortran column-major (i, j, panel) with the
 * reference's lower bounds (i, j from ips = 2 - DOF; panels 1..6); 2x2 matrices
 * are (2, 2, i, j, panel).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* constants_mod.F90:12-20 (radius is a run parameter here) */
#define GRAVITY 9.80616
#define OMEGA 7.292E-5
#define FILLVALUE (-9999999999999999.)

typedef struct {
  double *u, *v, *phi, *phiG, *contraU, *contraV, *zonal_wind, *meridional_wind;
} orc_stat;

typedef struct {
  double *u, *v, *phiG;
} orc_tend;

typedef struct orc_ctx {
  int DOF, scheme; /* scheme: 3 = RK3_TVD, 4 = RK4 */
  double radius, pi, D2R, dt, dx, dy, x_min, x_max, y_min, y_max;
  int Nx, Ny, nPVx, nPVy;
  int ids, ide, jds, jde, ics, ice, jcs, jce, its, ite, jts, jte, ips, ipe, jps, jpe;
  int nPVHalo, nsub;
  long npx, npy, ncx, ncy; /* padded PV and cell extents */
  long NP;                 /* padded points per field (6 panels) */
  /* mesh_mod.F90:9-45 */
  double *xP, *yP, *lonP, *latP, *sqrtG, *matrixG, *matrixIG, *matrixA, *matrixIA, *f, *phi_s;
  double *areaCell;
  double weightsOnPV[4][4];
  int *pvIdx; /* pvIdx(iDOF, iCell), iCell in ics..ice */
  /* ghost_mod.f90:11-18 */
  double *gX, *gY, *gCoef;
  int *gIref;
  /* stat(-nsub:1), tend(-nsub:1) */
  orc_stat stat[6];
  orc_tend tend[6];
  /* spatial_operator automatic arrays, allocated once */
  double *flux_x, *flux_y, *div_x, *div_y, *dvdx, *dudy, *vort;
  double *K, *E, *phiGu, *phiGv;
  /* CubedSphereFillGhost / unify temporaries */
  double *ghost_target, *field_inner, *field_raw;
  int old_slot, new_slot;
} orc_ctx;

/* ---- indexing helpers (Fortran bounds) ---- */
#define PIX(c, i, j, p) ((long)((i) - (c)->ips) + (c)->npx * ((long)((j) - (c)->jps) + (c)->npy * (long)((p) - 1)))
#define MIX(c, a, b, i, j, p) ((long)((a) - 1) + 2L * (long)((b) - 1) + 4L * PIX(c, i, j, p))
#define IIX(c, i, j, p) ((long)((i) - (c)->ids) + (long)(c)->nPVx * ((long)((j) - (c)->jds) + (long)(c)->nPVy * (long)((p) - 1)))
#define CIX(c, i, j, p) ((long)((i) - (c)->ics) + (c)->ncx * ((long)((j) - (c)->jcs) + (c)->ncy * (long)((p) - 1)))
#define PVIDX(c, d, cell) ((c)->pvIdx[((d) - 1) + (c)->DOF * ((cell) - (c)->ics)])
#define SLOT(c, t) ((t) + (c)->nsub) /* stat index t in -nsub..1 */

static double sq(double x) { return x * x; }

/* ------------------------------------------------------------------ */
/* projection_mod.F90                                                  */
/* ------------------------------------------------------------------ */

/* projection_mod.F90:8-38 */
static void pointProjPlane2Sphere(const orc_ctx *c, double *lambda, double *theta, double x, double y, int iPatch) {
  double a, b;
  if (iPatch >= 1 && iPatch <= 4) {
    *lambda = x + (double)(iPatch - 1) * c->pi / 2.;
    *theta = atan2(tan(y) * cos(x), 1.);
  } else if (iPatch == 5) {
    a = tan(x);
    b = tan(y);
    *lambda = atan2(a, -b);
    *theta = atan2(1., sqrt(a * a + b * b));
  } else {
    a = tan(x);
    b = tan(y);
    *lambda = atan2(a, b);
    *theta = -atan2(1., sqrt(a * a + b * b));
  }
}

/* projection_mod.F90:40-58 */
static void pointProjSphere2Plane(const orc_ctx *c, double *x, double *y, double lambda, double theta, int iPatch) {
  if (iPatch >= 1 && iPatch <= 4) {
    *x = atan(tan(lambda - (double)(iPatch - 1) * c->pi / 2.));
    *y = atan(tan(theta) / cos(lambda - (double)(iPatch - 1) * c->pi / 2.));
  } else {
    double sgn = ((iPatch + 1) % 2 == 0) ? 1. : -1.; /* (-1.)**(iPatch+1) */
    *x = atan(sgn * sin(lambda) / tan(theta));
    *y = atan(-cos(lambda) / tan(theta));
  }
}

/* matmul(A, B) for 2x2 column-major, as the Fortran intrinsic sums k=1,2 */
static void matmul22(double out[4], const double *A, const double *B) {
  for (int j = 0; j < 2; j++)
    for (int i = 0; i < 2; i++) out[i + 2 * j] = A[i + 0] * B[0 + 2 * j] + A[i + 2] * B[1 + 2 * j];
}

/* projection_mod.F90:60-77 */
static void covProjSphere2Plane(double *cov1, double *cov2, double sv1, double sv2, const double *IA, const double *G) {
  double m[4];
  matmul22(m, G, IA);
  *cov1 = m[0] * sv1 + m[2] * sv2;
  *cov2 = m[1] * sv1 + m[3] * sv2;
}

/* projection_mod.F90:79-96 */
static void covProjPlane2Sphere(double *sv1, double *sv2, double cov1, double cov2, const double *A, const double *IG) {
  double m[4];
  matmul22(m, A, IG);
  *sv1 = m[0] * cov1 + m[2] * cov2;
  *sv2 = m[1] * cov1 + m[3] * cov2;
}

/* projection_mod.F90:98-110 */
static void contravProjSphere2Plane(double *c1, double *c2, double sv1, double sv2, const double *IA) {
  *c1 = IA[0] * sv1 + IA[2] * sv2;
  *c2 = IA[1] * sv1 + IA[3] * sv2;
}

/* projection_mod.F90:138-148 */
static void cov2contrav(double *c1, double *c2, double cov1, double cov2, const double *IG) {
  *c1 = IG[0] * cov1 + IG[2] * cov2;
  *c2 = IG[1] * cov1 + IG[3] * cov2;
}

/* projection_mod.F90:150-170 */
static void calc_matrixG(const orc_ctx *c, double *G, double x, double y) {
  double rho = sqrt(1. + pow(tan(x), 2.) + pow(tan(y), 2.));
  G[0] = 1. + pow(tan(x), 2.);
  G[2] = -tan(x) * tan(y);
  G[1] = G[2];
  G[3] = 1. + pow(tan(y), 2.);
  double fac = sq(c->radius) / (pow(rho, 4.) * pow(cos(x), 2.) * pow(cos(y), 2.));
  for (int k = 0; k < 4; k++) G[k] = fac * G[k];
}

/* projection_mod.F90:172-192 */
static void calc_matrixIG(const orc_ctx *c, double *IG, double x, double y) {
  double rho = sqrt(1. + pow(tan(x), 2.) + pow(tan(y), 2.));
  IG[0] = 1. + pow(tan(y), 2.);
  IG[2] = tan(x) * tan(y);
  IG[1] = IG[2];
  IG[3] = 1. + pow(tan(x), 2.);
  double fac = (pow(rho, 2.) * pow(cos(x), 2.) * pow(cos(y), 2.)) / sq(c->radius);
  for (int k = 0; k < 4; k++) IG[k] = fac * IG[k];
}

/* projection_mod.F90:194-211 */
static void calc_Jacobian(const orc_ctx *c, double *jab, double x, double y) {
  double rho = sqrt(1 + sq(tan(x)) + sq(tan(y)));
  *jab = 1. / (sq(cos(x)) * sq(cos(y)) * (rho * rho * rho));
  *jab = *jab * sq(c->radius);
}

/* projection_mod.F90:213-267 */
static void calc_matrixIA(const orc_ctx *c, double *IA, double lambda, double theta, int iPatch) {
  double al, at, a, b, cc, d, temp;
  if (iPatch <= 4) {
    al = lambda - (double)(iPatch - 1) * c->pi / 2.;
    at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    temp = d * d * b * b + cc * cc;
    IA[0] = 1. / d;
    IA[2] = 0.;
    IA[1] = a * cc / temp;
    IA[3] = b / temp;
  } else if (iPatch == 5) {
    al = lambda; at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    temp = cc + a * a * d * d / cc;
    IA[0] = b / temp;
    IA[2] = -(a / cc / temp);
    temp = cc + b * b * d * d / cc;
    IA[1] = a / temp;
    IA[3] = b / cc / temp;
  } else {
    al = lambda; at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    temp = cc + a * a * d * d / cc;
    IA[0] = -(b / temp);
    IA[2] = a / cc / temp;
    temp = cc + b * b * d * d / cc;
    IA[1] = a / temp;
    IA[3] = b / cc / temp;
  }
  for (int k = 0; k < 4; k++) IA[k] = IA[k] / c->radius;
}

/* projection_mod.F90:269-322 */
static void calc_matrixA(const orc_ctx *c, double *A, double lambda, double theta, int iPatch) {
  double al, at, a, b, cc, d, temp;
  if (iPatch <= 4) {
    al = lambda - (double)(iPatch - 1) * c->pi / 2.;
    at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    A[0] = d;
    A[2] = 0.;
    A[1] = -(cc * d * a / b);
    A[3] = b * d * d + cc * cc / b;
  } else if (iPatch == 5) {
    al = lambda; at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    temp = 1. + a * a * d * d / cc / cc;
    A[0] = b * cc * temp;
    A[1] = -(cc * cc * a * temp);
    temp = 1. + b * b * d * d / cc / cc;
    A[2] = a * cc * temp;
    A[3] = b * cc * cc * temp;
  } else {
    al = lambda; at = theta;
    a = sin(al); b = cos(al); cc = sin(at); d = cos(at);
    temp = 1. + a * a * d * d / cc / cc;
    A[0] = -(b * cc * temp);
    A[1] = cc * cc * a * temp;
    temp = 1. + b * b * d * d / cc / cc;
    A[2] = a * cc * temp;
    A[3] = b * cc * cc * temp;
  }
  for (int k = 0; k < 4; k++) A[k] = A[k] * c->radius;
}

/* ------------------------------------------------------------------ */
/* parameters_mod.F90:134-239 (namelist values passed in)              */
/* ------------------------------------------------------------------ */
static int init_parameters(orc_ctx *c, int dof, double dx_deg, double dt, int scheme, double radius) {
  c->DOF = dof;
  c->radius = radius;
  c->pi = 2. * asin(1.);
  c->D2R = c->pi / 180.;
  c->dt = dt;
  c->x_min = -45.; c->x_max = 45.; c->y_min = -45.; c->y_max = 45.;
  double dx = dx_deg, dy = dx_deg;
  if ((c->x_max - c->x_min) / dx - (double)(int)((c->x_max - c->x_min) / dx) != 0.) return -1;
  c->Nx = (int)((c->x_max - c->x_min) / dx);
  c->Ny = (int)((c->y_max - c->y_min) / dy);
  c->nPVx = c->Nx * (dof - 1) + 1;
  c->nPVy = c->Ny * (dof - 1) + 1;
  c->ids = 1; c->ide = c->nPVx; c->jds = 1; c->jde = c->nPVy;
  int xhalo = 1, yhalo = 1;
  c->ics = 1 - xhalo; c->ice = c->Nx + xhalo; c->jcs = 1 - yhalo; c->jce = c->Ny + yhalo;
  c->its = 1; c->ite = c->Nx; c->jts = 1; c->jte = c->Ny;
  c->ips = 1 - xhalo * (dof - 1); c->ipe = c->nPVx + xhalo * (dof - 1);
  c->jps = 1 - yhalo * (dof - 1); c->jpe = c->nPVy + yhalo * (dof - 1);
  c->nPVHalo = xhalo * (dof - 1);
  c->dx = dx * c->D2R; c->dy = dy * c->D2R;
  c->x_min = c->x_min * c->D2R; c->x_max = c->x_max * c->D2R;
  c->y_min = c->y_min * c->D2R; c->y_max = c->y_max * c->D2R;
  if (scheme == 3) c->nsub = 3;
  else if (scheme == 4) c->nsub = 4;
  else return -2;
  c->scheme = scheme;
  c->npx = c->ipe - c->ips + 1; c->npy = c->jpe - c->jps + 1;
  c->ncx = c->ice - c->ics + 1; c->ncy = c->jce - c->jcs + 1;
  c->NP = c->npx * c->npy * 6;
  return 0;
}

/* ------------------------------------------------------------------ */
/* mesh_mod.F90:57-276                                                 */
/* ------------------------------------------------------------------ */
static void EquiangularAllAreas(const orc_ctx *c, int icube, double *dA) {
  double *gp = malloc(sizeof(double) * (icube + 1));
  double *ang = malloc(sizeof(double) * (icube + 1) * (icube + 1));
  for (int k = 1; k <= icube + 1; k++) gp[k - 1] = -0.25 * c->pi + (c->pi / (double)(2 * icube)) * (double)(k - 1);
  for (int k2 = 1; k2 <= icube + 1; k2++)
    for (int k1 = 1; k1 <= icube + 1; k1++)
      ang[(k1 - 1) + (icube + 1) * (k2 - 1)] = acos(-sin(gp[k1 - 1]) * sin(gp[k2 - 1]));
#define ANG(a, b) ang[((a) - 1) + (icube + 1) * ((b) - 1)]
  for (int k2 = 1; k2 <= icube; k2++)
    for (int k1 = 1; k1 <= icube; k1++) {
      double a1 = ANG(k1, k2), a2 = c->pi - ANG(k1 + 1, k2), a3 = c->pi - ANG(k1, k2 + 1), a4 = ANG(k1 + 1, k2 + 1);
      dA[(k1 - 1) + icube * (k2 - 1)] = -2.0 * c->pi + a1 + a2 + a3 + a4;
    }
#undef ANG
  free(gp);
  free(ang);
}

static void init_mesh(orc_ctx *c) {
  long NP = c->NP;
  c->xP = calloc(NP, sizeof(double)); c->yP = calloc(NP, sizeof(double));
  c->lonP = calloc(NP, sizeof(double)); c->latP = calloc(NP, sizeof(double));
  c->sqrtG = calloc(NP, sizeof(double)); c->f = calloc(NP, sizeof(double)); c->phi_s = calloc(NP, sizeof(double));
  c->matrixG = calloc(4 * NP, sizeof(double)); c->matrixIG = calloc(4 * NP, sizeof(double));
  c->matrixA = calloc(4 * NP, sizeof(double)); c->matrixIA = calloc(4 * NP, sizeof(double));
  c->areaCell = calloc(c->ncx * c->ncy * 6, sizeof(double));
  c->pvIdx = calloc((size_t)c->DOF * c->ncx, sizeof(int));
  int DOF = c->DOF;
  for (int iCell = c->ics; iCell <= c->ice; iCell++)
    for (int iDOF = 1; iDOF <= DOF; iDOF++) PVIDX(c, iDOF, iCell) = (iCell - 1) * DOF + (iDOF - iCell + 1);

#pragma omp parallel for collapse(2) schedule(static)
  for (int iPatch = 1; iPatch <= 6; iPatch++)
    for (int jPV = c->jps; jPV <= c->jpe; jPV++)
      for (int iPV = c->ips; iPV <= c->ipe; iPV++) {
        long k = PIX(c, iPV, jPV, iPatch);
        c->xP[k] = (double)(iPV - 1) * c->dx / (double)(DOF - 1) + c->x_min;
        c->yP[k] = (double)(jPV - 1) * c->dy / (double)(DOF - 1) + c->y_min;
        pointProjPlane2Sphere(c, &c->lonP[k], &c->latP[k], c->xP[k], c->yP[k], iPatch);
        calc_matrixG(c, &c->matrixG[4 * k], c->xP[k], c->yP[k]);
        calc_matrixIG(c, &c->matrixIG[4 * k], c->xP[k], c->yP[k]);
        calc_matrixA(c, &c->matrixA[4 * k], c->lonP[k], c->latP[k], iPatch);
        calc_matrixIA(c, &c->matrixIA[4 * k], c->lonP[k], c->latP[k], iPatch);
        calc_Jacobian(c, &c->sqrtG[k], c->xP[k], c->yP[k]);
        c->f[k] = 2. * OMEGA * sin(c->latP[k]);
      }

  /* mesh_mod.F90:183-203 */
  if (DOF == 3) {
    double w[3] = {1., 4., 1.};
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) c->weightsOnPV[a][b] = w[a] * w[b] / 36.;
  } else {
    double w[4] = {1., 3., 3., 1.};
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) c->weightsOnPV[a][b] = w[a] * w[b] / 80.;
  }
  /* mesh_mod.F90:205-212 */
  double *tmp = malloc(sizeof(double) * c->Nx * c->Nx);
  EquiangularAllAreas(c, c->Nx, tmp);
  for (int k = 0; k < c->Nx * c->Nx; k++) tmp[k] = tmp[k] * sq(c->radius);
  for (int p = 1; p <= 6; p++)
    for (int j = 1; j <= c->Ny; j++)
      for (int i = 1; i <= c->Nx; i++) c->areaCell[CIX(c, i, j, p)] = tmp[(i - 1) + c->Nx * (j - 1)];
  free(tmp);
}

/* ------------------------------------------------------------------ */
/* ghost_mod.f90:21-79                                                 */
/* ------------------------------------------------------------------ */
static int init_ghost(orc_ctx *c) {
  int n = c->nPVx, H = c->nPVHalo;
  c->gX = calloc((size_t)n * H, sizeof(double));
  c->gY = calloc((size_t)n * H, sizeof(double));
  c->gCoef = calloc((size_t)n * H, sizeof(double));
  c->gIref = calloc((size_t)n * H, sizeof(int));
#define GIX(i, j) (((i) - c->ids) + (long)n * ((j) - 1))
  int iPatch = 1, gPatch = 5;
  for (int j = c->jde + 1; j <= c->jpe; j++)
    for (int i = c->ids; i <= c->ide; i++) {
      int ihalo = j - c->jde;
      double lambda, theta;
      long k = PIX(c, i, j, iPatch);
      pointProjPlane2Sphere(c, &lambda, &theta, c->xP[k], c->yP[k], iPatch);
      pointProjSphere2Plane(c, &c->gX[GIX(i, ihalo)], &c->gY[GIX(i, ihalo)], lambda, theta, gPatch);
    }
  double *X_RAW = malloc(sizeof(double) * (c->Nx + 2));
  for (int i = 1; i <= c->Nx + 1; i++) X_RAW[i] = c->xP[PIX(c, PVIDX(c, 1, i), 1, iPatch)];
  for (int j = 1; j <= H; j++) {
    int iref = 1;
    for (int i = c->ids; i <= c->ide; i++) {
      while (c->gX[GIX(i, j)] > X_RAW[iref]) {
        iref = iref + 1;
        if (iref > c->Nx + 1) { free(X_RAW); return -3; }
      }
      if (iref >= 2 && c->gX[GIX(i, j)] >= X_RAW[iref - 1] && c->gX[GIX(i, j)] <= X_RAW[iref]) {
        c->gCoef[GIX(i, j)] = c->gX[GIX(i, j)] - X_RAW[iref - 1];
        c->gIref[GIX(i, j)] = iref - 1;
      } else {
        free(X_RAW);
        return -3; /* 'Ghost cell location error' */
      }
    }
  }
#undef GIX
  free(X_RAW);
  return 0;
}

/* ------------------------------------------------------------------ */
/* stat_mod.F90 / tend_mod.F90                                         */
/* ------------------------------------------------------------------ */
static void alloc_stat(orc_ctx *c, orc_stat *s) {
  long NP = c->NP;
  s->u = calloc(NP, 8); s->v = calloc(NP, 8); s->phi = calloc(NP, 8); s->phiG = calloc(NP, 8);
  s->contraU = calloc(NP, 8); s->contraV = calloc(NP, 8);
  s->zonal_wind = calloc(NP, 8); s->meridional_wind = calloc(NP, 8);
}
static void free_stat(orc_stat *s) {
  free(s->u); free(s->v); free(s->phi); free(s->phiG); free(s->contraU); free(s->contraV);
  free(s->zonal_wind); free(s->meridional_wind);
}

/* stat_mod.F90:47-59 (copyStat) and :61-73 (switch_stat) copy the same 8 fields */
static void copy_stat(const orc_ctx *c, orc_stat *out, const orc_stat *in) {
  size_t b = (size_t)c->NP * 8;
  memcpy(out->u, in->u, b); memcpy(out->v, in->v, b); memcpy(out->phi, in->phi, b); memcpy(out->phiG, in->phiG, b);
  memcpy(out->contraU, in->contraU, b); memcpy(out->contraV, in->contraV, b);
  memcpy(out->zonal_wind, in->zonal_wind, b); memcpy(out->meridional_wind, in->meridional_wind, b);
}

/* ------------------------------------------------------------------ */
/* spatial_operators_mod.F90                                           */
/* ------------------------------------------------------------------ */

/* :204-218 */
static double polyfitL(int DOF, const double *pv, double dh) {
  if (DOF == 3) return -(pv[2] - 4. * pv[1] + 3. * pv[0]) / dh;
  return (-(11. * pv[0]) + 18. * pv[1] - 9. * pv[2] + 2. * pv[3]) / (2. * dh);
}
/* :220-234 */
static double polyfitR(int DOF, const double *pv, double dh) {
  if (DOF == 3) return (pv[0] - 4. * pv[1] + 3. * pv[2]) / dh;
  return (11. * pv[3] - 18. * pv[2] + 9. * pv[1] - 2. * pv[0]) / (2. * dh);
}
/* :236-246 */
static double riemann_solver(double fxL, double fxR, double qxL, double qxR, double eigenvalue) {
  return 0.5 * ((fxL + fxR) - eigenvalue * (qxR - qxL));
}
/* :248-263 (and :265-280 with G22) */
static double eigenvalue_1d(double contra, double phi, double Gii) {
  double l1 = contra - sqrt(Gii * phi);
  double l2 = contra + sqrt(Gii * phi);
  return fmax(fabs(l1), fabs(l2));
}

/* :136-202; f and q hold the 3*DOF-2 window values */
static void calc_tendP(const orc_ctx *c, double *derivP, const double *f, const double *q, double eL, double eR) {
  int DOF = c->DOF;
  double fCell[3][4], qCell[3][4];
  for (int iCell = 1; iCell <= 3; iCell++)
    for (int d = 1; d <= DOF; d++) {
      int k = (iCell - 1) * (DOF - 1) + d; /* pvIdx(d, iCell) inside the window */
      fCell[iCell - 1][d - 1] = f[k - 1];
      qCell[iCell - 1][d - 1] = q[k - 1];
    }
  double dx = c->dx;
  double fxL1 = polyfitR(DOF, fCell[0], dx), fxL2 = polyfitR(DOF, fCell[1], dx);
  double fxR1 = polyfitL(DOF, fCell[1], dx), fxR2 = polyfitL(DOF, fCell[2], dx);
  double qxL1 = polyfitR(DOF, qCell[0], dx), qxL2 = polyfitR(DOF, qCell[1], dx);
  double qxR1 = polyfitL(DOF, qCell[1], dx), qxR2 = polyfitL(DOF, qCell[2], dx);
  derivP[0] = riemann_solver(fxL1, fxR1, qxL1, qxR1, eL);
  derivP[DOF - 1] = riemann_solver(fxL2, fxR2, qxL2, qxR2, eR);
  if (DOF == 3) {
    double f1 = fCell[1][0], f3 = fCell[1][2];
    double fxVIA = (f3 - f1) / dx;
    derivP[1] = 1.5 * fxVIA - 0.25 * (derivP[0] + derivP[DOF - 1]);
  } else {
    double f1 = fCell[1][0], f2 = fCell[1][1], f3 = fCell[1][2], f4 = fCell[1][3];
    double fxVIA = (f4 - f1) / dx;
    double fxxc = 4.5 * (f1 - f2 - f3 + f4) / (dx * dx);
    derivP[1] = 4. / 3. * fxVIA - (4. * derivP[0] + 5. * derivP[DOF - 1]) / 27. - 4. / 27. * dx * fxxc;
    derivP[2] = 4. / 3. * fxVIA - (5. * derivP[0] + 4. * derivP[DOF - 1]) / 27. + 4. / 27. * dx * fxxc;
  }
}

/* :12-133 */
static void spatial_operator(orc_ctx *c, const orc_stat *s, orc_tend *t) {
  int DOF = c->DOF, W = 3 * DOF - 2;
  long NP = c->NP;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < NP; k++) {
    c->phiGu[k] = s->phiG[k] * s->contraU[k];
    c->phiGv[k] = s->phiG[k] * s->contraV[k];
    c->K[k] = 0.5 * (s->contraU[k] * s->u[k] + s->contraV[k] * s->v[k]);
    c->E[k] = s->phi[k] + c->phi_s[k] + c->K[k];
  }
  /* x direction, :63-93 */
  for (int iPatch = 1; iPatch <= 6; iPatch++) {
#pragma omp parallel for schedule(static)
    for (int j = c->jds; j <= c->jde; j++) {
      double Ex[10], ux[10], vx[10], cUx[10], phiGux[10], phiGx[10], dP[4];
      for (int i = c->its; i <= c->ite; i++) {
        int Pl = PVIDX(c, 1, i), Pr = PVIDX(c, DOF, i);
        int Ps = Pl - DOF + 1;
        for (int w = 0; w < W; w++) {
          long k = PIX(c, Ps + w, j, iPatch);
          Ex[w] = c->E[k]; ux[w] = s->u[k]; vx[w] = s->v[k];
          cUx[w] = s->contraU[k]; phiGux[w] = c->phiGu[k]; phiGx[w] = s->phiG[k];
        }
        double lamL = eigenvalue_1d(s->contraU[PIX(c, Pl, j, iPatch)], s->phi[PIX(c, Pl, j, iPatch)],
                                    c->matrixIG[MIX(c, 1, 1, Pl, j, iPatch)]);
        double lamR = eigenvalue_1d(s->contraU[PIX(c, Pr, j, iPatch)], s->phi[PIX(c, Pr, j, iPatch)],
                                    c->matrixIG[MIX(c, 1, 1, Pr, j, iPatch)]);
        for (int w = 0; w < W; w++)
          if (cUx[w] == 0) cUx[w] = 1.;
        double upL = cUx[DOF - 1] / fabs(cUx[DOF - 1]);
        double upR = cUx[2 * DOF - 2] / fabs(cUx[2 * DOF - 2]);
        calc_tendP(c, dP, Ex, ux, lamL, lamR);
        for (int d = 0; d < DOF; d++) c->flux_x[IIX(c, Pl + d, j, iPatch)] = dP[d];
        calc_tendP(c, dP, phiGux, phiGx, lamL, lamR);
        for (int d = 0; d < DOF; d++) c->div_x[IIX(c, Pl + d, j, iPatch)] = dP[d];
        calc_tendP(c, dP, vx, vx, upL, upR);
        for (int d = 0; d < DOF; d++) c->dvdx[IIX(c, Pl + d, j, iPatch)] = dP[d];
      }
    }
  }
  /* y direction, :95-125 */
  for (int iPatch = 1; iPatch <= 6; iPatch++) {
#pragma omp parallel for schedule(static)
    for (int i = c->ids; i <= c->ide; i++) {
      double Ey[10], uy[10], vy[10], cVy[10], phiGvy[10], phiGy[10], dP[4];
      for (int j = c->jts; j <= c->jte; j++) {
        int Pl = PVIDX(c, 1, j), Pr = PVIDX(c, DOF, j);
        int Ps = Pl - DOF + 1;
        for (int w = 0; w < W; w++) {
          long k = PIX(c, i, Ps + w, iPatch);
          Ey[w] = c->E[k]; uy[w] = s->u[k]; vy[w] = s->v[k];
          cVy[w] = s->contraV[k]; phiGvy[w] = c->phiGv[k]; phiGy[w] = s->phiG[k];
        }
        double lamL = eigenvalue_1d(s->contraV[PIX(c, i, Pl, iPatch)], s->phi[PIX(c, i, Pl, iPatch)],
                                    c->matrixIG[MIX(c, 2, 2, i, Pl, iPatch)]);
        double lamR = eigenvalue_1d(s->contraV[PIX(c, i, Pr, iPatch)], s->phi[PIX(c, i, Pr, iPatch)],
                                    c->matrixIG[MIX(c, 2, 2, i, Pr, iPatch)]);
        for (int w = 0; w < W; w++)
          if (cVy[w] == 0) cVy[w] = 1.;
        double upL = cVy[DOF - 1] / fabs(cVy[DOF - 1]);
        double upR = cVy[2 * DOF - 2] / fabs(cVy[2 * DOF - 2]);
        calc_tendP(c, dP, Ey, vy, lamL, lamR);
        for (int d = 0; d < DOF; d++) c->flux_y[IIX(c, i, Pl + d, iPatch)] = dP[d];
        calc_tendP(c, dP, phiGvy, phiGy, lamL, lamR);
        for (int d = 0; d < DOF; d++) c->div_y[IIX(c, i, Pl + d, iPatch)] = dP[d];
        calc_tendP(c, dP, uy, uy, upL, upR);
        for (int d = 0; d < DOF; d++) c->dudy[IIX(c, i, Pl + d, iPatch)] = dP[d];
      }
    }
  }
  /* :127-131 */
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 1; p <= 6; p++)
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ide; i++) {
        long ii = IIX(c, i, j, p), pk = PIX(c, i, j, p);
        double sG = c->sqrtG[pk];
        double vort = (c->dvdx[ii] - c->dudy[ii]) / sG;
        c->vort[ii] = vort;
        t->phiG[ii] = -c->div_x[ii] - c->div_y[ii];
        t->u[ii] = -c->flux_x[ii] + sG * (vort + c->f[pk]) * s->contraV[pk];
        t->v[ii] = -c->flux_y[ii] - sG * (vort + c->f[pk]) * s->contraU[pk];
      }
}

/* :291-388; field holds a full padded array, only (ids:ide, jds:jde) is touched */
static void unify_bdy_field(orc_ctx *c, double *field) {
  int ids = c->ids, ide = c->ide, jds = c->jds, jde = c->jde, n = c->nPVx;
  double *raw = c->field_raw; /* field_raw = field over the interior */
  for (int p = 1; p <= 6; p++)
    for (int j = jds; j <= jde; j++)
      for (int i = ids; i <= ide; i++) raw[IIX(c, i, j, p)] = field[PIX(c, i, j, p)];
#define F(i, j, p) field[PIX(c, i, j, p)]
#define R(i, j, p) raw[IIX(c, i, j, p)]
  for (int k = 1; k <= n; k++) { /* edge(1,4) */
    F(ids, k, 1) = 0.5 * (R(ide, k, 4) + R(ids, k, 1));
    F(ide, k, 4) = F(ids, k, 1);
  }
  for (int k = 1; k <= n; k++) { /* edge(1,2) */
    F(ids, k, 2) = 0.5 * (R(ide, k, 1) + R(ids, k, 2));
    F(ide, k, 1) = F(ids, k, 2);
  }
  for (int k = 1; k <= n; k++) { /* edge(2,3) */
    F(ids, k, 3) = 0.5 * (R(ide, k, 2) + R(ids, k, 3));
    F(ide, k, 2) = F(ids, k, 3);
  }
  for (int k = 1; k <= n; k++) { /* edge(3,4) */
    F(ids, k, 4) = 0.5 * (R(ide, k, 3) + R(ids, k, 4));
    F(ide, k, 3) = F(ids, k, 4);
  }
  for (int k = 1; k <= n; k++) { /* edge(1,5) */
    F(k, jde, 1) = 0.5 * (R(k, jds, 5) + R(k, jde, 1));
    F(k, jds, 5) = F(k, jde, 1);
  }
  for (int k = 1; k <= n; k++) { /* edge(1,6) */
    F(k, jds, 1) = 0.5 * (R(k, jds, 1) + R(k, jde, 6));
    F(k, jde, 6) = F(k, jds, 1);
  }
  for (int k = 1; k <= n; k++) { /* edge(2,5) */
    F(k, jde, 2) = 0.5 * (R(ide, k, 5) + R(k, jde, 2));
    F(ide, k, 5) = F(k, jde, 2);
  }
  for (int k = 1; k <= n; k++) { /* edge(2,6): field_raw(ide, jde:jds:-1, 6) */
    F(k, jds, 2) = 0.5 * (R(k, jds, 2) + R(ide, n + 1 - k, 6));
    F(ide, n + 1 - k, 6) = F(k, jds, 2);
  }
  for (int k = 1; k <= n; k++) { /* edge(3,5): field_raw(ide:ids:-1, jde, 5) */
    F(k, jde, 3) = 0.5 * (R(k, jde, 3) + R(n + 1 - k, jde, 5));
    F(n + 1 - k, jde, 5) = F(k, jde, 3);
  }
  for (int k = 1; k <= n; k++) { /* edge(3,6): field_raw(ide:ids:-1, jds, 6) */
    F(k, jds, 3) = 0.5 * (R(k, jds, 3) + R(n + 1 - k, jds, 6));
    F(n + 1 - k, jds, 6) = F(k, jds, 3);
  }
  for (int k = 1; k <= n; k++) { /* edge(4,5): field_raw(ids, jde:jds:-1, 5) */
    F(k, jde, 4) = 0.5 * (R(k, jde, 4) + R(ids, n + 1 - k, 5));
    F(ids, n + 1 - k, 5) = F(k, jde, 4);
  }
  for (int k = 1; k <= n; k++) { /* edge(4,6) */
    F(k, jds, 4) = 0.5 * (R(k, jds, 4) + R(ids, k, 6));
    F(ids, k, 6) = F(k, jds, 4);
  }
  /* vertex points, :347-386 */
  F(ids, jde, 1) = (R(ids, jde, 1) + R(ide, jde, 4) + R(ids, jds, 5)) / 3.;
  F(ids, jds, 5) = F(ids, jde, 1); F(ide, jde, 4) = F(ids, jde, 1);
  F(ide, jde, 1) = (R(ide, jde, 1) + R(ids, jde, 2) + R(ide, jds, 5)) / 3.;
  F(ids, jde, 2) = F(ide, jde, 1); F(ide, jds, 5) = F(ide, jde, 1);
  F(ids, jds, 1) = (R(ids, jds, 1) + R(ide, jds, 4) + R(ids, jde, 6)) / 3.;
  F(ide, jds, 4) = F(ids, jds, 1); F(ids, jde, 6) = F(ids, jds, 1);
  F(ide, jds, 1) = (R(ide, jds, 1) + R(ids, jds, 2) + R(ide, jde, 6)) / 3.;
  F(ids, jds, 2) = F(ide, jds, 1); F(ide, jde, 6) = F(ide, jds, 1);
  F(ids, jde, 3) = (R(ids, jde, 3) + R(ide, jde, 2) + R(ide, jde, 5)) / 3.;
  F(ide, jde, 2) = F(ids, jde, 3); F(ide, jde, 5) = F(ids, jde, 3);
  F(ide, jde, 3) = (R(ide, jde, 3) + R(ids, jde, 4) + R(ids, jde, 5)) / 3.;
  F(ids, jde, 4) = F(ide, jde, 3); F(ids, jde, 5) = F(ide, jde, 3);
  F(ids, jds, 3) = (R(ide, jds, 2) + R(ids, jds, 3) + R(ide, jds, 6)) / 3.;
  F(ide, jds, 2) = F(ids, jds, 3); F(ide, jds, 6) = F(ids, jds, 3);
  F(ide, jds, 3) = (R(ide, jds, 3) + R(ids, jds, 4) + R(ids, jds, 6)) / 3.;
  F(ids, jds, 4) = F(ide, jds, 3); F(ids, jds, 6) = F(ide, jds, 3);
#undef F
#undef R
}

/* :282-289 */
static void unify_bdy_stat(orc_ctx *c, orc_stat *s) {
  unify_bdy_field(c, s->phi);
  unify_bdy_field(c, s->zonal_wind);
  unify_bdy_field(c, s->meridional_wind);
}

static void p2sp_point(orc_ctx *c, orc_stat *s, int i, int j, int p) {
  long k = PIX(c, i, j, p);
  covProjPlane2Sphere(&s->zonal_wind[k], &s->meridional_wind[k], s->u[k], s->v[k], &c->matrixA[4 * k],
                      &c->matrixIG[4 * k]);
}
static void sp2p_point(orc_ctx *c, orc_stat *s, int i, int j, int p) {
  long k = PIX(c, i, j, p);
  covProjSphere2Plane(&s->u[k], &s->v[k], s->zonal_wind[k], s->meridional_wind[k], &c->matrixIA[4 * k],
                      &c->matrixG[4 * k]);
}

/* :391-405 */
static void convert_wind_P2SP(orc_ctx *c, orc_stat *s) {
#pragma omp parallel for schedule(static)
  for (int p = 1; p <= 6; p++)
    for (int j = c->jps; j <= c->jpe; j++)
      for (int i = c->ips; i <= c->ipe; i++) p2sp_point(c, s, i, j, p);
}

/* :408-441 */
static void convert_ghost_wind_P2SP(orc_ctx *c, orc_stat *s) {
  int H = c->nPVHalo;
#pragma omp parallel for schedule(static)
  for (int p = 1; p <= 6; p++) {
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ids + H; i++) p2sp_point(c, s, i, j, p);
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ide - H; i <= c->ide; i++) p2sp_point(c, s, i, j, p);
    for (int j = c->jde - H; j <= c->jde; j++)
      for (int i = c->ids + H; i <= c->ide - H; i++) p2sp_point(c, s, i, j, p);
    for (int j = c->jds; j <= c->jds + H; j++)
      for (int i = c->ids + H; i <= c->ide - H; i++) p2sp_point(c, s, i, j, p);
  }
}

/* :459-492 */
static void convert_ghost_wind_SP2P(orc_ctx *c, orc_stat *s) {
#pragma omp parallel for schedule(static)
  for (int p = 1; p <= 6; p++) {
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ips; i <= c->ids; i++) sp2p_point(c, s, i, j, p);
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ide; i <= c->ipe; i++) sp2p_point(c, s, i, j, p);
    for (int j = c->jde; j <= c->jpe; j++)
      for (int i = c->ids; i <= c->ide; i++) sp2p_point(c, s, i, j, p);
    for (int j = c->jps; j <= c->jds; j++)
      for (int i = c->ids; i <= c->ide; i++) sp2p_point(c, s, i, j, p);
  }
}

/* :494-508 */
static void convert_wind_cov2contrav(orc_ctx *c, orc_stat *s) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < c->NP; k++) cov2contrav(&s->contraU[k], &s->contraV[k], s->u[k], s->v[k], &c->matrixIG[4 * k]);
}

/* ------------------------------------------------------------------ */
/* ghost_mod.f90:88-237                                                */
/* ------------------------------------------------------------------ */
static void CubedSphereFillHalo(orc_ctx *c, double *field) {
  int ids = c->ids, ide = c->ide, jds = c->jds, jde = c->jde, n = c->nPVx, H = c->nPVHalo;
  double *in = c->field_inner;
  for (int p = 1; p <= 6; p++)
    for (int j = jds; j <= jde; j++)
      for (int i = ids; i <= ide; i++) in[IIX(c, i, j, p)] = field[PIX(c, i, j, p)];
#define F(i, j, p) field[PIX(c, i, j, p)]
#define IN(i, j, p) in[IIX(c, i, j, p)]
  for (int h = 1; h <= H; h++)
    for (int k = 1; k <= n; k++) {
      /* panel 1 */
      F(1 - h, k, 1) = IN(ide - h, k, 4);
      F(ide + h, k, 1) = IN(h + 1, k, 2);
      F(k, 1 - h, 1) = IN(k, jde - h, 6);
      F(k, jde + h, 1) = IN(k, h + 1, 5);
      /* panel 2 */
      F(1 - h, k, 2) = IN(ide - h, k, 1);
      F(ide + h, k, 2) = IN(h + 1, k, 3);
      F(k, 1 - h, 2) = IN(ide - h, jde + 1 - k, 6);
      F(k, jde + h, 2) = IN(ide - h, k, 5);
      /* panel 3 */
      F(1 - h, k, 3) = IN(ide - h, k, 2);
      F(ide + h, k, 3) = IN(h + 1, k, 4);
      F(k, 1 - h, 3) = IN(ide + 1 - k, h + 1, 6);
      F(k, jde + h, 3) = IN(ide + 1 - k, jde - h, 5);
      /* panel 4 */
      F(1 - h, k, 4) = IN(ide - h, k, 3);
      F(ide + h, k, 4) = IN(h + 1, k, 1);
      F(k, 1 - h, 4) = IN(h + 1, k, 6);
      F(k, jde + h, 4) = IN(h + 1, jde + 1 - k, 5);
      /* panel 5 */
      F(1 - h, k, 5) = IN(ide + 1 - k, jde - h, 4);
      F(ide + h, k, 5) = IN(k, jde - h, 2);
      F(k, 1 - h, 5) = IN(k, jde - h, 1);
      F(k, jde + h, 5) = IN(ide + 1 - k, jde - h, 3);
      /* panel 6 */
      F(1 - h, k, 6) = IN(k, h + 1, 4);
      F(ide + h, k, 6) = IN(ide + 1 - k, h + 1, 2);
      F(k, 1 - h, 6) = IN(ide + 1 - k, h + 1, 3);
      F(k, jde + h, 6) = IN(k, h + 1, 1);
    }
  (void)jds;
#undef F
#undef IN
}

/* :183-227; src and dest are strided views of n points */
static void linear_interp(const orc_ctx *c, double *dest, long dstride, const double *src, long sstride, int h) {
  int n = c->nPVx;
  double dx = c->dx;
  for (int i = 1; i <= n; i++) {
    int iref = c->gIref[(i - 1) + (long)n * (h - 1)];
    double coef = c->gCoef[(i - 1) + (long)n * (h - 1)];
    if (c->DOF == 3) {
      double q1 = src[(PVIDX(c, 1, iref) - 1) * sstride];
      double q2 = src[(PVIDX(c, 2, iref) - 1) * sstride];
      double q3 = src[(PVIDX(c, 3, iref) - 1) * sstride];
      dest[(i - 1) * dstride] =
          q1 - (3. * q1 - 4. * q2 + q3) * coef / dx + 2. * (q1 - 2. * q2 + q3) * sq(coef) / sq(dx);
    } else {
      double q1 = src[(PVIDX(c, 1, iref) - 1) * sstride];
      double q2 = src[(PVIDX(c, 2, iref) - 1) * sstride];
      double q3 = src[(PVIDX(c, 3, iref) - 1) * sstride];
      double q4 = src[(PVIDX(c, 4, iref) - 1) * sstride];
      dest[(i - 1) * dstride] =
          (2. * pow(dx, 3.) * q1 + pow(dx, 2.) * (-(11. * q1) + 18. * q2 - 9. * q3 + 2. * q4) * coef +
           9. * dx * (2. * q1 - 5. * q2 + 4. * q3 - q4) * pow(coef, 2.) +
           9. * (-q1 + 3. * q2 - 3. * q3 + q4) * pow(coef, 3.)) /
          (2. * pow(dx, 3.));
    }
  }
}

/* :154-181 */
static void CubedSphereFillGhost(orc_ctx *c, double *field) {
  double *gt = c->ghost_target;
  long NP = c->NP;
  for (long k = 0; k < NP; k++) gt[k] = FILLVALUE;
  for (int p = 1; p <= 6; p++)
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ide; i++) gt[PIX(c, i, j, p)] = field[PIX(c, i, j, p)];
  CubedSphereFillHalo(c, field);
  long sx = 1, sy = c->npx;
  for (int p = 1; p <= 6; p++)
    for (int h = 1; h <= c->nPVHalo; h++) {
      linear_interp(c, &gt[PIX(c, c->ids - h, c->jds, p)], sy, &field[PIX(c, c->ids - h, c->jds, p)], sy, h);
      linear_interp(c, &gt[PIX(c, c->ide + h, c->jds, p)], sy, &field[PIX(c, c->ide + h, c->jds, p)], sy, h);
      linear_interp(c, &gt[PIX(c, c->ids, c->jde + h, p)], sx, &field[PIX(c, c->ids, c->jde + h, p)], sx, h);
      linear_interp(c, &gt[PIX(c, c->ids, c->jds - h, p)], sx, &field[PIX(c, c->ids, c->jds - h, p)], sx, h);
    }
  memcpy(field, gt, (size_t)NP * 8);
}

/* :230-237 */
static void fill_ghost(orc_ctx *c, orc_stat *s) {
  CubedSphereFillGhost(c, s->phi);
  CubedSphereFillGhost(c, s->zonal_wind);
  CubedSphereFillGhost(c, s->meridional_wind);
}

/* ------------------------------------------------------------------ */
/* time_scheme_mod.F90                                                 */
/* ------------------------------------------------------------------ */

/* :125-142 (scheme 2) */
static void correct_bdy_ghost(orc_ctx *c, orc_stat *s) {
  convert_ghost_wind_P2SP(c, s);
  fill_ghost(c, s);
  unify_bdy_stat(c, s);
  convert_ghost_wind_SP2P(c, s);
  convert_wind_cov2contrav(c, s);
}

static void phi_from_phiG(orc_ctx *c, orc_stat *s) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < c->NP; k++) s->phi[k] = s->phiG[k] / c->sqrtG[k];
}
static void phiG_from_phi(orc_ctx *c, orc_stat *s) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < c->NP; k++) s->phiG[k] = s->phi[k] * c->sqrtG[k];
}

/* :71-87 */
static void update_stat(orc_ctx *c, orc_stat *sn, const orc_stat *so, const orc_tend *t, double inc_t) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 1; p <= 6; p++)
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ide; i++) {
        long k = PIX(c, i, j, p), ii = IIX(c, i, j, p);
        sn->phiG[k] = so->phiG[k] + inc_t * t->phiG[ii];
        sn->u[k] = so->u[k] + inc_t * t->u[ii];
        sn->v[k] = so->v[k] + inc_t * t->v[ii];
      }
  phi_from_phiG(c, sn);
  correct_bdy_ghost(c, sn);
  phiG_from_phi(c, sn);
}

/* :89-105 */
static void update_stat_RK3_TVD_1(orc_ctx *c, orc_stat *sn, const orc_stat *so, const orc_stat *s1, const orc_tend *t) {
  double dt = c->dt;
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 1; p <= 6; p++)
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ide; i++) {
        long k = PIX(c, i, j, p), ii = IIX(c, i, j, p);
        sn->phiG[k] = 0.75 * so->phiG[k] + 0.25 * s1->phiG[k] + 0.25 * dt * t->phiG[ii];
        sn->u[k] = 0.75 * so->u[k] + 0.25 * s1->u[k] + 0.25 * dt * t->u[ii];
        sn->v[k] = 0.75 * so->v[k] + 0.25 * s1->v[k] + 0.25 * dt * t->v[ii];
      }
  phi_from_phiG(c, sn);
  correct_bdy_ghost(c, sn);
  phiG_from_phi(c, sn);
}

/* :107-123 */
static void update_stat_RK3_TVD_2(orc_ctx *c, orc_stat *sn, const orc_stat *so, const orc_stat *s2, const orc_tend *t) {
  double dt = c->dt;
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 1; p <= 6; p++)
    for (int j = c->jds; j <= c->jde; j++)
      for (int i = c->ids; i <= c->ide; i++) {
        long k = PIX(c, i, j, p), ii = IIX(c, i, j, p);
        sn->phiG[k] = so->phiG[k] / 3. + 2. / 3. * s2->phiG[k] + 2. / 3. * dt * t->phiG[ii];
        sn->u[k] = so->u[k] / 3. + 2. / 3. * s2->u[k] + 2. / 3. * dt * t->u[ii];
        sn->v[k] = so->v[k] / 3. + 2. / 3. * s2->v[k] + 2. / 3. * dt * t->v[ii];
      }
  phi_from_phiG(c, sn);
  correct_bdy_ghost(c, sn);
  phiG_from_phi(c, sn);
}

/* :13-44 */
static void RK4(orc_ctx *c, orc_stat *snew, orc_stat *sold) {
  orc_stat *one = &c->stat[SLOT(c, -1)], *two = &c->stat[SLOT(c, -2)], *three = &c->stat[SLOT(c, -3)],
           *four = &c->stat[SLOT(c, -4)];
  orc_tend *t1 = &c->tend[SLOT(c, -1)], *t2 = &c->tend[SLOT(c, -2)], *t3 = &c->tend[SLOT(c, -3)],
           *t4 = &c->tend[SLOT(c, -4)], *tn = &c->tend[SLOT(c, 1)];
  double dt = c->dt;
  copy_stat(c, one, sold);
  spatial_operator(c, one, t1);
  update_stat(c, two, one, t1, 0.5 * dt);
  spatial_operator(c, two, t2);
  update_stat(c, three, one, t2, 0.5 * dt);
  spatial_operator(c, three, t3);
  update_stat(c, four, one, t3, dt);
  spatial_operator(c, four, t4);
  long NI = (long)c->nPVx * c->nPVy * 6;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < NI; k++) {
    tn->phiG[k] = (t1->phiG[k] + 2. * t2->phiG[k] + 2. * t3->phiG[k] + t4->phiG[k]) / 6.;
    tn->u[k] = (t1->u[k] + 2. * t2->u[k] + 2. * t3->u[k] + t4->u[k]) / 6.;
    tn->v[k] = (t1->v[k] + 2. * t2->v[k] + 2. * t3->v[k] + t4->v[k]) / 6.;
  }
  update_stat(c, snew, sold, tn, dt);
}

/* :46-69 */
static void RK3_TVD(orc_ctx *c, orc_stat *snew, orc_stat *sold) {
  orc_stat *one = &c->stat[SLOT(c, -1)], *two = &c->stat[SLOT(c, -2)], *three = &c->stat[SLOT(c, -3)];
  orc_tend *t1 = &c->tend[SLOT(c, -1)], *t2 = &c->tend[SLOT(c, -2)], *t3 = &c->tend[SLOT(c, -3)];
  copy_stat(c, one, sold);
  spatial_operator(c, one, t1);
  update_stat(c, two, one, t1, c->dt);
  spatial_operator(c, two, t2);
  update_stat_RK3_TVD_1(c, three, one, two, t2);
  spatial_operator(c, three, t3);
  update_stat_RK3_TVD_2(c, snew, one, three, t3);
}

/* ------------------------------------------------------------------ */
/* diag_mod.F90:10-93                                                  */
/* ------------------------------------------------------------------ */
static double calc_total_mass(const orc_ctx *c, const orc_stat *s) {
  int DOF = c->DOF, Nx = c->Nx, Ny = c->Ny;
  double *mc = calloc((size_t)Nx * Ny * 6, 8);
  for (int p = 1; p <= 6; p++)
    for (int jC = 1; jC <= Ny; jC++)
      for (int iC = 1; iC <= Nx; iC++)
        for (int jD = 1; jD <= DOF; jD++)
          for (int iD = 1; iD <= DOF; iD++) {
            int iPV = PVIDX(c, iD, iC), jPV = PVIDX(c, jD, jC);
            long m = (iC - 1) + (long)Nx * ((jC - 1) + (long)Ny * (p - 1));
            mc[m] = mc[m] + c->weightsOnPV[iD - 1][jD - 1] * s->phiG[PIX(c, iPV, jPV, p)];
          }
  double total = 0.;
  for (long m = 0; m < (long)Nx * Ny * 6; m++) total = total + mc[m];
  free(mc);
  return total;
}

static double calc_total_energy(const orc_ctx *c, const orc_stat *s) {
  int DOF = c->DOF, Nx = c->Nx, Ny = c->Ny;
  double *ec = calloc((size_t)Nx * Ny * 6, 8);
  for (int p = 1; p <= 6; p++)
    for (int jC = 1; jC <= Ny; jC++)
      for (int iC = 1; iC <= Nx; iC++)
        for (int jD = 1; jD <= DOF; jD++)
          for (int iD = 1; iD <= DOF; iD++) {
            int iPV = PVIDX(c, iD, iC), jPV = PVIDX(c, jD, jC);
            long k = PIX(c, iPV, jPV, p);
            double KE = 0.5 * s->phi[k] * (s->u[k] * s->contraU[k] + s->v[k] * s->contraV[k]);
            double PE = 0.5 * sq(s->phi[k] + c->phi_s[k]);
            long m = (iC - 1) + (long)Nx * ((jC - 1) + (long)Ny * (p - 1));
            ec[m] = ec[m] + c->weightsOnPV[iD - 1][jD - 1] * c->sqrtG[k] * (KE + PE);
          }
  double total = 0.;
  for (long m = 0; m < (long)Nx * Ny * 6; m++) total = total + ec[m];
  free(ec);
  return total;
}

/* diag_mod.F90:69-93; out has (ics:ice, jcs:jce, 6) layout */
static void calc_VIA(const orc_ctx *c, double *out, const double *field) {
  int DOF = c->DOF;
  memset(out, 0, sizeof(double) * c->ncx * c->ncy * 6);
  for (int p = 1; p <= 6; p++)
    for (int jC = 1; jC <= c->Ny; jC++)
      for (int iC = 1; iC <= c->Nx; iC++)
        for (int jD = 1; jD <= DOF; jD++)
          for (int iD = 1; iD <= DOF; iD++) {
            int iPV = PVIDX(c, iD, iC), jPV = PVIDX(c, jD, jC);
            long m = CIX(c, iC, jC, p);
            out[m] = out[m] + c->weightsOnPV[iD - 1][jD - 1] * field[PIX(c, iPV, jPV, p)];
          }
}

/* ================================================================== */
/* Exported C interface (ctypes).                                      */
/* ================================================================== */

orc_ctx *orc_create(int dof, double dx_deg, double dt, int scheme, double radius, int *status) {
  orc_ctx *c = calloc(1, sizeof(orc_ctx));
  int rc = init_parameters(c, dof, dx_deg, dt, scheme, radius);
  if (rc != 0) { free(c); *status = rc; return NULL; }
  init_mesh(c);
  rc = init_ghost(c);
  if (rc != 0) { *status = rc; return c; }
  for (int t = -c->nsub; t <= 1; t++) {
    alloc_stat(c, &c->stat[SLOT(c, t)]);
    long NI = (long)c->nPVx * c->nPVy * 6;
    c->tend[SLOT(c, t)].u = calloc(NI, 8);
    c->tend[SLOT(c, t)].v = calloc(NI, 8);
    c->tend[SLOT(c, t)].phiG = calloc(NI, 8);
  }
  long NI = (long)c->nPVx * c->nPVy * 6, NP = c->NP;
  c->flux_x = calloc(NI, 8); c->flux_y = calloc(NI, 8); c->div_x = calloc(NI, 8); c->div_y = calloc(NI, 8);
  c->dvdx = calloc(NI, 8); c->dudy = calloc(NI, 8); c->vort = calloc(NI, 8);
  c->K = calloc(NP, 8); c->E = calloc(NP, 8); c->phiGu = calloc(NP, 8); c->phiGv = calloc(NP, 8);
  c->ghost_target = calloc(NP, 8); c->field_inner = calloc(NI, 8); c->field_raw = calloc(NI, 8);
  c->old_slot = SLOT(c, 0);
  c->new_slot = SLOT(c, 1);
  *status = 0;
  return c;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  double *arr[] = {c->xP, c->yP, c->lonP, c->latP, c->sqrtG, c->f, c->phi_s, c->matrixG, c->matrixIG, c->matrixA,
                   c->matrixIA, c->areaCell, c->gX, c->gY, c->gCoef, c->flux_x, c->flux_y, c->div_x, c->div_y,
                   c->dvdx, c->dudy, c->vort, c->K, c->E, c->phiGu, c->phiGv, c->ghost_target, c->field_inner,
                   c->field_raw};
  for (size_t k = 0; k < sizeof(arr) / sizeof(arr[0]); k++) free(arr[k]);
  free(c->pvIdx); free(c->gIref);
  if (c->stat[SLOT(c, 1)].u)
    for (int t = -c->nsub; t <= 1; t++) {
      free_stat(&c->stat[SLOT(c, t)]);
      free(c->tend[SLOT(c, t)].u); free(c->tend[SLOT(c, t)].v); free(c->tend[SLOT(c, t)].phiG);
    }
  free(c);
}

/* sizes: [nPVx, nPVHalo, npx(padded), Nx, ncx(padded cells)] */
void orc_sizes(const orc_ctx *c, int *out) {
  out[0] = c->nPVx; out[1] = c->nPVHalo; out[2] = (int)c->npx; out[3] = c->Nx; out[4] = (int)c->ncx;
}
double orc_dx(const orc_ctx *c) { return c->dx; }
/* the time step (namelist dt, parameters_mod.F90:116) of an existing instance */
void orc_set_dt(orc_ctx *c, double dt) { c->dt = dt; }

/* Copy a mesh array out.  which: 0 xP,1 yP,2 lonP,3 latP,4 sqrtG,5 f,6 phi_s,
   7 matrixG,8 matrixIG,9 matrixA,10 matrixIA (4*NP), 11 areaCell (cells), 12 ghost coef (n*H),
   13 ghost X (n*H) */
int orc_get_mesh(const orc_ctx *c, int which, double *out) {
  long NP = c->NP;
  const double *src[] = {c->xP, c->yP, c->lonP, c->latP, c->sqrtG, c->f, c->phi_s};
  if (which >= 0 && which <= 6) { memcpy(out, src[which], NP * 8); return 0; }
  const double *m4[] = {c->matrixG, c->matrixIG, c->matrixA, c->matrixIA};
  if (which >= 7 && which <= 10) { memcpy(out, m4[which - 7], 4 * NP * 8); return 0; }
  if (which == 11) { memcpy(out, c->areaCell, c->ncx * c->ncy * 6 * 8); return 0; }
  if (which == 12) { memcpy(out, c->gCoef, (size_t)c->nPVx * c->nPVHalo * 8); return 0; }
  if (which == 13) { memcpy(out, c->gX, (size_t)c->nPVx * c->nPVHalo * 8); return 0; }
  return -1;
}
void orc_get_ghost_iref(const orc_ctx *c, int *out) { memcpy(out, c->gIref, sizeof(int) * c->nPVx * c->nPVHalo); }

void orc_set_phi_s(orc_ctx *c, const double *phi_s) { memcpy(c->phi_s, phi_s, c->NP * 8); }

/* test_case_mod.F90:13-39: stat(0) from sphere winds and phi on all padded points */
void orc_init_state(orc_ctx *c, const double *zonal, const double *merid, const double *phi) {
  orc_stat *s = &c->stat[c->old_slot];
  memcpy(s->zonal_wind, zonal, c->NP * 8);
  memcpy(s->meridional_wind, merid, c->NP * 8);
  memcpy(s->phi, phi, c->NP * 8);
  for (long k = 0; k < c->NP; k++) s->phiG[k] = s->phi[k] * c->sqrtG[k];
  for (long k = 0; k < c->NP; k++) {
    covProjSphere2Plane(&s->u[k], &s->v[k], s->zonal_wind[k], s->meridional_wind[k], &c->matrixIA[4 * k],
                        &c->matrixG[4 * k]);
    contravProjSphere2Plane(&s->contraU[k], &s->contraV[k], s->zonal_wind[k], s->meridional_wind[k],
                            &c->matrixIA[4 * k]);
  }
}

/* stat(0) from covariant winds: contraU/V = IG (u,v), as after any update (used for
   state hand-off tests where the caller already holds covariant winds) */
void orc_set_state_cov(orc_ctx *c, const double *u, const double *v, const double *phi) {
  orc_stat *s = &c->stat[c->old_slot];
  memcpy(s->u, u, c->NP * 8);
  memcpy(s->v, v, c->NP * 8);
  memcpy(s->phi, phi, c->NP * 8);
  for (long k = 0; k < c->NP; k++) {
    s->phiG[k] = s->phi[k] * c->sqrtG[k];
    cov2contrav(&s->contraU[k], &s->contraV[k], s->u[k], s->v[k], &c->matrixIG[4 * k]);
  }
}

/* MCV_SW.F90:57-77: nsteps of the selected RK scheme, then switch_stat */
void orc_step(orc_ctx *c, int nsteps) {
  orc_stat *sold = &c->stat[c->old_slot], *snew = &c->stat[c->new_slot];
  for (int it = 1; it <= nsteps; it++) {
    if (c->scheme == 3) RK3_TVD(c, snew, sold);
    else RK4(c, snew, sold);
    copy_stat(c, sold, snew);
  }
}

/* state of stat(old): which 0 u,1 v,2 phi,3 phiG,4 contraU,5 contraV,6 zonal,7 merid */
void orc_get_state(const orc_ctx *c, int which, double *out) {
  const orc_stat *s = &c->stat[c->old_slot];
  const double *src[] = {s->u, s->v, s->phi, s->phiG, s->contraU, s->contraV, s->zonal_wind, s->meridional_wind};
  memcpy(out, src[which], c->NP * 8);
}

/* spatial_operator on stat(old): tendencies (interior layout nPVx*nPVy*6) */
void orc_spatial_operator(orc_ctx *c, double *tphiG, double *tu, double *tv) {
  orc_tend *t = &c->tend[SLOT(c, 1)];
  spatial_operator(c, &c->stat[c->old_slot], t);
  long NI = (long)c->nPVx * c->nPVy * 6;
  memcpy(tphiG, t->phiG, NI * 8); memcpy(tu, t->u, NI * 8); memcpy(tv, t->v, NI * 8);
}

/* update_stat(stat(old) <- stat(old) + inc * tend) including correct_bdy_ghost;
   exposes one stage update for unit tests */
void orc_update_stat(orc_ctx *c, const double *tphiG, const double *tu, const double *tv, double inc_t) {
  orc_tend *t = &c->tend[SLOT(c, 1)];
  long NI = (long)c->nPVx * c->nPVy * 6;
  memcpy(t->phiG, tphiG, NI * 8); memcpy(t->u, tu, NI * 8); memcpy(t->v, tv, NI * 8);
  orc_stat *tmp = &c->stat[SLOT(c, -1)];
  copy_stat(c, tmp, &c->stat[c->old_slot]);
  update_stat(c, &c->stat[c->old_slot], tmp, t, inc_t);
}

/* the boundary/ghost correction alone on stat(old) (after phi = phiG/sqrtG) */
void orc_correct_bdy_ghost(orc_ctx *c) {
  orc_stat *s = &c->stat[c->old_slot];
  phi_from_phiG(c, s);
  correct_bdy_ghost(c, s);
  phiG_from_phi(c, s);
}

/* one-dimensional building blocks for known-answer tests */
double orc_polyfit(orc_ctx *c, int right, const double *pv) { return right ? polyfitR(c->DOF, pv, c->dx) : polyfitL(c->DOF, pv, c->dx); }
void orc_calc_tendP(orc_ctx *c, double *derivP, const double *f, const double *q, double eL, double eR) {
  calc_tendP(c, derivP, f, q, eL, eR);
}
/* interpolate one halo line h from src (n points, unit stride) */
void orc_linear_interp(orc_ctx *c, double *dest, const double *src, int h) { linear_interp(c, dest, 1, src, 1, h); }

double orc_total_mass(const orc_ctx *c) { return calc_total_mass(c, &c->stat[c->old_slot]); }
double orc_total_energy(const orc_ctx *c) { return calc_total_energy(c, &c->stat[c->old_slot]); }
void orc_calc_VIA(const orc_ctx *c, double *out, const double *field) { calc_VIA(c, out, field); }

/* output_mod.F90:230-248: FillValue in the four halo corner squares of u and v */
static void addFillValue(orc_ctx *c, orc_stat *s) {
  for (int p = 1; p <= 6; p++)
    for (int j = c->jps; j <= c->jpe; j++)
      for (int i = c->ips; i <= c->ipe; i++) {
        int xc = i < c->ids || i > c->ide, yc = j < c->jds || j > c->jde;
        if (xc && yc) {
          s->u[PIX(c, i, j, p)] = FILLVALUE;
          s->v[PIX(c, i, j, p)] = FILLVALUE;
        }
      }
}

/* MCV_SW.F90:62-67 on stat(old): addFillValue, convert_wind_P2SP, then calc_VIA
   of u, v, phi; copies out u, v, phi, zonal, meridional (padded) and uC, vC,
   phiC ((ics:ice, jcs:jce, 6), halo cells 0).  Any output may be NULL. */
void orc_history(orc_ctx *c, double *u, double *v, double *phi, double *zonal, double *merid, double *uC, double *vC,
                 double *phiC) {
  orc_stat *s = &c->stat[c->old_slot];
  addFillValue(c, s);
  convert_wind_P2SP(c, s);
  if (uC) calc_VIA(c, uC, s->u);
  if (vC) calc_VIA(c, vC, s->v);
  if (phiC) calc_VIA(c, phiC, s->phi);
  double *dst[5] = {u, v, phi, zonal, merid};
  const double *src[5] = {s->u, s->v, s->phi, s->zonal_wind, s->meridional_wind};
  for (int k = 0; k < 5; k++)
    if (dst[k]) memcpy(dst[k], src[k], c->NP * 8);
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
