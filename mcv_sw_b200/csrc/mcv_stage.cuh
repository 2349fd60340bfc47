// mcv_stage.cuh -- sm_100a stage kernel (K1) of one RK stage of MCV_SW.
//
//  stage_kernel   (K1): per panel tile, the whole spatial operator
//                 (src/spatial_operators_mod.F90:12-133) fused with the RK
//                 stage update (src/time_scheme_mod.F90:71-123, the RK4
//                 combine :38-42) and phi = phiG/sqrtG.  Contravariant winds,
//                 phiG, K and E are recomputed from (u, v, phi) in the tile.
//                 Two arithmetic policies share the kernel: FP64 throughout,
//                 and split precision (FP32 tendencies on phi - phibar from an
//                 FP64 state, FP32 stage increments, metric recomputed per
//                 point in FP64 from 1-D tables).
//  halo_kernel    (K2): correct_bdy_ghost (src/time_scheme_mod.F90:125-142):
//                 ghost fill with the FP64 edge interpolation
//                 (src/ghost_mod.f90:88-227), boundary unification of the 12
//                 edges and 8 vertices (src/spatial_operators_mod.F90:282-388),
//                 sphere<->panel wind rotations on the strips (:408-492).
//
// Device layout of a padded field: [member][panel][row j][pitch P] with
// padded indices (reference index - ips), P >= npx rounded up to 16 elements.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "mcv_tma.cuh"

namespace mcv {

// RK stage kinds: which combination of stage input, RK base and tendency
// makes the stage output.
enum StageKind : int {
  RK3_S1 = 0,  // y1 = y0 + dt L(y0)                          time_scheme_mod.F90:60-61
  RK3_S2 = 1,  // y2 = 3/4 y0 + 1/4 y1 + 1/4 dt L(y1)         :89-105
  RK3_S3 = 2,  // y  = 1/3 y0 + 2/3 y2 + 2/3 dt L(y2)         :107-123
  RK4_S1 = 3,  // y2 = y0 + dt/2 k1; acc = k1                  :27-28
  RK4_S2 = 4,  // y3 = y0 + dt/2 k2; acc += 2 k2               :30-31
  RK4_S3 = 5,  // y4 = y0 + dt k3;   acc += 2 k3               :33-34
  RK4_S4 = 6,  // y  = y0 + dt (acc + k4)/6                    :36-42
};
__host__ __device__ constexpr bool first_stage(int k) { return k == RK3_S1 || k == RK4_S1; }
__host__ __device__ constexpr bool last_stage(int k) { return k == RK3_S3 || k == RK4_S4; }

struct GridDesc {
  int n;      // PVs per panel edge (nPVx)
  int np;     // padded points per direction
  int P;      // row pitch in elements
  int Nc;     // cells per panel edge
  int tiles_x, tiles_y;
  long long plane;    // np * P
  long long mstride;  // 6 * plane
  double dx;          // cell width in radians
  double inv_dx, inv_2dx, inv_dx2;  // 1/dx, 1/(2 dx), 1/dx**2
};

struct StageArgs {
  // ---- FP64 policy ----
  const double *us, *vs, *ps;  // stage input u, v, phi (padded, halo valid)
  const double *u0, *v0, *p0;  // RK base (interior; may alias the outputs)
  double *uo, *vo, *po;        // stage output (interior written here)
  double *aU, *aV, *aP;        // RK4 tendency accumulators
  const double *sqrtG, *ig11, *ig12, *ig22, *fcor;  // metric planes [6][np][P]
  const double *phis;                               // [M][6][np][P]
  double4 *bnd;  // raw boundary copy [M][6][4][n] {u, v, phi, 0}
  double inc;    // dt or dt/2 (update_stat's inc_t) or the RK3 tendency weight
  int *err;      // set to 1 if a staged tile's copies did not arrive in time (TMA form)
  const int *active;  // member index of each grid z slice (the members this launch advances)
  int ident;          // 1 when active[k] == k for every slot: the slot is the member, no load
  // ---- split-precision policy ----
  const double *yu, *yv, *yp;  // FP64 state Y (RK base and stage-1 input), padded; the last
                               // stage writes Y + increment to uo/vo/po (the other state buffer)
  const float *du, *dv, *dp;  // FP32 increment of the stage input over Y (stages >= 2)
  float *eu, *ev, *ep;        // FP32 increment written by intermediate stages
  float *fU, *fV, *fP;        // FP32 RK4 accumulators
  const float *phis32;        // FP32 phi_s [M][6][np][P]
  const double4 *met1d;       // per padded index: {tan, cos^2/R^2, sin cos/R, R sec^2}
  const double *phibar;       // mean depth per member
  float4 *bnd32;              // raw boundary copy of the increment
  double *prec;  // TMA form: linear references of the step's first stage per (member, panel, tile), 12 words each
  double two_omega;
  double r2;  // radius squared (split precision: 1/sqrtG from the 1-D tables)
  float wd, wt;  // increment = wd * (input increment) + wt * tendency (RK3/RK4 weights)
};

// The grids one stage launch advances: one (a handle's own step) or, in a
// batched launch, up to kMaxGrids handles of the same order, arithmetic, tile
// shape and stage kind, each with its own Nc, dt and members.  Work items of
// the TMA form are numbered over all grids: first the items clear of the panel
// edges of every grid (in grid order), then the edge items of every grid, so
// that with programmatic dependent launch the edge-free items of every grid
// start while the previous halo kernels still run.
constexpr int kMaxGrids = 4;
template <int NB>
struct StageBatch {
  TileMaps tm[NB];  // tensor maps of each grid's staged fields (TMA form)
  GridDesc g[NB];
  StageArgs a[NB];
  int ngrids;
  int total;        // work items of all grids
  int nin;          // items clear of the panel edges, all grids
  int in0[NB + 1];  // first edge-free item of each grid
  int ed0[NB + 1];  // first edge item of each grid, counted from nin
  int slots[NB];    // active members of each grid
};

// ---------------------------------------------------------------------------
// One-dimensional MCV building blocks (src/spatial_operators_mod.F90:136-246).
// Divisions by the cell width are multiplications by precomputed reciprocals,
// one rounding away from the reference's quotient.
// ---------------------------------------------------------------------------
template <int D, typename R>
__device__ __forceinline__ R polyfit_left(const R *pv, R inv) {
  // inv = 1/dh (MCV3) or 1/(2 dh) (MCV4)
  if constexpr (D == 3) return -(pv[2] - R(4) * pv[1] + R(3) * pv[0]) * inv;
  else return (-(R(11) * pv[0]) + R(18) * pv[1] - R(9) * pv[2] + R(2) * pv[3]) * inv;
}
template <int D, typename R>
__device__ __forceinline__ R polyfit_right(const R *pv, R inv) {
  if constexpr (D == 3) return (pv[0] - R(4) * pv[1] + R(3) * pv[2]) * inv;
  else return (R(11) * pv[3] - R(18) * pv[2] + R(9) * pv[1] - R(2) * pv[0]) * inv;
}
template <typename R>
__device__ __forceinline__ R riemann(R fL, R fR, R qL, R qR, R lam) {
  return R(0.5) * ((fL + fR) - lam * (qR - qL));
}

// Cell-width constants in the arithmetic type of the sweep.
template <typename R>
struct Widths {
  R dx, inv_dx, inv_2dx, inv_dx2;
  __device__ explicit Widths(const GridDesc &g)
      : dx(R(g.dx)), inv_dx(R(g.inv_dx)), inv_2dx(R(g.inv_2dx)), inv_dx2(R(g.inv_dx2)) {}
};

// calc_tendP (src/spatial_operators_mod.F90:136-202) for the centre cell of a
// 3-cell window (3D-2 values with stride S): derivatives at its D points.
template <int D, int S, typename R>
__device__ __forceinline__ void cell_derivs(R out[D], const R *f, const R *q, R lamL, R lamR, const Widths<R> &w) {
  const R ip = (D == 3) ? w.inv_dx : w.inv_2dx;
  R c1[D], c2[D], c3[D], d1[D], d2[D], d3[D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    c1[m] = f[m * S];
    c2[m] = f[(D - 1 + m) * S];
    c3[m] = f[(2 * D - 2 + m) * S];
    d1[m] = q[m * S];
    d2[m] = q[(D - 1 + m) * S];
    d3[m] = q[(2 * D - 2 + m) * S];
  }
  const R fxL1 = polyfit_right<D>(c1, ip), fxL2 = polyfit_right<D>(c2, ip);
  const R fxR1 = polyfit_left<D>(c2, ip), fxR2 = polyfit_left<D>(c3, ip);
  const R qxL1 = polyfit_right<D>(d1, ip), qxL2 = polyfit_right<D>(d2, ip);
  const R qxR1 = polyfit_left<D>(d2, ip), qxR2 = polyfit_left<D>(d3, ip);
  out[0] = riemann(fxL1, fxR1, qxL1, qxR1, lamL);
  out[D - 1] = riemann(fxL2, fxR2, qxL2, qxR2, lamR);
  if constexpr (D == 3) {
    const R fxVIA = (c2[2] - c2[0]) * w.inv_dx;
    out[1] = R(1.5) * fxVIA - R(0.25) * (out[0] + out[2]);
  } else {
    const R fxVIA = (c2[3] - c2[0]) * w.inv_dx;
    const R fxxc = R(4.5) * (c2[0] - c2[1] - c2[2] + c2[3]) * w.inv_dx2;
    out[1] = R(4. / 3.) * fxVIA - (R(4) * out[0] + R(5) * out[3]) * R(1. / 27.) - R(4. / 27.) * w.dx * fxxc;
    out[2] = R(4. / 3.) * fxVIA - (R(5) * out[0] + R(4) * out[3]) * R(1. / 27.) + R(4. / 27.) * w.dx * fxxc;
  }
}

// Split precision: calc_tendP for two quantities at once, one in each half of
// a float2 (packed FP32 FMA, FFMA2); both use the same eigenvalues.  Same
// formulas as cell_derivs, with the sums ordered explicitly.
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

template <int D>
__device__ __forceinline__ float2 polyfit_left2(const float2 *p, float2 inv) {
  if constexpr (D == 3) {
    // -(p2 - 4 p1 + 3 p0) / dh
    const float2 t = fma2(bc2(3.f), p[0], fma2(bc2(-4.f), p[1], p[2]));
    return mul2(t, make_float2(-inv.x, -inv.y));
  } else {
    // (-11 p0 + 18 p1 - 9 p2 + 2 p3) / (2 dh)
    float2 t = mul2(bc2(2.f), p[3]);
    t = fma2(bc2(-9.f), p[2], t);
    t = fma2(bc2(18.f), p[1], t);
    t = fma2(bc2(-11.f), p[0], t);
    return mul2(t, inv);
  }
}
template <int D>
__device__ __forceinline__ float2 polyfit_right2(const float2 *p, float2 inv) {
  if constexpr (D == 3) {
    // (p0 - 4 p1 + 3 p2) / dh
    const float2 t = fma2(bc2(3.f), p[2], fma2(bc2(-4.f), p[1], p[0]));
    return mul2(t, inv);
  } else {
    // (11 p3 - 18 p2 + 9 p1 - 2 p0) / (2 dh)
    float2 t = mul2(bc2(-2.f), p[0]);
    t = fma2(bc2(9.f), p[1], t);
    t = fma2(bc2(-18.f), p[2], t);
    t = fma2(bc2(11.f), p[3], t);
    return mul2(t, inv);
  }
}
__device__ __forceinline__ float2 riemann2(float2 fL, float2 fR, float2 qL, float2 qR, float lam) {
  const float2 dq = fma2(bc2(-1.f), qL, qR);
  return mul2(bc2(0.5f), fma2(bc2(-lam), dq, add2(fL, fR)));
}

template <int D, int S>
__device__ __forceinline__ void cell_derivs2(float2 out[D], const float2 *f, const float2 *q, float lamL, float lamR,
                                             const Widths<float> &w) {
  const float ipf = (D == 3) ? w.inv_dx : w.inv_2dx;
  const float2 ip = bc2(ipf);
  float2 c1[D], c2[D], c3[D], d1[D], d2[D], d3[D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    c1[m] = f[m * S];
    c2[m] = f[(D - 1 + m) * S];
    c3[m] = f[(2 * D - 2 + m) * S];
    d1[m] = q[m * S];
    d2[m] = q[(D - 1 + m) * S];
    d3[m] = q[(2 * D - 2 + m) * S];
  }
  out[0] = riemann2(polyfit_right2<D>(c1, ip), polyfit_left2<D>(c2, ip), polyfit_right2<D>(d1, ip),
                    polyfit_left2<D>(d2, ip), lamL);
  out[D - 1] = riemann2(polyfit_right2<D>(c2, ip), polyfit_left2<D>(c3, ip), polyfit_right2<D>(d2, ip),
                        polyfit_left2<D>(d3, ip), lamR);
  const float2 via = mul2(fma2(bc2(-1.f), c2[0], c2[D - 1]), bc2(w.inv_dx));  // (f_R - f_L)/dx
  if constexpr (D == 3) {
    out[1] = fma2(bc2(1.5f), via, mul2(bc2(-0.25f), add2(out[0], out[2])));
  } else {
    // 4/27 dx * 4.5 (c0 - c1 - c2 + c3)/dx^2 = (2/3)(c0 - c1 - c2 + c3)/dx
    const float2 t = fma2(bc2(-1.f), c2[2], fma2(bc2(-1.f), c2[1], add2(c2[0], c2[3])));
    const float2 k = mul2(bc2(2.f / 3.f), mul2(t, bc2(w.inv_dx)));
    float2 a = fma2(bc2(-4.f / 27.f), out[0], mul2(bc2(4.f / 3.f), via));
    out[1] = fma2(bc2(-1.f), k, fma2(bc2(-5.f / 27.f), out[3], a));
    a = fma2(bc2(-5.f / 27.f), out[0], mul2(bc2(4.f / 3.f), via));
    out[2] = add2(k, fma2(bc2(-4.f / 27.f), out[3], a));
  }
}

// Interface eigenvalues or upwind signs along a walk, interface i = 0..ncells:
// read from an array (ArrLam), or formed at the interface point from the
// stored contravariant wind c and G^ii phi (EigLam: max(|c - s|, |c + s|) =
// |c| + s with s = sqrt(G^ii phi), spatial_operators_mod.F90:248-280; SgnLam:
// the upwind sign of c, :83-85), st = the interface points' stride.
template <typename R>
struct ArrLam {
  const R *p;
  __device__ __forceinline__ R operator()(int i) const { return p[i]; }
};
// (EigLam's square root is the hardware approximation, relative error ~2^-23:
// the wave speed only scales the interface dissipation, and both tiles at a
// seam form it from the same stored values, so their fluxes still agree.)
struct EigLam {
  const float *c, *gp;
  int st;
  __device__ __forceinline__ float operator()(int i) const {
    float s;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(gp[i * st]));
    return fabsf(c[i * st]) + s;
  }
};
struct SgnLam {
  const float *c;
  int st;
  __device__ __forceinline__ float operator()(int i) const { return (c[i * st] < 0.f) ? -1.f : 1.f; }
};

// calc_tendP (src/spatial_operators_mod.F90:136-202) applied to every cell of
// one grid line of `ncells` cells, as the x-sweep (:63-93) and y-sweep (:95-125)
// do for each row and column.  f and q point to the first point of the halo
// cell before the line (stride S), lam to the eigenvalue or upwind sign at the
// line's first interface (stride 1), out to the line's first point (stride OS).
// Walking the line carries the previous cell's one-sided derivatives, so each
// interface flux is formed once; it is the value both neighbouring cells'
// calc_tendP calls produce.  SAME: f and q are the same field (dvdx, dudy).
// The walk's last point is written only when the walk ends the line (`ends`):
// otherwise it is the next walk's first point, which that walk writes (one
// writer per point).
template <int D, int NMAX, int S, int OS, bool SAME, typename R, class L>
__device__ __forceinline__ void line_walk(const R *f, const R *q, const L &lam, int ncells, bool ends, R *out,
                                          const Widths<R> &w) {
  const R ip = (D == 3) ? w.inv_dx : w.inv_2dx;
  R cf[D], cq[D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    cf[m] = f[m * S];
    cq[m] = SAME ? cf[m] : q[m * S];
  }
  // right-end derivatives of the halo cell before the line
  R fR = polyfit_right<D>(cf, ip), qR = SAME ? fR : polyfit_right<D>(cq, ip);
  // first cell of the line
  {
    R nf[D], nq[D];
    nf[0] = cf[D - 1];
    nq[0] = cq[D - 1];
#pragma unroll
    for (int m = 1; m < D; ++m) {
      nf[m] = f[(D - 1 + m) * S];
      nq[m] = SAME ? nf[m] : q[(D - 1 + m) * S];
    }
#pragma unroll
    for (int m = 0; m < D; ++m) {
      cf[m] = nf[m];
      cq[m] = nq[m];
    }
  }
  R fL = polyfit_left<D>(cf, ip), qL = SAME ? fL : polyfit_left<D>(cq, ip);
  R fluxL = riemann(fR, fL, qR, qL, lam(0));
  fR = polyfit_right<D>(cf, ip);
  qR = SAME ? fR : polyfit_right<D>(cq, ip);
#pragma unroll
  for (int c = 0; c < NMAX; ++c) {
    if (c < ncells) {
      R nf[D], nq[D];
      nf[0] = cf[D - 1];
      nq[0] = cq[D - 1];
#pragma unroll
      for (int m = 1; m < D; ++m) {
        nf[m] = f[((c + 2) * (D - 1) + m) * S];
        nq[m] = SAME ? nf[m] : q[((c + 2) * (D - 1) + m) * S];
      }
      const R nfL = polyfit_left<D>(nf, ip), nqL = SAME ? nfL : polyfit_left<D>(nq, ip);
      const R fluxR = riemann(fR, nfL, qR, nqL, lam(c + 1));
      R o[D];
      o[0] = fluxL;
      o[D - 1] = fluxR;
      if constexpr (D == 3) {
        const R fxVIA = (cf[2] - cf[0]) * w.inv_dx;
        o[1] = R(1.5) * fxVIA - R(0.25) * (o[0] + o[2]);
      } else {
        const R fxVIA = (cf[3] - cf[0]) * w.inv_dx;
        const R fxxc = R(4.5) * (cf[0] - cf[1] - cf[2] + cf[3]) * w.inv_dx2;
        o[1] = R(4. / 3.) * fxVIA - (R(4) * o[0] + R(5) * o[3]) * R(1. / 27.) - R(4. / 27.) * w.dx * fxxc;
        o[2] = R(4. / 3.) * fxVIA - (R(5) * o[0] + R(4) * o[3]) * R(1. / 27.) + R(4. / 27.) * w.dx * fxxc;
      }
#pragma unroll
      for (int m = 0; m < D - 1; ++m) out[(c * (D - 1) + m) * OS] = o[m];
      if (c == ncells - 1 && ends) out[(c * (D - 1) + D - 1) * OS] = o[D - 1];
#pragma unroll
      for (int m = 0; m < D; ++m) {
        cf[m] = nf[m];
        cq[m] = nq[m];
      }
      fR = polyfit_right<D>(cf, ip);
      qR = SAME ? fR : polyfit_right<D>(cq, ip);
      fluxL = fluxR;
    }
  }
}

// The interior points of one cell from its end derivatives (packed pairs):
// the MCV constraint of calc_tendP (src/spatial_operators_mod.F90:179-200).
template <int D, int S>
__device__ __forceinline__ void cell_interior2(float2 o[D], const float2 *c, const Widths<float> &w) {
  const float2 via = mul2(fma2(bc2(-1.f), c[0], c[(D - 1) * S]), bc2(w.inv_dx));
  if constexpr (D == 3) {
    o[1] = fma2(bc2(1.5f), via, mul2(bc2(-0.25f), add2(o[0], o[2])));
  } else {
    const float2 t = fma2(bc2(-1.f), c[2 * S], fma2(bc2(-1.f), c[S], add2(c[0], c[3 * S])));
    const float2 k = mul2(bc2(2.f / 3.f), mul2(t, bc2(w.inv_dx)));
    float2 a = fma2(bc2(-4.f / 27.f), o[0], mul2(bc2(4.f / 3.f), via));
    o[1] = fma2(bc2(-1.f), k, fma2(bc2(-5.f / 27.f), o[3], a));
    a = fma2(bc2(-5.f / 27.f), o[0], mul2(bc2(4.f / 3.f), via));
    o[2] = add2(k, fma2(bc2(-4.f / 27.f), o[3], a));
  }
}

// line_walk for two quantities at once (packed FP32 pairs, one eigenvalue per
// interface): f and q point to the first point of the halo cell before the
// walk, the result pairs go to out.
template <int D, int NMAX, int S, int OS, class L>
__device__ __forceinline__ void line_walk2(const float2 *f, const float2 *q, const L &lam, int ncells, bool ends,
                                           float2 *out, const Widths<float> &w) {
  const float2 ip = bc2((D == 3) ? w.inv_dx : w.inv_2dx);
  float2 cf[D], cq[D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    cf[m] = f[m * S];
    cq[m] = q[m * S];
  }
  float2 fR = polyfit_right2<D>(cf, ip), qR = polyfit_right2<D>(cq, ip);
  cf[0] = cf[D - 1];  // the point the halo cell and the first cell share
  cq[0] = cq[D - 1];
#pragma unroll
  for (int m = 1; m < D; ++m) {
    cf[m] = f[(D - 1 + m) * S];
    cq[m] = q[(D - 1 + m) * S];
  }
  float2 fluxL = riemann2(fR, polyfit_left2<D>(cf, ip), qR, polyfit_left2<D>(cq, ip), lam(0));
  fR = polyfit_right2<D>(cf, ip);
  qR = polyfit_right2<D>(cq, ip);
#pragma unroll
  for (int c = 0; c < NMAX; ++c) {
    if (c < ncells) {
      float2 nf[D], nq[D];
      nf[0] = cf[D - 1];
      nq[0] = cq[D - 1];
#pragma unroll
      for (int m = 1; m < D; ++m) {
        nf[m] = f[((c + 2) * (D - 1) + m) * S];
        nq[m] = q[((c + 2) * (D - 1) + m) * S];
      }
      const float2 fluxR = riemann2(fR, polyfit_left2<D>(nf, ip), qR, polyfit_left2<D>(nq, ip), lam(c + 1));
      float2 o[D];
      o[0] = fluxL;
      o[D - 1] = fluxR;
      cell_interior2<D, 1>(o, cf, w);
#pragma unroll
      for (int m = 0; m < D - 1; ++m) out[(c * (D - 1) + m) * OS] = o[m];
      if (c == ncells - 1 && ends) out[(c * (D - 1) + D - 1) * OS] = o[D - 1];
#pragma unroll
      for (int m = 0; m < D; ++m) {
        cf[m] = nf[m];
        cq[m] = nq[m];
      }
      fR = polyfit_right2<D>(cf, ip);
      qR = polyfit_right2<D>(cq, ip);
      fluxL = fluxR;
    }
  }
}

// ---------------------------------------------------------------------------
// K1: fused spatial operator + RK stage on one tile of CX x CY cells.
// ---------------------------------------------------------------------------
template <int D, int CX, int CY, typename R>
struct Tile {
  static constexpr int H = D - 1;
  static constexpr int TX = CX * (D - 1) + 1;  // tile points per row (max)
  static constexpr int TY = CY * (D - 1) + 1;
  static constexpr int LX = TX + 2 * H;        // loaded row length (odd: no bank conflicts on column walks)
  static constexpr int LY = TY + 2 * H;
  static constexpr int A = LX * LY;  // loaded rectangle (corners unused)
  static constexpr int I = TX * TY;  // tile interior
  // shared-memory carve (elements of R): full-rectangle arrays -- FP64 policy:
  // u, v, E, phiG, phiG cU, phiG cV; split precision: u, v and the sweep pairs
  // as float2 [A] each: XF = (E, phiG cU), XQ = (u, phiG), YF = (E, phiG cV),
  // YQ = (v, phiG) (the x and y sweeps' flux and Riemann fields) ...
  static constexpr bool PAIRED = std::is_same<R, float>::value;
  static constexpr int U = 0, V = A, E = 2 * A, PG = 3 * A, PGU = 4 * A, PGV = 5 * A;
  static constexpr int XF = 2 * A, XQ = 4 * A, YF = 6 * A, YQ = 8 * A;  // in floats (even: float2-aligned)
  // ... interior-only arrays: sqrtG, cU, cV (split precision: 1/sqrtG, cU,
  // cV, sqrtG f) ...
  static constexpr int SG = (PAIRED ? 10 : 6) * A, CU = SG + I, CV = CU + I, FC = CV + I;
  // ... interface eigenvalues and upwind signs (FP64 policy); split precision
  // keeps G^11 phi and G^22 phi per interior point (GPX, GPY) instead and
  // forms the eigenvalues and signs in the sweeps ...
  static constexpr int LAMX = CV + (PAIRED ? 2 : 1) * I;  // [TY][CX+1]
  static constexpr int SGNX = LAMX + TY * (CX + 1);
  static constexpr int LAMY = SGNX + TY * (CX + 1);  // [TX][CY+1]
  static constexpr int SGNY = LAMY + TX * (CY + 1);
  static constexpr int GPX = LAMX, GPY = LAMX + I;  // split precision [TY][TX] each
  // ... sweep results [3][TY][TX] each (split precision: the first two as
  // float2 pairs [TY][TX] {flux, divergence}, then the third) ...
  static constexpr int XR = PAIRED ? GPY + I : SGNY + TX * (CY + 1);
  static constexpr int YR = XR + 3 * I + (PAIRED ? (I & 1) : 0);  // float2-aligned
  static constexpr int TOTAL = YR + 3 * I;
  // split precision, after the R arrays: 1-D metric tables [LX] and [LY] double4,
  // then two buffers (alternate work items of the TMA form) of the per-tile
  // linear references of E, u, v: planes [3][3] double and slopes [2][3] float
  // (together the 96-byte record a first stage stores and later stages load),
  // then reference-point values [3][3] double
  static constexpr size_t MET_OFF = ((size_t)TOTAL * sizeof(R) + 31) / 32 * 32;
  static constexpr size_t PLANE_OFF = MET_OFF + (size_t)(LX + LY) * sizeof(double4);
  static constexpr size_t PLANE_BYTES = 176;  // 18 doubles + 6 floats, a 16-byte multiple
  __host__ __device__ static constexpr size_t bytes(bool mixed) {
    return mixed ? PLANE_OFF + 2 * PLANE_BYTES : (size_t)TOTAL * sizeof(R);
  }
  // TMA form, after all of the above: one work item's input fields as staged
  // boxes [LY][BX] (FP64 policy: 8 FP64 fields; split precision: 3 FP64 then 4
  // FP32 fields), each slot 128-byte aligned, then the mbarrier
  static constexpr int BX = (LX + 3) / 4 * 4;  // box row: a 16-byte multiple for 4- and 8-byte elements
  static constexpr size_t FB64 = ((size_t)BX * LY * 8 + 127) / 128 * 128;
  static constexpr size_t FB32 = ((size_t)BX * LY * 4 + 127) / 128 * 128;
  __host__ __device__ static constexpr size_t stg_off(bool mixed) { return (bytes(mixed) + 127) / 128 * 128; }
  __host__ __device__ static constexpr size_t field_off(bool mixed, int f) {
    return stg_off(mixed) + (mixed ? (f < 3 ? f * FB64 : 3 * FB64 + (f - 3) * FB32) : f * FB64);
  }
  __host__ __device__ static constexpr uint32_t field_bytes(bool mixed, int f) {
    return (uint32_t)BX * LY * ((mixed && f >= 3) ? 4u : 8u);
  }
  __host__ __device__ static constexpr size_t bar_off(bool mixed) { return field_off(mixed, mixed ? 7 : 8); }
  __host__ __device__ static constexpr size_t bytes_tma(bool mixed) { return bar_off(mixed) + 16; }
  static_assert(LX % 2 == 1, "odd shared row length");
  static_assert(!PAIRED || (XR % 2 == 0 && YR % 2 == 0), "float2 sweep results");
};

// Split precision: the FP64 quantities of one loaded point.  q = {E - phibar,
// u, v, phiG, phiG cU, phiG cV} are the fields the sweeps difference.
struct MixPoint {
  double q[6];
  double sg, cu, cv, g11, g22, fc, rsg;
};
__device__ __forceinline__ void mix_point(MixPoint &o, const double4 mx, const double4 my, double u, double v,
                                          double p, double phs, double phibar, int panel, double two_omega,
                                          double r2) {
  // equiangular metric from the separable 1-D tables {tan, cos^2/R^2, sin cos/R,
  // R/cos^2} (projection_mod.F90:150-211 with cos^2 y (1 + tan^2 y) = 1)
  const double rho2 = 1. + mx.x * mx.x + my.x * my.x;
  // 1/sqrt(rho2), rho2 in [1, 3): the FP32 hardware approximation (relative
  // error < 2^-22) refined by one Newton-Raphson step for 1/sqrt,
  // y' = y + y (1 - rho2 y^2) / 2: relative error 1.5 e^2 < 1.5e-13 for a seed
  // error e < 2^-22 (tests/test_rsqrt_newton.py).
  // Only sqrtG, 1/sqrtG and f use it, and each is rounded to FP32.
  float y32;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y32) : "f"((float)rho2));
  const double y0 = (double)y32;
  const double rinv = __fma_rn(0.5 * y0, __fma_rn(-rho2 * y0, y0, 1.), y0);
  o.sg = mx.w * my.w * (rinv * rinv * rinv);
  o.rsg = (rho2 * rho2 * rinv) * ((mx.y * my.y) * r2);  // 1/sqrtG: 1/(R sec^2) = R cos^2/R^2
  o.g11 = rho2 * mx.y;
  o.g22 = rho2 * my.y;
  const double g12 = rho2 * (mx.z * my.z);
  o.cu = o.g11 * u + g12 * v;  // cov2contrav, projection_mod.F90:138-148
  o.cv = g12 * u + o.g22 * v;
  const double pg = p * o.sg;
  o.q[0] = (p - phibar) + phs + 0.5 * (o.cu * u + o.cv * v);  // E = phi + phi_s + K
  o.q[1] = u;
  o.q[2] = v;
  o.q[3] = pg;
  o.q[4] = pg * o.cu;
  o.q[5] = pg * o.cv;
  // Coriolis f = 2 Omega sin(lat): sin(lat) = tan y / rho on panels 1-4, +-1/rho on 5, 6
  o.fc = two_omega * (panel < 4 ? my.x * rinv : (panel == 4 ? rinv : -rinv));
}

// Work item wi of a TMA-form launch -> tile (tx, ty), panel and active-member
// slot.  Items whose tiles lie away from the panel edges come first: with
// programmatic dependent launch they start while the previous halo kernel
// still runs (they read nothing it writes), and the edge items, which wait for
// it, come last.  nslots = active members of the launch.
struct WorkItem {
  int tx, ty, panel, slot;
};
// Edge-free items of one grid (tiles_x - 2)(tiles_y - 2) x 6 x nslots and its
// edge items, each numbered from 0 (interior: j < nin x 6 x nslots).
__host__ __device__ inline int edge_free_tiles(int tiles_x, int tiles_y) {
  return (tiles_x > 2 ? tiles_x - 2 : 0) * (tiles_y > 2 ? tiles_y - 2 : 0);
}
__device__ __forceinline__ WorkItem decode_item(int wi, int tiles_x, int tiles_y, int nslots) {
  const int ix = max(tiles_x - 2, 0), iy = max(tiles_y - 2, 0);
  const int nin = ix * iy, nedge = tiles_x * tiles_y - nin;
  WorkItem w;
  int ps;
  if (wi < nin * 6 * nslots) {
    ps = wi / nin;
    const int r = wi - ps * nin;
    w.tx = 1 + r % ix;
    w.ty = 1 + r / ix;
  } else {
    const int wj = wi - nin * 6 * nslots;
    ps = wj / nedge;
    const int e = wj - ps * nedge;
    if (e < tiles_x) {
      w.tx = e;
      w.ty = 0;
    } else if (e < 2 * tiles_x) {
      w.tx = e - tiles_x;
      w.ty = tiles_y - 1;
    } else {
      const int f = e - 2 * tiles_x;
      w.tx = (f < iy) ? 0 : tiles_x - 1;
      w.ty = 1 + ((f < iy) ? f : f - iy);
    }
  }
  w.panel = ps % 6;
  w.slot = ps / 6;
  return w;
}

// Work item wi of a (batched) TMA-form launch: its grid k and the item within
// that grid (decode_item's numbering: edge-free items first).
template <int NB>
__device__ __forceinline__ WorkItem decode_batch(const StageBatch<NB> &b, int wi, int &k) {
  k = 0;
  int local;
  if (wi < b.nin) {
#pragma unroll
    for (int j = 1; j < NB; ++j)
      if (j < b.ngrids && wi >= b.in0[j]) k = j;
    local = wi - b.in0[k];
  } else {
    const int e = wi - b.nin;
#pragma unroll
    for (int j = 1; j < NB; ++j)
      if (j < b.ngrids && e >= b.ed0[j]) k = j;
    local = (b.in0[k + 1] - b.in0[k]) + (e - b.ed0[k]);
  }
  return decode_item(local, b.g[k].tiles_x, b.g[k].tiles_y, b.slots[k]);
}

// PTX programmatic dependent launch: wait until the preceding kernel (the halo
// kernel) has completed and its writes are visible; let the next kernel launch.
// The member an active slot advances.  With an identity list (ident) it is the
// slot itself; the load sits in inline assembly so that it is not hoisted
// above the test and waited for on the identity path.
__device__ __forceinline__ int active_member(const int *active, int ident, int slot) {
  if (ident) return slot;
  int m;
  asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(m) : "l"(active + slot));
  return m;
}
__device__ __forceinline__ void wait_prerequisite_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependent_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// MINB: CTAs per SM the register allocation must allow (launch bounds).
// WALK: 0 -- sweeps as per-cell items; n -- sweeps as walks of n cells.
// OPT bit 1 (split precision with walks): balanced sweeps -- the one-quantity
// walks are twice as long as the packed-pair walks, so that items cost alike
// (all stages but the last, whose longer walks would spill registers).
// OPT bit 2 (TMA form, rows of 28..32 points): each thread forms its loaded
// column's linear references once per work item instead of once per point.
// TMA: persistent form -- each CTA walks work items (tile, panel, member)
// blockIdx.x, blockIdx.x + gridDim.x, ...; the next item's input fields are
// copied into a shared-memory staging area by TMA while the current item's
// sweeps and update run.  A work item has three block barriers (after the
// copy wait, after phase 0, after the sweeps); split precision fits the
// linear references in the step's first stage and stores them, and the later
// stages' copies bring them in with the tile.  Otherwise one CTA per (tile,
// panel, member) loads its fields with ordinary loads.
// IDENT: a one-grid launch whose active list is the identity (the member of a
// slot is the slot, known to the compiler); otherwise the list is read, or
// skipped at run time when StageArgs::ident says it is the identity.
template <int D, int CX, int CY, int NT, int MINB, int KIND, bool MIXED, int WALK, bool TMA, int OPT, int NB,
          bool IDENT = false>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const __grid_constant__ StageBatch<NB> b) {
  using R = std::conditional_t<MIXED, float, double>;
  using T = Tile<D, CX, CY, R>;
  constexpr int H = T::H, LX = T::LX;
  extern __shared__ __align__(128) unsigned char smraw[];
  R *sm = reinterpret_cast<R *>(smraw);
  double4 *metx = reinterpret_cast<double4 *>(smraw + T::MET_OFF);  // split precision: [LX] then [LY]
  const double4 *mety = metx + LX;
  double *plane = reinterpret_cast<double *>(smraw + T::PLANE_OFF);  // [3] {value at (H, H), d/dlx, d/dly}
  float *slope = reinterpret_cast<float *>(plane + 9);                 // [x, y][3]: derivative per radian
  double *qref = plane + 12;                                           // [3 points][3]
  int pb = 0;  // TMA form: plane buffer of the current work item
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + T::bar_off(MIXED));
  // TMA form, loaded rows of 28..32 points: phase 0 maps lanes to columns
  constexpr bool ROWMAP = TMA && LX >= 28 && LX <= 32 && NT % 32 == 0;
  // number of staged fields (split precision: the first stage has no input increment)
  constexpr int NF = MIXED ? (first_stage(KIND) ? 4 : 7) : 8;

  // the loaded rectangle of tile (tx, ty) of grid g reaches a panel boundary
  // line or the halo, which the previous halo kernel writes
  auto touches_edge = [&](const GridDesc &g, int tx, int ty) {
    const int cx = min(CX, g.Nc - tx * CX), cy = min(CY, g.Nc - ty * CY);
    const int x0 = tx * CX * (D - 1) - H, x1 = tx * CX * (D - 1) + cx * (D - 1) + H;  // interior indices
    const int y0 = ty * CY * (D - 1) - H, y1 = ty * CY * (D - 1) + cy * (D - 1) + H;
    return x0 < 1 || y0 < 1 || x1 > g.n - 2 || y1 > g.n - 2;
  };
  bool waited = false;  // TMA form, thread 0: the prerequisite grid has completed
  // TMA: issue the copies of work item wi's input fields (one thread)
  auto issue = [&](int wi) {
    int k;
    const WorkItem it = decode_batch(b, wi, k);
    const GridDesc &g = b.g[k];
    const StageArgs &a = b.a[k];
    const TileMaps &tm = b.tm[k];
    const int ntile = g.tiles_x * g.tiles_y;
    if (!waited && touches_edge(g, it.tx, it.ty)) {
      wait_prerequisite_grid();
      waited = true;
    }
    const int panel = it.panel, mem = IDENT ? it.slot : active_member(a.active, a.ident, it.slot);
    const int X0 = it.tx * CX * (D - 1), Y0 = it.ty * CY * (D - 1);
    uint32_t bytes = 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) bytes += T::field_bytes(MIXED, f);
    int nx = 0, ny = 0;
    if constexpr (MIXED) {
      nx = min(LX, g.np - X0);
      ny = min(T::LY, g.np - Y0);
      bytes += (uint32_t)(nx + ny) * sizeof(double4);
      if constexpr (!first_stage(KIND)) bytes += 96;  // the item's linear references
    }
    mbar_arrive_expect_tx(bar, bytes);
    const int srow = (mem * 6 + panel) * g.np + Y0;  // row of a per-member field
    const int mrow = panel * g.np + Y0;              // row of a metric plane
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma_load_2d(smraw + T::field_off(MIXED, f), &tm.f[f], X0, (!MIXED && f >= 4) ? mrow : srow, bar);
    if constexpr (MIXED) {
      bulk_load(metx, a.met1d + X0, (uint32_t)nx * sizeof(double4), bar);
      bulk_load(metx + LX, a.met1d + Y0, (uint32_t)ny * sizeof(double4), bar);
      // later stages of a step take the linear references the step's first
      // stage fitted for this tile, into the buffer the item will use
      if constexpr (!first_stage(KIND))
        bulk_load(smraw + T::PLANE_OFF + pb * T::PLANE_BYTES,
                  a.prec + ((long long)(mem * 6 + panel) * ntile + it.ty * g.tiles_x + it.tx) * 12, 96u, bar);
    }
  };
  uint32_t parity = 0;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && (int)blockIdx.x < b.total) issue(blockIdx.x);
  }
  const int wfirst = TMA ? (int)blockIdx.x : 0, wstep = TMA ? (int)gridDim.x : 1, wend = TMA ? b.total : 1;
  for (int wi = wfirst; wi < wend; wi += wstep) {
  int kgrid = 0;  // the item's grid
  WorkItem item{};
  if constexpr (TMA) item = decode_batch(b, wi, kgrid);
  const GridDesc &g = b.g[kgrid];
  const StageArgs &a = b.a[kgrid];
  const int ntile = g.tiles_x * g.tiles_y;
  // 1 / (full tile width in radians), x and y (split precision's linear references)
  const double2 inv_full_w = MIXED ? make_double2(1. / ((double)CX * g.dx), 1. / ((double)CY * g.dx))
                                   : make_double2(0., 0.);
  if constexpr (TMA && MIXED) {
    // alternate buffers: the next item's references (fitted by warp 0, or
    // copied in with the tile) land while other warps may still read this
    // item's slopes in phase A
    plane = reinterpret_cast<double *>(smraw + T::PLANE_OFF + pb * T::PLANE_BYTES);
    slope = reinterpret_cast<float *>(plane + 9);
    qref = plane + 12;
    pb ^= 1;
  }
  int tx, ty, panel, mem;
  if constexpr (TMA) {
    tx = item.tx;
    ty = item.ty;
    panel = item.panel;
    mem = IDENT ? item.slot : active_member(a.active, a.ident, item.slot);
    // the CTA's last item: the halo kernel that follows may become resident
    // (it waits for this grid's completion before reading what it writes)
    if (wi + wstep >= wend) allow_dependent_launch();
  } else {
    // one CTA per (tile, panel, member) in panel order, which keeps the
    // neighbours' halo reads in L2; it starts once the previous kernel is done
    tx = blockIdx.x % g.tiles_x;
    ty = blockIdx.x / g.tiles_x;
    panel = blockIdx.y;
    mem = IDENT ? (int)blockIdx.z : active_member(a.active, a.ident, (int)blockIdx.z);
    wait_prerequisite_grid();
  }
  const int c0x = tx * CX, c0y = ty * CY;
  const int ncx = min(CX, g.Nc - c0x), ncy = min(CY, g.Nc - c0y);
  const int X0 = c0x * (D - 1), Y0 = c0y * (D - 1);  // padded coords of the first loaded point
  const int lxe = ncx * (D - 1) + 1 + 2 * H, lye = ncy * (D - 1) + 1 + 2 * H;
  const long long pbase = (long long)panel * g.plane;
  const long long mbase = (long long)mem * g.mstride + pbase;
  const int txe = ncx * (D - 1) + 1, tye = ncy * (D - 1) + 1;  // tile points per row / column
  const double phibar = MIXED ? a.phibar[mem] : 0.;

  // ---- phase 0: load the tile and its halo cross, pointwise quantities ----
  // (spatial_operators_mod.F90:58-61, eigenvalues :248-280, upwind signs :83-85)
  // Per-tile base pointers: every field shares the pitch, so one 32-bit offset
  // per point addresses all of them.
  // Split precision: E, u and v -- the fields of the momentum tendencies, whose
  // pressure-gradient and Coriolis terms nearly cancel -- are formed in FP64,
  // and a linear function of (lx, ly) fitted to three points of the tile is
  // subtracted before rounding to FP32.  The reconstruction and the Riemann
  // fluxes are linear in the fields and exact for linear data (equal one-sided
  // derivatives, no jump), so the sweeps of the residual plus the plane's exact
  // derivative equal the sweeps of the field, while FP32 holds only the
  // residual's leading digits.  phiG and its fluxes are rounded as they are:
  // both neighbours of a tile seam then see the same FP32 values, the seam
  // fluxes agree bit for bit and the flux form keeps conserving mass.
  const long long tbase = (long long)Y0 * g.P + X0;
  const double *t_us = a.us + mbase + tbase, *t_vs = a.vs + mbase + tbase, *t_ps = a.ps + mbase + tbase;
  const double *t_ph = a.phis + mbase + tbase, *t_sg = a.sqrtG + pbase + tbase;
  const double *t_11 = a.ig11 + pbase + tbase, *t_12 = a.ig12 + pbase + tbase, *t_22 = a.ig22 + pbase + tbase;
  const double *t_yu = a.yu + mbase + tbase, *t_yv = a.yv + mbase + tbase, *t_yp = a.yp + mbase + tbase;
  const float *t_du = a.du + mbase + tbase, *t_dv = a.dv + mbase + tbase, *t_dp = a.dp + mbase + tbase;
  const float *t_p32 = a.phis32 + mbase + tbase;

  // staged field f at loaded point (lx, ly) (TMA form)
  auto stg64 = [&](int f, int lx, int ly) {
    return reinterpret_cast<const double *>(smraw + T::field_off(MIXED, f))[ly * T::BX + lx];
  };
  auto stg32 = [&](int f, int lx, int ly) {
    return reinterpret_cast<const float *>(smraw + T::field_off(MIXED, f))[ly * T::BX + lx];
  };

  // split precision, direct form: the per-tile linear references (two block barriers)
  auto make_planes = [&]() {
    if (threadIdx.x < 3) {
      // reference points (H, H), (txe - 1 + H, H), (H, tye - 1 + H): interior
      const int lx = H + (threadIdx.x == 1 ? txe - 1 : 0), ly = H + (threadIdx.x == 2 ? tye - 1 : 0);
      const int o = ly * g.P + lx;
      double u = __ldg(t_yu + o), v = __ldg(t_yv + o), p = __ldg(t_yp + o);
      const double phs = (double)__ldg(t_p32 + o);
      if constexpr (!first_stage(KIND)) {
        u += (double)__ldg(t_du + o);
        v += (double)__ldg(t_dv + o);
        p += (double)__ldg(t_dp + o);
      }
      MixPoint mp;
      mix_point(mp, a.met1d[X0 + lx], a.met1d[Y0 + ly], u, v, p, phs, phibar, panel, a.two_omega, a.r2);
#pragma unroll
      for (int q = 0; q < 3; ++q) qref[threadIdx.x * 3 + q] = mp.q[q];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      // The derivative added back is FP32, so the plane takes its slope from
      // the rounded value: the two agree to FP64 rounding.
      const int q = threadIdx.x;
      const double q0 = qref[q];
      const float sx = (float)((qref[3 + q] - q0) / ((double)ncx * g.dx));
      const float sy = (float)((qref[6 + q] - q0) / ((double)ncy * g.dx));
      plane[3 * q] = q0;
      plane[3 * q + 1] = (double)sx * (g.dx / (double)(D - 1));  // per point index
      plane[3 * q + 2] = (double)sy * (g.dx / (double)(D - 1));
      slope[q] = sx;
      slope[3 + q] = sy;
    }
    __syncthreads();
  };

  // TMA form, split precision: make_planes from the staged tile, by warp 0
  // alone and without block barriers (the caller's barrier publishes it).
  // The widths' reciprocals replace the division (the slopes are rounded to
  // FP32 anyway and the plane takes its slope from the rounded value).
  auto fit_planes_warp0 = [&]() {
    const int lane = threadIdx.x;
    double q[3] = {0., 0., 0.};
    if (lane < 3) {
      const int lx = H + (lane == 1 ? txe - 1 : 0), ly = H + (lane == 2 ? tye - 1 : 0);
      double u = stg64(0, lx, ly), v = stg64(1, lx, ly), p = stg64(2, lx, ly);
      const double phs = (double)stg32(3, lx, ly);
      if constexpr (!first_stage(KIND)) {
        u += (double)stg32(4, lx, ly);
        v += (double)stg32(5, lx, ly);
        p += (double)stg32(6, lx, ly);
      }
      MixPoint mp;
      mix_point(mp, metx[lx], mety[ly], u, v, p, phs, phibar, panel, a.two_omega, a.r2);
#pragma unroll
      for (int j = 0; j < 3; ++j) q[j] = mp.q[j];
    }
    double r[3][3];  // [reference point][quantity]
#pragma unroll
    for (int pnt = 0; pnt < 3; ++pnt)
#pragma unroll
      for (int j = 0; j < 3; ++j) r[pnt][j] = __shfl_sync(0xffffffffu, q[j], pnt);
    if (lane < 3) {
      const double q0 = (lane == 0) ? r[0][0] : (lane == 1) ? r[0][1] : r[0][2];
      const double qx = (lane == 0) ? r[1][0] : (lane == 1) ? r[1][1] : r[1][2];
      const double qy = (lane == 0) ? r[2][0] : (lane == 1) ? r[2][1] : r[2][2];
      const double iwx = (ncx == CX) ? inv_full_w.x : 1. / ((double)ncx * g.dx);
      const double iwy = (ncy == CY) ? inv_full_w.y : 1. / ((double)ncy * g.dx);
      const float sx = (float)((qx - q0) * iwx);
      const float sy = (float)((qy - q0) * iwy);
      plane[3 * lane] = q0;
      plane[3 * lane + 1] = (double)sx * (g.dx / (double)(D - 1));  // per point index
      plane[3 * lane + 2] = (double)sy * (g.dx / (double)(D - 1));
      slope[lane] = sx;
      slope[3 + lane] = sy;
    }
  };

  // the linear references on column X (split precision; unused in FP64)
  auto column_refs = [&](double X, double *pref) {
    if constexpr (MIXED) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        pref[q] = __fma_rn(plane[3 * q + 1], X, plane[3 * q]);
        pref[3 + q] = plane[3 * q + 2];
      }
    }
  };

  // one loaded point: r = {u, v, phi, phi_s, sqrtG, G^11, G^12, G^22} (FP64
  // policy) or {Y_u, Y_v, Y_phi} with f = {phi_s, d_u, d_v, d_phi} (split)
  // (X, Y) = (lx - H, ly - H) as doubles, the linear references' coordinates
  // pref: the linear references' values on the point's column, {E, u, v} at
  // (X, 0) (pref[0..2]) and their slopes per point index in y (pref[3..5]):
  // the reference at (X, Y) is fma(pref[3+q], Y, pref[q])
  auto point = [&](int idx, int lx, int ly, double Y, const double *pref, const double *r, const float *f,
                   const double4 &mx, const double4 &my) {
    // interior points also keep sqrtG, cU, cV (and f) and form the interface
    // eigenvalues and upwind signs; split precision rounds those to FP32 here
    auto interior = [&](R sg, R cu, R cv, R fc, R g11, R g22, R phi) {
      const int ix = lx - H, iy = ly - H;
      const int ii = iy * T::TX + ix;
      sm[T::SG + ii] = sg;
      sm[T::CU + ii] = cu;
      sm[T::CV + ii] = cv;
      if constexpr (MIXED) {
        // the sweeps form the interface eigenvalues and signs from these
        sm[T::FC + ii] = fc;
        sm[T::GPX + ii] = g11 * phi;
        sm[T::GPY + ii] = g22 * phi;
        return;
      }
      // max(|c - s|, |c + s|) with s = sqrt(G^ii phi) >= 0 is exactly |c| + s
      if (ix % (D - 1) == 0) {
        sm[T::LAMX + iy * (CX + 1) + ix / (D - 1)] = fabs(cu) + sqrt(g11 * phi);
        sm[T::SGNX + iy * (CX + 1) + ix / (D - 1)] = (cu < R(0)) ? R(-1) : R(1);
      }
      if (iy % (D - 1) == 0) {
        sm[T::LAMY + ix * (CY + 1) + iy / (D - 1)] = fabs(cv) + sqrt(g22 * phi);
        sm[T::SGNY + ix * (CY + 1) + iy / (D - 1)] = (cv < R(0)) ? R(-1) : R(1);
      }
    };
    const bool inner = !((lx < H) || (lx >= lxe - H) || (ly < H) || (ly >= lye - H));
    if constexpr (!MIXED) {
      const double u = r[0], v = r[1], phi = r[2], phs = r[3], sg = r[4];
      const double g11 = r[5], g12 = r[6], g22 = r[7];
      const double pg = phi * sg;
      const double cu = g11 * u + g12 * v;  // cov2contrav, projection_mod.F90:138-148
      const double cv = g12 * u + g22 * v;
      sm[T::U + idx] = u;
      sm[T::V + idx] = v;
      sm[T::PG + idx] = pg;
      sm[T::PGU + idx] = pg * cu;
      sm[T::PGV + idx] = pg * cv;
      sm[T::E + idx] = phi + phs + 0.5 * (cu * u + cv * v);  // E = phi + phi_s + K
      if (inner) interior(sg, cu, cv, 0., g11, g22, phi);
    } else {
      double u64 = r[0], v64 = r[1], p64 = r[2];
      if constexpr (!first_stage(KIND)) {
        u64 += (double)f[1];
        v64 += (double)f[2];
        p64 += (double)f[3];
      }
      MixPoint mp;
      mix_point(mp, mx, my, u64, v64, p64, (double)f[0], phibar, panel, a.two_omega, a.r2);
      const float e = (float)(mp.q[0] - __fma_rn(pref[3], Y, pref[0]));
      const float uu = (float)(mp.q[1] - __fma_rn(pref[4], Y, pref[1]));
      const float vv = (float)(mp.q[2] - __fma_rn(pref[5], Y, pref[2]));
      // the mass fluxes as FP32 products of the rounded phiG and winds
      const float pg = (float)mp.q[3], cu = (float)mp.cu, cv = (float)mp.cv;
      float2 *s2 = reinterpret_cast<float2 *>(sm);
      sm[T::U + idx] = uu;
      sm[T::V + idx] = vv;
      s2[T::XF / 2 + idx] = make_float2(e, pg * cu);
      s2[T::XQ / 2 + idx] = make_float2(uu, pg);
      s2[T::YF / 2 + idx] = make_float2(e, pg * cv);
      s2[T::YQ / 2 + idx] = make_float2(vv, pg);
      // split precision keeps 1/sqrtG and sqrtG f for the assembly
      if (inner) interior((float)mp.rsg, cu, cv, (float)(mp.sg * mp.fc), (float)mp.g11, (float)mp.g22, (float)p64);
    }
  };

  if constexpr (TMA) {
    // wait for this item's copies; every thread agrees before anyone leaves
    bool bad;
    if constexpr (MIXED) {
      // warp 0 alone waits, then fits the linear references (lanes 0-2, values
      // exchanged by shuffles); one block barrier publishes both
      bool got = true;
      if (threadIdx.x < 32) {
        got = __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity));
        if constexpr (first_stage(KIND)) {
          // the step's first stage fits the item's references and stores them
          // for the later stages (whose copies bring them in with the tile)
          if (got) {
            fit_planes_warp0();
            __syncwarp();
            if (threadIdx.x < 12) {
              double w;  // one 8-byte word of the record (planes, then the packed slopes)
              memcpy(&w, reinterpret_cast<const char *>(plane) + 8 * threadIdx.x, 8);
              a.prec[((long long)(mem * 6 + panel) * ntile + ty * g.tiles_x + tx) * 12 + threadIdx.x] = w;
            }
          }
        }
      }
      bad = __syncthreads_or(!got);
    } else {
      bad = __syncthreads_or(!mbar_wait_bounded(bar, parity));
    }
    if (bad) {
      if (threadIdx.x == 0) atomicExch(a.err, 1);
      mbar_wait_bounded(bar, parity);  // the copies in flight land before the CTA exits
      return;
    }
    parity ^= 1u;
    // one staged point's input fields
    auto staged = [&](int lx, int ly, double *r, float *f) {
      if constexpr (!MIXED) {
#pragma unroll
        for (int k = 0; k < 8; ++k) r[k] = stg64(k, lx, ly);
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) r[k] = stg64(k, lx, ly);
        f[0] = stg32(3, lx, ly);
        if constexpr (!first_stage(KIND)) {
          f[1] = stg32(4, lx, ly);
          f[2] = stg32(5, lx, ly);
          f[3] = stg32(6, lx, ly);
        }
      }
    };
    if constexpr (ROWMAP) {
      // lane = loaded column, warps stride over the rows: the column's halo
      // flag, interface flags and metric entry are formed once per thread, and
      // a warp reads one staged row (no bank conflicts across rows)
      const int lx = threadIdx.x & 31;
      if (lx < lxe) {
        const bool xh = (lx < H) || (lx >= lxe - H);
        const double4 mx = MIXED ? metx[lx] : double4{};
        double pref[6];  // the column's linear references (OPT bit 2: once per item)
        if constexpr ((OPT & 2) != 0) column_refs((double)(lx - H), pref);
        double Y = (double)((int)(threadIdx.x >> 5) - H);
        for (int ly = threadIdx.x >> 5; ly < lye; ly += NT / 32, Y += (double)(NT / 32)) {
          const bool yh = (ly < H) || (ly >= lye - H);
          if (xh && yh) continue;  // tile corners are never read
          if constexpr ((OPT & 2) == 0) column_refs((double)(lx - H), pref);
          double r[8];
          float f[4];
          staged(lx, ly, r, f);
          point(ly * LX + lx, lx, ly, Y, pref, r, f, mx, MIXED ? mety[ly] : mx);
        }
      }
    } else {
      for (int idx = threadIdx.x; idx < T::A; idx += NT) {
        const int ly = idx / LX, lx = idx - ly * LX;
        const bool xh = (lx < H) || (lx >= lxe - H), yh = (ly < H) || (ly >= lye - H);
        if (lx >= lxe || ly >= lye || (xh && yh)) continue;  // tile corners are never read
        double r[8];
        float f[4];
        staged(lx, ly, r, f);
        const double4 zero{};
        double pref[6];
        column_refs((double)(lx - H), pref);
        point(idx, lx, ly, (double)(ly - H), pref, r, f, MIXED ? metx[lx] : zero, MIXED ? mety[ly] : zero);
      }
    }
  } else {
    constexpr int CH = 3;  // points per thread whose loads are in flight together
    constexpr int NL = MIXED ? 3 : 8;
    for (int base = 0; base < T::A; base += NT * CH) {
      double r[NL][CH];
      float f[4][CH];
      bool ok[CH];
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int idx = base + threadIdx.x + k * NT;
        const int ly = idx / LX, lx = idx - ly * LX;
        const bool xh = (lx < H) || (lx >= lxe - H);
        const bool yh = (ly < H) || (ly >= lye - H);
        ok[k] = idx < T::A && lx < lxe && ly < lye && !(xh && yh);  // tile corners are never read
        if (ok[k]) {
          const int o = ly * g.P + lx;
          if constexpr (!MIXED) {
            r[0][k] = __ldg(t_us + o);
            r[1][k] = __ldg(t_vs + o);
            r[2][k] = __ldg(t_ps + o);
            r[3][k] = __ldg(t_ph + o);
            r[4][k] = __ldg(t_sg + o);
            r[5][k] = __ldg(t_11 + o);
            r[6][k] = __ldg(t_12 + o);
            r[7][k] = __ldg(t_22 + o);
          } else {
            r[0][k] = __ldg(t_yu + o);
            r[1][k] = __ldg(t_yv + o);
            r[2][k] = __ldg(t_yp + o);
            f[0][k] = __ldg(t_p32 + o);
            if constexpr (!first_stage(KIND)) {
              f[1][k] = __ldg(t_du + o);
              f[2][k] = __ldg(t_dv + o);
              f[3][k] = __ldg(t_dp + o);
            }
          }
        }
      }
      if constexpr (MIXED) {
        if (base == 0) {  // block-uniform: runs once, while the first points' loads are in flight
          for (int k = threadIdx.x; k < LX + T::LY; k += NT) {
            const int gidx = (k < LX) ? X0 + k : Y0 + (k - LX);
            if (gidx < g.np) metx[k] = a.met1d[gidx];
          }
          make_planes();
        }
      }
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        if (!ok[k]) continue;
        const int idx = base + threadIdx.x + k * NT;
        const int ly = idx / LX, lx = idx - ly * LX;
        double rr[8];
        float ff[4];
#pragma unroll
        for (int j = 0; j < NL; ++j) rr[j] = r[j][k];
#pragma unroll
        for (int j = 0; j < 4; ++j) ff[j] = f[j][k];
        const double4 zero{};
        double pref[6];
        column_refs((double)(lx - H), pref);
        point(idx, lx, ly, (double)(ly - H), pref, rr, ff, MIXED ? metx[lx] : zero, MIXED ? mety[ly] : zero);
      }
    }
  }
  __syncthreads();
  if constexpr (TMA) {
    // the staging area is free: start the copies of this CTA's next item
    if (threadIdx.x == 0 && wi + wstep < wend) {
      fence_proxy_async();
      issue(wi + wstep);
    }
  }
  const Widths<R> w(g);

  if constexpr (MIXED && WALK > 0 && (OPT & 1) && !last_stage(KIND)) {
    // ---- phase W (split precision), balanced: kind 0 (the (E, phiG c^i)
    // pair with Riemann on (wind component, phiG), packed FP32 pairs) walks
    // segments of WALK cells, kind 1 (dvdx / dudy upwinded by sign(c^i), one
    // quantity) segments of 2 WALK cells, so that every item costs about the
    // same; items: x kind 0, y kind 0, x kind 1, y kind 1 (line fastest)
    constexpr int S0X = WALK < CX ? WALK : CX, S0Y = WALK < CY ? WALK : CY;
    constexpr int S1X = 2 * WALK < CX ? 2 * WALK : CX, S1Y = 2 * WALK < CY ? 2 * WALK : CY;
    constexpr int N0X = (CX + S0X - 1) / S0X, N0Y = (CY + S0Y - 1) / S0Y;
    constexpr int N1X = (CX + S1X - 1) / S1X, N1Y = (CY + S1Y - 1) / S1Y;
    constexpr int E0X = T::TY * N0X, E0Y = E0X + T::TX * N0Y, E1X = E0Y + T::TY * N1X, E1Y = E1X + T::TX * N1Y;
    const float2 *s2 = reinterpret_cast<const float2 *>(sm);
    for (int it = threadIdx.x; it < E1Y; it += NT) {
      if (it < E0X) {
        const int r = it % T::TY, c0 = (it / T::TY) * S0X;
        if (r >= tye || c0 >= ncx) continue;
        const int w0 = (r + H) * LX + c0 * (D - 1);
        float2 *xp = reinterpret_cast<float2 *>(sm + T::XR) + r * T::TX + c0 * (D - 1);
        line_walk2<D, S0X, 1, 1>(s2 + T::XF / 2 + w0, s2 + T::XQ / 2 + w0, EigLam{sm + T::CU + r * T::TX + c0 * (D - 1), sm + T::GPX + r * T::TX + c0 * (D - 1), D - 1},
                                 min(S0X, ncx - c0), c0 + S0X >= ncx, xp, w);
      } else if (it < E0Y) {
        const int j = it - E0X, q = j % T::TX, c0 = (j / T::TX) * S0Y;
        if (q >= txe || c0 >= ncy) continue;
        const int w0 = c0 * (D - 1) * LX + (q + H);
        float2 *yp = reinterpret_cast<float2 *>(sm + T::YR) + q + c0 * (D - 1) * T::TX;
        line_walk2<D, S0Y, LX, T::TX>(s2 + T::YF / 2 + w0, s2 + T::YQ / 2 + w0, EigLam{sm + T::CV + c0 * (D - 1) * T::TX + q, sm + T::GPY + c0 * (D - 1) * T::TX + q, (D - 1) * T::TX},
                                      min(S0Y, ncy - c0), c0 + S0Y >= ncy, yp, w);
      } else if (it < E1X) {
        const int j = it - E0Y, r = j % T::TY, c0 = (j / T::TY) * S1X;
        if (r >= tye || c0 >= ncx) continue;
        const int w0 = (r + H) * LX + c0 * (D - 1);
        R *xr = sm + T::XR + 2 * T::I + r * T::TX + c0 * (D - 1);
        line_walk<D, S1X, 1, 1, true, R>(sm + T::V + w0, sm + T::V + w0, SgnLam{sm + T::CU + r * T::TX + c0 * (D - 1), D - 1},
                                         min(S1X, ncx - c0), c0 + S1X >= ncx, xr, w);
      } else {
        const int j = it - E1X, q = j % T::TX, c0 = (j / T::TX) * S1Y;
        if (q >= txe || c0 >= ncy) continue;
        const int w0 = c0 * (D - 1) * LX + (q + H);
        R *yr = sm + T::YR + 2 * T::I + q + c0 * (D - 1) * T::TX;
        line_walk<D, S1Y, LX, T::TX, true, R>(sm + T::U + w0, sm + T::U + w0, SgnLam{sm + T::CV + c0 * (D - 1) * T::TX + q, (D - 1) * T::TX},
                                              min(S1Y, ncy - c0), c0 + S1Y >= ncy, yr, w);
      }
    }
    __syncthreads();
  } else if constexpr (MIXED && WALK > 0) {
    // ---- phase W (split precision): walks of WALK cells, item = (line,
    // segment, kind); kind 0: the (E, phiG c^i) pair with Riemann on (wind
    // component, phiG); kind 1: dvdx / dudy upwinded by sign(c^i)
    constexpr int SEGX = WALK < CX ? WALK : CX, SEGY = WALK < CY ? WALK : CY;
    constexpr int NSX = (CX + SEGX - 1) / SEGX, NSY = (CY + SEGY - 1) / SEGY;
    const float2 *s2 = reinterpret_cast<const float2 *>(sm);
    for (int it = threadIdx.x; it < 2 * (T::TY * NSX + T::TX * NSY); it += NT) {
      if (it < 2 * T::TY * NSX) {
        const int r = it % T::TY, rest = it / T::TY;
        const int sx = rest % NSX, kk = rest / NSX;
        const int c0 = sx * SEGX;
        if (r >= tye || c0 >= ncx) continue;
        const int nseg = min(SEGX, ncx - c0), w0 = (r + H) * LX + c0 * (D - 1);
        const bool ends = c0 + nseg == ncx;
        R *xr = sm + T::XR + r * T::TX + c0 * (D - 1);
        if (kk == 0)
          line_walk2<D, SEGX, 1, 1>(s2 + T::XF / 2 + w0, s2 + T::XQ / 2 + w0, EigLam{sm + T::CU + r * T::TX + c0 * (D - 1), sm + T::GPX + r * T::TX + c0 * (D - 1), D - 1}, nseg,
                                    ends, reinterpret_cast<float2 *>(sm + T::XR) + r * T::TX + c0 * (D - 1), w);
        else
          line_walk<D, SEGX, 1, 1, true, R>(sm + T::V + w0, sm + T::V + w0, SgnLam{sm + T::CU + r * T::TX + c0 * (D - 1), D - 1}, nseg,
                                            ends, xr + 2 * T::I, w);
      } else {
        const int j = it - 2 * T::TY * NSX;
        const int q = j % T::TX, rest = j / T::TX;
        const int sy = rest % NSY, kk = rest / NSY;
        const int c0 = sy * SEGY;
        if (q >= txe || c0 >= ncy) continue;
        const int nseg = min(SEGY, ncy - c0), w0 = c0 * (D - 1) * LX + (q + H);
        const bool ends = c0 + nseg == ncy;
        R *yr = sm + T::YR + q + c0 * (D - 1) * T::TX;
        if (kk == 0)
          line_walk2<D, SEGY, LX, T::TX>(s2 + T::YF / 2 + w0, s2 + T::YQ / 2 + w0, EigLam{sm + T::CV + c0 * (D - 1) * T::TX + q, sm + T::GPY + c0 * (D - 1) * T::TX + q, (D - 1) * T::TX},
                                         nseg, ends, reinterpret_cast<float2 *>(sm + T::YR) + q + c0 * (D - 1) * T::TX, w);
        else
          line_walk<D, SEGY, LX, T::TX, true, R>(sm + T::U + w0, sm + T::U + w0, SgnLam{sm + T::CV + c0 * (D - 1) * T::TX + q, (D - 1) * T::TX},
                                                 nseg, ends, yr + 2 * T::I, w);
      }
    }
    __syncthreads();
  } else if constexpr (MIXED) {
    // ---- phase X: x-sweep (spatial_operators_mod.F90:63-93), item = (row, cell, kind) ----
    // kind 0: flux_x = d(E)/dx (Riemann on u) and div_x = d(phiG cU)/dx (Riemann
    // on phiG) as one float2 pair; kind 1: dvdx, upwinded by sign(cU)
    const float2 *s2 = reinterpret_cast<const float2 *>(sm);
    for (int it = threadIdx.x; it < T::TY * CX * 2; it += NT) {
      const int r = it % T::TY, rest = it / T::TY;
      const int c = rest % CX, kk = rest / CX;
      if (r >= tye || c >= ncx) continue;
      const int w0 = (r + H) * LX + c * (D - 1);
      const int mmax = (c == ncx - 1) ? D : D - 1;
      R *xr = sm + T::XR + r * T::TX + c * (D - 1);
      if (kk == 0) {
        float2 d[D];
        const EigLam lam{sm + T::CU + r * T::TX + c * (D - 1), sm + T::GPX + r * T::TX + c * (D - 1), D - 1};
        cell_derivs2<D, 1>(d, s2 + T::XF / 2 + w0, s2 + T::XQ / 2 + w0, lam(0), lam(1), w);
        float2 *xp = reinterpret_cast<float2 *>(sm + T::XR) + r * T::TX + c * (D - 1);
#pragma unroll
        for (int m = 0; m < D; ++m)
          if (m < mmax) xp[m] = d[m];
      } else {
        R d[D];
        const SgnLam sgn{sm + T::CU + r * T::TX + c * (D - 1), D - 1};
        cell_derivs<D, 1, R>(d, sm + T::V + w0, sm + T::V + w0, sgn(0), sgn(1), w);
#pragma unroll
        for (int m = 0; m < D; ++m)
          if (m < mmax) xr[2 * T::I + m] = d[m];
      }
    }
    // ---- phase Y: y-sweep (:95-125), item = (column, cell, kind) ----
    // kind 0: flux_y = d(E)/dy (Riemann on v) and div_y = d(phiG cV)/dy; kind 1: dudy
    for (int it = threadIdx.x; it < T::TX * CY * 2; it += NT) {
      const int q = it % T::TX, rest = it / T::TX;
      const int c = rest % CY, kk = rest / CY;
      if (q >= txe || c >= ncy) continue;
      const int w0 = (c * (D - 1)) * LX + (q + H);
      const int mmax = (c == ncy - 1) ? D : D - 1;
      R *yr = sm + T::YR + (c * (D - 1)) * T::TX + q;
      if (kk == 0) {
        float2 d[D];
        const EigLam lam{sm + T::CV + c * (D - 1) * T::TX + q, sm + T::GPY + c * (D - 1) * T::TX + q, (D - 1) * T::TX};
        cell_derivs2<D, LX>(d, s2 + T::YF / 2 + w0, s2 + T::YQ / 2 + w0, lam(0), lam(1), w);
        float2 *yp = reinterpret_cast<float2 *>(sm + T::YR) + (c * (D - 1)) * T::TX + q;
#pragma unroll
        for (int m = 0; m < D; ++m)
          if (m < mmax) yp[m * T::TX] = d[m];
      } else {
        R d[D];
        const SgnLam sgn{sm + T::CV + c * (D - 1) * T::TX + q, (D - 1) * T::TX};
        cell_derivs<D, LX, R>(d, sm + T::U + w0, sm + T::U + w0, sgn(0), sgn(1), w);
#pragma unroll
        for (int m = 0; m < D; ++m)
          if (m < mmax) yr[2 * T::I + m * T::TX] = d[m];
      }
    }
    __syncthreads();
  } else if constexpr (!WALK) {
    // ---- phase X: x-sweep (spatial_operators_mod.F90:63-93), item = (row, cell, quantity) ----
    // quantity 0: flux_x = d(E)/dx, Riemann on u; 1: div_x = d(phiG cU)/dx, Riemann
    // on phiG; 2: dvdx, upwinded by sign(cU)
    for (int it = threadIdx.x; it < T::TY * CX * 3; it += NT) {
      const int r = it % T::TY, rest = it / T::TY;
      const int c = rest % CX, k = rest / CX;
      if (r >= tye || c >= ncx) continue;
      const int w0 = (r + H) * LX + c * (D - 1);
      const int fo = (k == 0) ? T::E : (k == 1) ? T::PGU : T::V;
      const int qo = (k == 0) ? T::U : (k == 1) ? T::PG : T::V;
      const int lo = (k == 2) ? T::SGNX : T::LAMX;
      R d[D];
      cell_derivs<D, 1, R>(d, sm + fo + w0, sm + qo + w0, sm[lo + r * (CX + 1) + c], sm[lo + r * (CX + 1) + c + 1],
                           w);
      R *xr = sm + T::XR + k * T::I + r * T::TX + c * (D - 1);
      const int mmax = (c == ncx - 1) ? D : D - 1;
#pragma unroll
      for (int m = 0; m < D; ++m)
        if (m < mmax) xr[m] = d[m];
    }
    // ---- phase Y: y-sweep (:95-125), item = (column, cell, quantity) ----
    for (int it = threadIdx.x; it < T::TX * CY * 3; it += NT) {
      const int q = it % T::TX, rest = it / T::TX;
      const int c = rest % CY, k = rest / CY;
      if (q >= txe || c >= ncy) continue;
      const int w0 = (c * (D - 1)) * LX + (q + H);
      const int fo = (k == 0) ? T::E : (k == 1) ? T::PGV : T::U;
      const int qo = (k == 0) ? T::V : (k == 1) ? T::PG : T::U;
      const int lo = (k == 2) ? T::SGNY : T::LAMY;
      R d[D];
      cell_derivs<D, LX, R>(d, sm + fo + w0, sm + qo + w0, sm[lo + q * (CY + 1) + c],
                            sm[lo + q * (CY + 1) + c + 1], w);
      R *yr = sm + T::YR + k * T::I + (c * (D - 1)) * T::TX + q;
      const int mmax = (c == ncy - 1) ? D : D - 1;
#pragma unroll
      for (int m = 0; m < D; ++m)
        if (m < mmax) yr[m * T::TX] = d[m];
    }
    __syncthreads();
  } else {
    // ---- phase W: x-walks along rows (spatial_operators_mod.F90:63-93) and
    // y-walks down columns (:95-125), one item per (line, segment of WALK
    // cells, quantity): quantity 0: flux = d(E)/dx^i, Riemann on the covariant
    // wind component; 1: div = d(phiG c^i)/dx^i, Riemann on phiG; 2: dvdx /
    // dudy upwinded by sign(c^i).  A walk forms each interface flux inside its
    // segment once.
    constexpr int SEGX = WALK < CX ? WALK : CX, SEGY = WALK < CY ? WALK : CY;
    constexpr int NSX = (CX + SEGX - 1) / SEGX, NSY = (CY + SEGY - 1) / SEGY;
    for (int it = threadIdx.x; it < 3 * (T::TY * NSX + T::TX * NSY); it += NT) {
      if (it < 3 * T::TY * NSX) {
        const int r = it % T::TY, rest = it / T::TY;
        const int sx = rest % NSX, k = rest / NSX;
        const int c0 = sx * SEGX;
        if (r >= tye || c0 >= ncx) continue;
        const int nseg = min(SEGX, ncx - c0);
        const R *row = sm + (r + H) * LX + c0 * (D - 1);
        R *xr = sm + T::XR + k * T::I + r * T::TX + c0 * (D - 1);
        const ArrLam<R> lam{sm + T::LAMX + r * (CX + 1) + c0};
        const bool ends = c0 + nseg == ncx;
        if (k == 0)
          line_walk<D, SEGX, 1, 1, false, R>(row + T::E, row + T::U, lam, nseg, ends, xr, w);
        else if (k == 1)
          line_walk<D, SEGX, 1, 1, false, R>(row + T::PGU, row + T::PG, lam, nseg, ends, xr, w);
        else
          line_walk<D, SEGX, 1, 1, true, R>(row + T::V, row + T::V, ArrLam<R>{sm + T::SGNX + r * (CX + 1) + c0}, nseg, ends,
                                            xr, w);
      } else {
        const int j = it - 3 * T::TY * NSX;
        const int q = j % T::TX, rest = j / T::TX;
        const int sy = rest % NSY, k = rest / NSY;
        const int c0 = sy * SEGY;
        if (q >= txe || c0 >= ncy) continue;
        const int nseg = min(SEGY, ncy - c0);
        const R *col = sm + (q + H) + c0 * (D - 1) * LX;
        R *yr = sm + T::YR + k * T::I + q + c0 * (D - 1) * T::TX;
        const ArrLam<R> lam{sm + T::LAMY + q * (CY + 1) + c0};
        const bool ends = c0 + nseg == ncy;
        if (k == 0)
          line_walk<D, SEGY, LX, T::TX, false, R>(col + T::E, col + T::V, lam, nseg, ends, yr, w);
        else if (k == 1)
          line_walk<D, SEGY, LX, T::TX, false, R>(col + T::PGV, col + T::PG, lam, nseg, ends, yr, w);
        else
          line_walk<D, SEGY, LX, T::TX, true, R>(col + T::U, col + T::U, ArrLam<R>{sm + T::SGNY + q * (CY + 1) + c0}, nseg,
                                                 ends, yr, w);
      }
    }
    __syncthreads();
  }

  // ---- phase A: tendency assembly (:127-131), RK stage update, store ----
  const bool last_x = (c0x + ncx == g.Nc), last_y = (c0y + ncy == g.Nc);
  const int qown = last_x ? txe : txe - 1;  // seam points belong to the left / lower tile
  const int rown = last_y ? tye : tye - 1;
  // Each thread first loads the global operands of its next CHA points (RK
  // base, accumulators, input increments, Coriolis), so their latencies
  // overlap, then assembles and stores them.
  constexpr int CHA = 2;
  // split precision: the linear references' exact derivatives (E and v along
  // x, E and u along y), the same for every point of the item
  float sl[4] = {0.f, 0.f, 0.f, 0.f};
  if constexpr (MIXED) {
    sl[0] = slope[0];
    sl[1] = slope[2];
    sl[2] = slope[3 + 0];
    sl[3] = slope[3 + 1];
  }
  constexpr bool NEED_BASE = MIXED ? last_stage(KIND) : !first_stage(KIND);
  constexpr bool NEED_ACC = (KIND == RK4_S2 || KIND == RK4_S3 || KIND == RK4_S4);
  constexpr bool NEED_INC = MIXED && (KIND == RK3_S2 || KIND == RK3_S3);
  for (int base0 = 0; base0 < T::I; base0 += NT * CHA) {
    double gb[CHA][3], ga[CHA][3], gf[CHA];
    float gd[CHA][3];
    bool val[CHA];
#pragma unroll
    for (int k = 0; k < CHA; ++k) {
      const int it = base0 + threadIdx.x + k * NT;
      const int r = it / T::TX, q = it - r * T::TX;
      val[k] = it < T::I && q < qown && r < rown;
      if (!val[k]) continue;
      const long long go = mbase + tbase + ((H + r) * g.P + (H + q));
      if constexpr (!MIXED) {
        gf[k] = __ldg(a.fcor + pbase + tbase + ((H + r) * g.P + (H + q)));
        if constexpr (NEED_BASE) {
          gb[k][0] = a.u0[go];
          gb[k][1] = a.v0[go];
          gb[k][2] = a.p0[go];
        }
        if constexpr (NEED_ACC) {
          ga[k][0] = a.aU[go];
          ga[k][1] = a.aV[go];
          ga[k][2] = a.aP[go];
        }
      } else {
        if constexpr (NEED_BASE) {
          gb[k][0] = a.yu[go];
          gb[k][1] = a.yv[go];
          gb[k][2] = a.yp[go];
        }
        if constexpr (NEED_ACC) {
          gd[k][0] = a.fU[go];
          gd[k][1] = a.fV[go];
          gd[k][2] = a.fP[go];
        } else if constexpr (NEED_INC) {
          gd[k][0] = a.du[go];
          gd[k][1] = a.dv[go];
          gd[k][2] = a.dp[go];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < CHA; ++k) {
    if (!val[k]) continue;
    const int it = base0 + threadIdx.x + k * NT;
    const int r = it / T::TX, q = it - r * T::TX;
    const long long go = mbase + tbase + ((H + r) * g.P + (H + q));
    // FP64 policy: SG = sqrtG; split precision: SG = 1/sqrtG, FC = sqrtG f
    const R sg = sm[T::SG + it], cu = sm[T::CU + it], cv = sm[T::CV + it];
    const R fc = MIXED ? sm[T::FC + it] : (R)gf[k];
    const R rsg = MIXED ? sg : R(1) / sg;
    R flux_x, div_x, flux_y, div_y;
    if constexpr (MIXED) {
      const float2 px = reinterpret_cast<const float2 *>(sm + T::XR)[it];
      const float2 py = reinterpret_cast<const float2 *>(sm + T::YR)[it];
      flux_x = px.x;
      div_x = px.y;
      flux_y = py.x;
      div_y = py.y;
    } else {
      flux_x = sm[T::XR + it];
      div_x = sm[T::XR + T::I + it];
      flux_y = sm[T::YR + it];
      div_y = sm[T::YR + T::I + it];
    }
    R dvdx = sm[T::XR + 2 * T::I + it], dudy = sm[T::YR + 2 * T::I + it];
    if constexpr (MIXED) {
      // the linear references' exact derivatives: E and v along x, E and u along y
      flux_x += sl[0];
      dvdx += sl[1];
      flux_y += sl[2];
      dudy += sl[3];
    }
    const R tP = -div_x - div_y;
    R tU, tV;
    if constexpr (MIXED) {
      // sqrtG (vort + f) = (dvdx - dudy) + sqrtG f
      const R ab = (dvdx - dudy) + fc;
      tU = -flux_x + ab * cv;
      tV = -flux_y - ab * cu;
    } else {
      const R vort = (dvdx - dudy) * rsg;
      tU = -flux_x + sg * (vort + fc) * cv;
      tV = -flux_y - sg * (vort + fc) * cu;
    }
    const int sidx = (r + H) * LX + (q + H);
    double uo, vo, po;  // values the boundary copy records
    if constexpr (!MIXED) {
      const double us = sm[T::U + sidx], vs = sm[T::V + sidx], pgs = sm[T::PG + sidx];
      double pgo;
      if constexpr (first_stage(KIND)) {
        uo = us + a.inc * tU;
        vo = vs + a.inc * tV;
        pgo = pgs + a.inc * tP;
        if constexpr (KIND == RK4_S1) {
          a.aU[go] = tU;
          a.aV[go] = tV;
          a.aP[go] = tP;
        }
      } else {
        const double ub = gb[k][0], vb = gb[k][1], pgb = gb[k][2] * sg;
        if constexpr (KIND == RK4_S2 || KIND == RK4_S3) {
          uo = ub + a.inc * tU;
          vo = vb + a.inc * tV;
          pgo = pgb + a.inc * tP;
          a.aU[go] = ga[k][0] + 2. * tU;
          a.aV[go] = ga[k][1] + 2. * tV;
          a.aP[go] = ga[k][2] + 2. * tP;
        } else if constexpr (KIND == RK4_S4) {
          uo = ub + a.inc * ((ga[k][0] + tU) * (1. / 6.));
          vo = vb + a.inc * ((ga[k][1] + tV) * (1. / 6.));
          pgo = pgb + a.inc * ((ga[k][2] + tP) * (1. / 6.));
        } else if constexpr (KIND == RK3_S2) {
          uo = 0.75 * ub + 0.25 * us + a.inc * tU;
          vo = 0.75 * vb + 0.25 * vs + a.inc * tV;
          pgo = 0.75 * pgb + 0.25 * pgs + a.inc * tP;
        } else {  // RK3_S3
          uo = ub * (1. / 3.) + 2. / 3. * us + a.inc * tU;
          vo = vb * (1. / 3.) + 2. / 3. * vs + a.inc * tV;
          pgo = pgb * (1. / 3.) + 2. / 3. * pgs + a.inc * tP;
        }
      }
      po = pgo * rsg;  // phi = phiG / sqrtG, time_scheme_mod.F90:81
      a.uo[go] = uo;
      a.vo[go] = vo;
      a.po[go] = po;
    } else {
      // tendency of phi = (tendency of phiG) / sqrtG
      const float tp = tP * rsg;
      float iu, iv, ip;  // increment over Y
      if constexpr (KIND == RK4_S4) {
        iu = a.wt * ((gd[k][0] + tU) * (1.f / 6.f));
        iv = a.wt * ((gd[k][1] + tV) * (1.f / 6.f));
        ip = a.wt * ((gd[k][2] + tp) * (1.f / 6.f));
      } else {
        iu = a.wt * tU;
        iv = a.wt * tV;
        ip = a.wt * tp;
        if constexpr (KIND == RK3_S2 || KIND == RK3_S3) {
          iu += a.wd * gd[k][0];
          iv += a.wd * gd[k][1];
          ip += a.wd * gd[k][2];
        }
      }
      if constexpr (KIND == RK4_S1) {
        a.fU[go] = tU;
        a.fV[go] = tV;
        a.fP[go] = tp;
      } else if constexpr (KIND == RK4_S2 || KIND == RK4_S3) {
        a.fU[go] = gd[k][0] + 2.f * tU;
        a.fV[go] = gd[k][1] + 2.f * tV;
        a.fP[go] = gd[k][2] + 2.f * tp;
      }
      if constexpr (last_stage(KIND)) {
        // FP64 accumulation of the state into the other state buffer
        uo = gb[k][0] + (double)iu;
        vo = gb[k][1] + (double)iv;
        po = gb[k][2] + (double)ip;
        a.uo[go] = uo;
        a.vo[go] = vo;
        a.po[go] = po;
      } else {
        a.eu[go] = iu;
        a.ev[go] = iv;
        a.ep[go] = ip;
        uo = iu;
        vo = iv;
        po = ip;
      }
    }
    const int gi = X0 + q, gj = Y0 + r;  // 0-based interior indices
    const int nn = g.n;
    if (gi == 0 || gi == nn - 1 || gj == 0 || gj == nn - 1) {
      // pre-unification boundary values for the halo kernel
      const long long bo = ((long long)mem * 6 + panel) * 4 * nn;
      if (!MIXED || last_stage(KIND)) {
        const double4 val = make_double4(uo, vo, po, 0.);
        double4 *b = a.bnd + bo;
        if (gi == 0) b[0 * nn + gj] = val;
        if (gi == nn - 1) b[1 * nn + gj] = val;
        if (gj == 0) b[2 * nn + gi] = val;
        if (gj == nn - 1) b[3 * nn + gi] = val;
      } else {
        const float4 val = make_float4((float)uo, (float)vo, (float)po, 0.f);
        float4 *b = a.bnd32 + bo;
        if (gi == 0) b[0 * nn + gj] = val;
        if (gi == nn - 1) b[1 * nn + gj] = val;
        if (gj == 0) b[2 * nn + gi] = val;
        if (gj == nn - 1) b[3 * nn + gi] = val;
      }
    }
  }
  }
  // (TMA form: no barrier here.  The next item writes the shared arrays only
  // after its own first block barrier, which every thread reaches after this
  // item's phase A; before it, warp 0 writes only the other plane buffer.)
  }
}

// ---------------------------------------------------------------------------
// Launch table of one tile shape (used by the tile-shape autotuner).
// ---------------------------------------------------------------------------
// pdl: launched with programmatic stream serialization (in a step, after a
// halo kernel); the autotuner's back-to-back timing launches go without it
using StageLaunchFn = void (*)(dim3 grid, cudaStream_t s, const StageBatch<1> &b, bool pdl);
using StageBatchFn = void (*)(dim3 grid, cudaStream_t s, const StageBatch<kMaxGrids> &b, bool pdl);

struct StageLauncher {
  int CX, CY, NT, minb;
  int walk;   // 0: sweeps as per-cell items; n: walks of n cells
  bool tma;   // persistent CTAs with TMA-staged tiles
  size_t smem;
  int box_x, box_y;              // staged box of one field (TMA form)
  StageLaunchFn launch[7];       // one grid, indexed by StageKind
  StageLaunchFn launch_ident[7]; // one grid whose active list is the identity
  StageBatchFn launch_batch[7];  // up to kMaxGrids grids in one launch (TMA form; else null)
  cudaError_t (*prepare)();      // raises the dynamic shared-memory limit of every kind
  int (*blocks_per_sm)();        // resident CTAs per SM (sizes the persistent grid)
};

template <int D, int CX, int CY, int NT, int MINB, bool MIXED, int WALK, bool TMA = false, int OPT = 0>
struct StageConfig {
  using T = Tile<D, CX, CY, std::conditional_t<MIXED, float, double>>;
  static constexpr size_t SMEM = TMA ? T::bytes_tma(MIXED) : T::bytes(MIXED);
  // TMA box x coordinates are tile origins X0 = tile * CX * (D - 1): their byte
  // offsets must be multiples of 16 (FP32 fields: X0 % 4 == 0; FP64: even)
  static_assert(!TMA || (CX * (D - 1)) % (MIXED ? 4 : 2) == 0, "TMA box origin not 16-byte aligned");
  // launched with programmatic stream serialization: the kernel's CTAs may
  // become resident while the preceding halo kernel finishes (TMA form: items
  // clear of the panel edges also run then; the rest wait for it)
  template <int KIND, int NB, bool IDENT = false>
  static void launch_nb(dim3 grid, cudaStream_t s, const StageBatch<NB> &b, bool pdl) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, stage_kernel<D, CX, CY, NT, MINB, KIND, MIXED, WALK, TMA, OPT, NB, IDENT>, b);
  }
  template <int KIND>
  static void launch(dim3 grid, cudaStream_t s, const StageBatch<1> &b, bool pdl) {
    launch_nb<KIND, 1>(grid, s, b, pdl);
  }
  template <int KIND>
  static void launch_ident(dim3 grid, cudaStream_t s, const StageBatch<1> &b, bool pdl) {
    launch_nb<KIND, 1, true>(grid, s, b, pdl);
  }
  template <int KIND>
  static void launch_batch(dim3 grid, cudaStream_t s, const StageBatch<kMaxGrids> &b, bool pdl) {
    if constexpr (TMA) launch_nb<KIND, kMaxGrids>(grid, s, b, pdl);
  }
  template <int KIND>
  static cudaError_t attr() {
    // (the driver's own carveout choice: forcing the largest shared-memory
    // carveout shrank L1 and slowed the FP64 kernels by up to 20%)
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<D, CX, CY, NT, MINB, KIND, MIXED, WALK, TMA, OPT, 1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(stage_kernel<D, CX, CY, NT, MINB, KIND, MIXED, WALK, TMA, OPT, 1, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if constexpr (TMA)
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stage_kernel<D, CX, CY, NT, MINB, KIND, MIXED, WALK, TMA, OPT, kMaxGrids>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    return e;
  }
  static cudaError_t prepare() {
    cudaError_t e;
    if ((e = attr<0>()) || (e = attr<1>()) || (e = attr<2>()) || (e = attr<3>()) || (e = attr<4>()) ||
        (e = attr<5>()) || (e = attr<6>()))
      return e;
    return cudaSuccess;
  }
  // resident CTAs per SM (the smallest over the one-grid and the batched forms)
  static int blocks_per_sm() {
    int n = 0, ni = 0, nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, stage_kernel<D, CX, CY, NT, MINB, 1, MIXED, WALK, TMA, OPT, 1>, NT, SMEM) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &ni, stage_kernel<D, CX, CY, NT, MINB, 1, MIXED, WALK, TMA, OPT, 1, true>, NT, SMEM) != cudaSuccess)
      return 0;
    if (ni < n) n = ni;
    if constexpr (TMA) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
              &nb, stage_kernel<D, CX, CY, NT, MINB, 1, MIXED, WALK, TMA, OPT, kMaxGrids>, NT, SMEM) != cudaSuccess)
        return 0;
      return nb < n ? nb : n;
    }
    return n;
  }
  static StageLauncher make() {
    static_assert(SMEM <= 227 * 1024, "tile does not fit in shared memory");
    static_assert(MINB * (SMEM + 1024) <= 228 * 1024, "MINB tiles do not fit in one SM's shared memory");
    StageLauncher L{CX, CY, NT, MINB, WALK, TMA, SMEM, T::BX, T::LY,
                    {&launch<0>, &launch<1>, &launch<2>, &launch<3>, &launch<4>, &launch<5>, &launch<6>},
                    {&launch_ident<0>, &launch_ident<1>, &launch_ident<2>, &launch_ident<3>, &launch_ident<4>,
                     &launch_ident<5>, &launch_ident<6>},
                    {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr}, &prepare, &blocks_per_sm};
    if constexpr (TMA) {
      StageBatchFn fb[7] = {&launch_batch<0>, &launch_batch<1>, &launch_batch<2>, &launch_batch<3>,
                            &launch_batch<4>, &launch_batch<5>, &launch_batch<6>};
      for (int k = 0; k < 7; ++k) L.launch_batch[k] = fb[k];
    }
    return L;
  }
};

// Candidate tile shapes per (order, arithmetic), defined in stage_d{3,4}_{f64,mix}.cu.
const StageLauncher *stage_launchers(int order, bool mixed, int *count);

}  // namespace mcv
