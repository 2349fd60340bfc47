// mcv_kernels.cuh -- sm_100a kernels of one RK stage of MCV_SW.
//
//  stage_kernel   (K1): per panel tile, the whole spatial operator
//                 (src/spatial_operators_mod.F90:12-133) fused with the RK
//                 stage update (src/time_scheme_mod.F90:71-123, the RK4
//                 combine :38-42) and phi = phiG/sqrtG.  Contravariant winds,
//                 phiG, K and E are recomputed from (u, v, phi) in the tile.
//  halo_kernel    (K2): correct_bdy_ghost (src/time_scheme_mod.F90:125-142):
//                 ghost fill with the FP64 edge interpolation
//                 (src/ghost_mod.f90:88-227), boundary unification of the 12
//                 edges and 8 vertices (src/spatial_operators_mod.F90:282-388),
//                 sphere<->panel wind rotations on the strips (:408-492).
//
// Device layout of a padded field: [member][panel][row j][pitch P] with
// padded indices (reference index - ips), P >= npx rounded up to 16 doubles.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

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
  const double *us, *vs, *ps;  // stage input u, v, phi (padded, halo valid)
  const double *u0, *v0, *p0;  // RK base (interior; may alias the outputs)
  double *uo, *vo, *po;        // stage output (interior written here)
  double *aU, *aV, *aP;        // RK4 tendency accumulators
  const double *sqrtG, *ig11, *ig12, *ig22, *fcor;  // metric planes [6][np][P]
  const double *phis;                               // [M][6][np][P]
  double4 *bnd;  // raw boundary copy [M][6][4][n] {u, v, phi, 0}
  double inc;    // dt or dt/2 (update_stat's inc_t) or the RK3 tendency weight
};

struct HaloArgs {
  double *u, *v, *phi;        // state being completed [M][6][np][P]
  const double4 *bnd;         // raw boundary values written by the stage
  const double4 *Mtab;        // A*IG on inside strips [6][4][H+1][n]
  const double4 *Ntab;        // G*IA on outside strips [6][4][H+1][n]
  const int *giref;           // ghost%iref [H][n] (1-based cell)
  const double2 *gcoef;       // {ghost%coef, ghost%coef**3.} [H][n]
  double dx, dx2, dx3;        // dx, dx**2., dx**3.
  int members;
};

// Cube connectivity: panel p's edge e borders panel q's edge e2; rev says the
// position along the edge runs the other way.  Edges: 0 W (i = ids),
// 1 E (i = ide), 2 S (j = jds), 3 N (j = jde).  Derived from
// CubedSphereFillHalo (src/ghost_mod.f90:104-146).
struct EdgeLink {
  int8_t q, e2, rev, pad;
};
// One cube vertex as unify_bdy_field orders its three terms
// (src/spatial_operators_mod.F90:347-386): panel and corner of each term.
// Corners: 0 SW, 1 SE, 2 NW, 3 NE.
struct VertexRef {
  int8_t panel[3], corner[3];
};

__constant__ EdgeLink c_links[6][4];
__constant__ VertexRef c_vertex[6][4];  // indexed by (panel, corner) of the owner

// ---------------------------------------------------------------------------
// One-dimensional MCV building blocks (src/spatial_operators_mod.F90:136-246).
// Divisions by the cell width are multiplications by precomputed reciprocals
// (GridDesc::inv_dx, inv_2dx), one rounding away from the reference's quotient.
// ---------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ double polyfit_left(const double *pv, double inv) {
  // inv = 1/dh (MCV3) or 1/(2 dh) (MCV4)
  if constexpr (D == 3) return -(pv[2] - 4. * pv[1] + 3. * pv[0]) * inv;
  else return (-(11. * pv[0]) + 18. * pv[1] - 9. * pv[2] + 2. * pv[3]) * inv;
}
template <int D>
__device__ __forceinline__ double polyfit_right(const double *pv, double inv) {
  if constexpr (D == 3) return (pv[0] - 4. * pv[1] + 3. * pv[2]) * inv;
  else return (11. * pv[3] - 18. * pv[2] + 9. * pv[1] - 2. * pv[0]) * inv;
}
__device__ __forceinline__ double riemann(double fL, double fR, double qL, double qR, double lam) {
  return 0.5 * ((fL + fR) - lam * (qR - qL));
}

// Derivatives at the D points of the centre cell of a 3-cell window
// (3D-2 values with stride S): calc_tendP, src/spatial_operators_mod.F90:136-202.
template <int D, int S>
__device__ __forceinline__ void cell_derivs(double out[D], const double *f, const double *q, double lamL,
                                            double lamR, const GridDesc &g) {
  const double ip = (D == 3) ? g.inv_dx : g.inv_2dx;
  double c1[D], c2[D], c3[D], d1[D], d2[D], d3[D];
#pragma unroll
  for (int m = 0; m < D; ++m) {
    c1[m] = f[m * S];
    c2[m] = f[(D - 1 + m) * S];
    c3[m] = f[(2 * D - 2 + m) * S];
    d1[m] = q[m * S];
    d2[m] = q[(D - 1 + m) * S];
    d3[m] = q[(2 * D - 2 + m) * S];
  }
  const double fxL1 = polyfit_right<D>(c1, ip), fxL2 = polyfit_right<D>(c2, ip);
  const double fxR1 = polyfit_left<D>(c2, ip), fxR2 = polyfit_left<D>(c3, ip);
  const double qxL1 = polyfit_right<D>(d1, ip), qxL2 = polyfit_right<D>(d2, ip);
  const double qxR1 = polyfit_left<D>(d2, ip), qxR2 = polyfit_left<D>(d3, ip);
  out[0] = riemann(fxL1, fxR1, qxL1, qxR1, lamL);
  out[D - 1] = riemann(fxL2, fxR2, qxL2, qxR2, lamR);
  if constexpr (D == 3) {
    const double fxVIA = (c2[2] - c2[0]) * g.inv_dx;
    out[1] = 1.5 * fxVIA - 0.25 * (out[0] + out[2]);
  } else {
    const double fxVIA = (c2[3] - c2[0]) * g.inv_dx;
    const double fxxc = 4.5 * (c2[0] - c2[1] - c2[2] + c2[3]) * g.inv_dx2;
    out[1] = 4. / 3. * fxVIA - (4. * out[0] + 5. * out[3]) / 27. - 4. / 27. * g.dx * fxxc;
    out[2] = 4. / 3. * fxVIA - (5. * out[0] + 4. * out[3]) / 27. + 4. / 27. * g.dx * fxxc;
  }
}

// ---------------------------------------------------------------------------
// K1: fused spatial operator + RK stage on one tile of CX x CY cells.
// ---------------------------------------------------------------------------
template <int D, int CX, int CY>
struct Tile {
  static constexpr int H = D - 1;
  static constexpr int TX = CX * (D - 1) + 1;  // tile points per row (max)
  static constexpr int TY = CY * (D - 1) + 1;
  static constexpr int LX = TX + 2 * H;        // loaded row length (odd: no bank conflicts on column walks)
  static constexpr int LY = TY + 2 * H;
  static constexpr int A = LX * LY;
  static constexpr int I = TX * TY;
  // shared-memory carve (doubles)
  static constexpr int U = 0, V = A, E = 2 * A, PG = 3 * A, PGU = 4 * A, PGV = 5 * A, CU = 6 * A, CV = 7 * A,
                       SG = 8 * A;
  static constexpr int LAMX = 9 * A;                 // [TY][CX+1]
  static constexpr int SGNX = LAMX + TY * (CX + 1);
  static constexpr int LAMY = SGNX + TY * (CX + 1);  // [TX][CY+1]
  static constexpr int SGNY = LAMY + TX * (CY + 1);
  static constexpr int XR = SGNY + TX * (CY + 1);    // x-sweep results [3][TY][TX]
  static constexpr int YR = XR + 3 * I;              // y-sweep results [3][TY][TX]
  static constexpr int TOTAL = YR + 3 * I;
  static constexpr size_t BYTES = (size_t)TOTAL * sizeof(double);
  static_assert(LX % 2 == 1, "odd shared row length");
};

template <int D, int CX, int CY, int NT, int KIND>
__global__ void __launch_bounds__(NT) stage_kernel(const GridDesc g, const StageArgs a) {
  using T = Tile<D, CX, CY>;
  constexpr int H = T::H, LX = T::LX;
  extern __shared__ double sm[];
  const int tile = blockIdx.x, panel = blockIdx.y, mem = blockIdx.z;
  const int tx = tile % g.tiles_x, ty = tile / g.tiles_x;
  const int c0x = tx * CX, c0y = ty * CY;
  const int ncx = min(CX, g.Nc - c0x), ncy = min(CY, g.Nc - c0y);
  const int X0 = c0x * (D - 1), Y0 = c0y * (D - 1);  // padded coords of the first loaded point
  const int lxe = ncx * (D - 1) + 1 + 2 * H, lye = ncy * (D - 1) + 1 + 2 * H;
  const long long pbase = (long long)panel * g.plane;
  const long long mbase = (long long)mem * g.mstride + pbase;

  // ---- phase 0: load the tile and its halo cross, pointwise quantities ----
  // (spatial_operators_mod.F90:58-61, eigenvalues :248-280, upwind signs :83-85)
  {
    constexpr int PPT = (T::A + NT - 1) / NT;
    double ru[PPT], rv[PPT], rp[PPT], rs[PPT], r11[PPT], r12[PPT], r22[PPT], rh[PPT];
    bool ok[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      const int idx = threadIdx.x + k * NT;
      const int ly = idx / LX, lx = idx - ly * LX;
      const bool xh = (lx < H) || (lx >= lxe - H);
      const bool yh = (ly < H) || (ly >= lye - H);
      ok[k] = idx < T::A && lx < lxe && ly < lye && !(xh && yh);  // tile corners are never read
      if (ok[k]) {
        const long long go = (long long)(Y0 + ly) * g.P + (X0 + lx);
        ru[k] = __ldg(a.us + mbase + go);
        rv[k] = __ldg(a.vs + mbase + go);
        rp[k] = __ldg(a.ps + mbase + go);
        rh[k] = __ldg(a.phis + mbase + go);
        rs[k] = __ldg(a.sqrtG + pbase + go);
        r11[k] = __ldg(a.ig11 + pbase + go);
        r12[k] = __ldg(a.ig12 + pbase + go);
        r22[k] = __ldg(a.ig22 + pbase + go);
      }
    }
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      if (!ok[k]) continue;
      const int idx = threadIdx.x + k * NT;
      const int ly = idx / LX, lx = idx - ly * LX;
      const double u = ru[k], v = rv[k], phi = rp[k], sg = rs[k], g11 = r11[k], g12 = r12[k], g22 = r22[k];
      const double cu = g11 * u + g12 * v;  // cov2contrav, projection_mod.F90:138-148
      const double cv = g12 * u + g22 * v;
      const double pg = phi * sg;
      const double K = 0.5 * (cu * u + cv * v);
      sm[T::U + idx] = u;
      sm[T::V + idx] = v;
      sm[T::CU + idx] = cu;
      sm[T::CV + idx] = cv;
      sm[T::PG + idx] = pg;
      sm[T::PGU + idx] = pg * cu;
      sm[T::PGV + idx] = pg * cv;
      sm[T::E + idx] = phi + rh[k] + K;
      sm[T::SG + idx] = sg;
      const bool xh = (lx < H) || (lx >= lxe - H), yh = (ly < H) || (ly >= lye - H);
      if (!xh && !yh) {
        const int ix = lx - H, iy = ly - H;
        // max(|c - s|, |c + s|) with s = sqrt(G^ii phi) >= 0 is exactly |c| + s
        if (ix % (D - 1) == 0) {
          sm[T::LAMX + iy * (CX + 1) + ix / (D - 1)] = fabs(cu) + sqrt(g11 * phi);
          sm[T::SGNX + iy * (CX + 1) + ix / (D - 1)] = (cu < 0.) ? -1. : 1.;
        }
        if (iy % (D - 1) == 0) {
          sm[T::LAMY + ix * (CY + 1) + iy / (D - 1)] = fabs(cv) + sqrt(g22 * phi);
          sm[T::SGNY + ix * (CY + 1) + iy / (D - 1)] = (cv < 0.) ? -1. : 1.;
        }
      }
    }
  }
  __syncthreads();

  const int txe = ncx * (D - 1) + 1, tye = ncy * (D - 1) + 1;

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
    double d[D];
    cell_derivs<D, 1>(d, sm + fo + w0, sm + qo + w0, sm[lo + r * (CX + 1) + c], sm[lo + r * (CX + 1) + c + 1], g);
    double *xr = sm + T::XR + k * T::I + r * T::TX + c * (D - 1);
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
    double d[D];
    cell_derivs<D, LX>(d, sm + fo + w0, sm + qo + w0, sm[lo + q * (CY + 1) + c], sm[lo + q * (CY + 1) + c + 1], g);
    double *yr = sm + T::YR + k * T::I + (c * (D - 1)) * T::TX + q;
    const int mmax = (c == ncy - 1) ? D : D - 1;
#pragma unroll
    for (int m = 0; m < D; ++m)
      if (m < mmax) yr[m * T::TX] = d[m];
  }
  __syncthreads();

  // ---- phase A: tendency assembly (:127-131), RK stage update, store ----
  const bool last_x = (c0x + ncx == g.Nc), last_y = (c0y + ncy == g.Nc);
  const int qown = last_x ? txe : txe - 1;  // seam points belong to the left / lower tile
  const int rown = last_y ? tye : tye - 1;
  for (int it = threadIdx.x; it < T::I; it += NT) {
    const int r = it / T::TX, q = it - r * T::TX;
    if (q >= qown || r >= rown) continue;
    const long long go = (long long)(Y0 + H + r) * g.P + (X0 + H + q);
    const double fc = __ldg(a.fcor + pbase + go);
    double ub = 0., vb = 0., pb = 0., aU = 0., aV = 0., aP = 0.;
    if constexpr (KIND != RK3_S1 && KIND != RK4_S1) {
      ub = a.u0[mbase + go];
      vb = a.v0[mbase + go];
      pb = a.p0[mbase + go];
    }
    if constexpr (KIND == RK4_S2 || KIND == RK4_S3 || KIND == RK4_S4) {
      aU = a.aU[mbase + go];
      aV = a.aV[mbase + go];
      aP = a.aP[mbase + go];
    }
    const int sidx = (r + H) * LX + (q + H);
    const int ridx = r * T::TX + q;
    const double sg = sm[T::SG + sidx], cu = sm[T::CU + sidx], cv = sm[T::CV + sidx];
    const double rsg = 1. / sg;
    const double flux_x = sm[T::XR + ridx], div_x = sm[T::XR + T::I + ridx], dvdx = sm[T::XR + 2 * T::I + ridx];
    const double flux_y = sm[T::YR + ridx], div_y = sm[T::YR + T::I + ridx], dudy = sm[T::YR + 2 * T::I + ridx];
    const double vort = (dvdx - dudy) * rsg;
    const double tP = -div_x - div_y;
    const double tU = -flux_x + sg * (vort + fc) * cv;
    const double tV = -flux_y - sg * (vort + fc) * cu;
    const double us = sm[T::U + sidx], vs = sm[T::V + sidx], pgs = sm[T::PG + sidx];
    double uo, vo, pgo;
    if constexpr (KIND == RK3_S1 || KIND == RK4_S1) {
      uo = us + a.inc * tU;
      vo = vs + a.inc * tV;
      pgo = pgs + a.inc * tP;
      if constexpr (KIND == RK4_S1) {
        a.aU[mbase + go] = tU;
        a.aV[mbase + go] = tV;
        a.aP[mbase + go] = tP;
      }
    } else {
      const double pgb = pb * sg;
      if constexpr (KIND == RK4_S2 || KIND == RK4_S3) {
        uo = ub + a.inc * tU;
        vo = vb + a.inc * tV;
        pgo = pgb + a.inc * tP;
        a.aU[mbase + go] = aU + 2. * tU;
        a.aV[mbase + go] = aV + 2. * tV;
        a.aP[mbase + go] = aP + 2. * tP;
      } else if constexpr (KIND == RK4_S4) {
        uo = ub + a.inc * ((aU + tU) * (1. / 6.));
        vo = vb + a.inc * ((aV + tV) * (1. / 6.));
        pgo = pgb + a.inc * ((aP + tP) * (1. / 6.));
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
    const double po = pgo * rsg;  // phi = phiG / sqrtG, time_scheme_mod.F90:81
    a.uo[mbase + go] = uo;
    a.vo[mbase + go] = vo;
    a.po[mbase + go] = po;
    const int gi = X0 + q, gj = Y0 + r;  // 0-based interior indices
    const int nn = g.n;
    if (gi == 0 || gi == nn - 1 || gj == 0 || gj == nn - 1) {
      // pre-unification boundary values for the halo kernel
      const double4 val = make_double4(uo, vo, po, 0.);
      double4 *b = a.bnd + ((long long)mem * 6 + panel) * 4 * nn;
      if (gi == 0) b[0 * nn + gj] = val;
      if (gi == nn - 1) b[1 * nn + gj] = val;
      if (gj == 0) b[2 * nn + gi] = val;
      if (gj == nn - 1) b[3 * nn + gi] = val;
    }
  }
}

// ---------------------------------------------------------------------------
// K2: ghost fill + boundary unification for one (member, panel, edge, position).
// ---------------------------------------------------------------------------

// Interior-relative coordinates (0-based, may be negative in the halo) of the
// point at signed inside-distance d from edge e at position k along it.
__device__ __forceinline__ void strip_point(int e, int d, int k, int n, int &i, int &j) {
  switch (e) {
    case 0: i = d; j = k; break;
    case 1: i = n - 1 - d; j = k; break;
    case 2: i = k; j = d; break;
    default: i = k; j = n - 1 - d; break;
  }
}

// Raw (pre-unification) value of a boundary point (i, j) of panel q.
__device__ __forceinline__ double4 raw_boundary(const double4 *bnd_q, int i, int j, int n) {
  if (j == 0) return bnd_q[2 * n + i];
  if (j == n - 1) return bnd_q[3 * n + i];
  if (i == 0) return bnd_q[0 * n + j];
  return bnd_q[1 * n + j];
}

// linear_interp, src/ghost_mod.f90:183-227
template <int D>
__device__ __forceinline__ double ghost_interp(const double *q, double coef, double coef3, double dx, double dx2,
                                               double dx3) {
  if constexpr (D == 3) {
    return q[0] - (3. * q[0] - 4. * q[1] + q[2]) * coef / dx + 2. * (q[0] - 2. * q[1] + q[2]) * (coef * coef) / dx2;
  } else {
    return (2. * dx3 * q[0] + dx2 * (-(11. * q[0]) + 18. * q[1] - 9. * q[2] + 2. * q[3]) * coef +
            9. * dx * (2. * q[0] - 5. * q[1] + 4. * q[2] - q[3]) * (coef * coef) +
            9. * (-q[0] + 3. * q[1] - 3. * q[2] + q[3]) * coef3) /
           (2. * dx3);
  }
}

template <int D>
__global__ void __launch_bounds__(128) halo_kernel(const GridDesc g, const HaloArgs a) {
  constexpr int H = D - 1;
  const int n = g.n;
  // one thread per (member, panel, edge, halo line h = 0..H, position k)
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_member = 24LL * (H + 1) * n;
  if (gid >= per_member * a.members) return;
  const int mem = (int)(gid / per_member);
  int rem = (int)(gid - (long long)mem * per_member);
  const int k = rem % n;
  rem /= n;
  const int h = rem % (H + 1);
  const int pe = rem / (H + 1);
  const int p = pe / 4, e = pe % 4;
  const EdgeLink L = c_links[p][e];
  const int q = L.q, e2 = L.e2;
  const long long mb = (long long)mem * g.mstride;
  const double4 *bnd_m = a.bnd + (long long)mem * 24 * n;

  double zw, mw, ph;
  if (h > 0) {
    // halo line h: neighbour line h rotated to the sphere, interpolated along
    // the edge, rotated back to this panel (ghost_mod.f90:154-181)
    const int iref = a.giref[(h - 1) * n + k];
    const double2 cc = a.gcoef[(h - 1) * n + k];
    double qz[D], qm[D], qp[D];
#pragma unroll
    for (int m = 0; m < D; ++m) {
      const int kk = (iref - 1) * (D - 1) + m;
      const int ks = L.rev ? n - 1 - kk : kk;
      int si, sj;
      strip_point(e2, h, ks, n, si, sj);
      double su, sv, sp;
      if (ks == 0 || ks == n - 1) {
        const double4 b = raw_boundary(bnd_m + q * 4 * n, si, sj, n);
        su = b.x; sv = b.y; sp = b.z;
      } else {
        const long long o = mb + q * g.plane + (long long)(sj + H) * g.P + (si + H);
        su = a.u[o]; sv = a.v[o]; sp = a.phi[o];
      }
      const double4 M = a.Mtab[((q * 4 + e2) * (H + 1) + h) * n + ks];
      qz[m] = M.x * su + M.z * sv;  // covProjPlane2Sphere, projection_mod.F90:79-96
      qm[m] = M.y * su + M.w * sv;
      qp[m] = sp;
    }
    zw = ghost_interp<D>(qz, cc.x, cc.y, a.dx, a.dx2, a.dx3);
    mw = ghost_interp<D>(qm, cc.x, cc.y, a.dx, a.dx2, a.dx3);
    ph = ghost_interp<D>(qp, cc.x, cc.y, a.dx, a.dx2, a.dx3);
  } else if (k > 0 && k < n - 1) {
    // boundary line: edge average (spatial_operators_mod.F90:298-345)
    const int ks = L.rev ? n - 1 - k : k;
    const double4 bo = bnd_m[(p * 4 + e) * n + k];
    const double4 bn = bnd_m[(q * 4 + e2) * n + ks];
    const double4 Mo = a.Mtab[((p * 4 + e) * (H + 1) + 0) * n + k];
    const double4 Mn = a.Mtab[((q * 4 + e2) * (H + 1) + 0) * n + ks];
    zw = 0.5 * ((Mo.x * bo.x + Mo.z * bo.y) + (Mn.x * bn.x + Mn.z * bn.y));
    mw = 0.5 * ((Mo.y * bo.x + Mo.w * bo.y) + (Mn.y * bn.x + Mn.w * bn.y));
    ph = 0.5 * (bo.z + bn.z);
  } else if (e <= 1) {
    // cube vertex (:347-386), owned by the W/E edge threads
    const int corner = (e == 0) ? (k == 0 ? 0 : 2) : (k == 0 ? 1 : 3);
    const VertexRef V = c_vertex[p][corner];
    double z[3], mm[3], pp[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const int pt = V.panel[t], ct = V.corner[t];
      const int et = (ct == 0 || ct == 2) ? 0 : 1;  // W or E column holds the corner
      const int kt = (ct <= 1) ? 0 : n - 1;
      const double4 b = bnd_m[(pt * 4 + et) * n + kt];
      const double4 M = a.Mtab[((pt * 4 + et) * (H + 1) + 0) * n + kt];
      z[t] = M.x * b.x + M.z * b.y;
      mm[t] = M.y * b.x + M.w * b.y;
      pp[t] = b.z;
    }
    zw = (z[0] + z[1] + z[2]) / 3.;
    mw = (mm[0] + mm[1] + mm[2]) / 3.;
    ph = (pp[0] + pp[1] + pp[2]) / 3.;
  } else {
    return;
  }
  // back to this panel's covariant winds (covProjSphere2Plane, :459-492)
  const double4 N = a.Ntab[((p * 4 + e) * (H + 1) + h) * n + k];
  int di, dj;
  strip_point(e, -h, k, n, di, dj);
  const long long o = mb + p * g.plane + (long long)(dj + H) * g.P + (di + H);
  a.u[o] = N.x * zw + N.z * mw;
  a.v[o] = N.y * zw + N.w * mw;
  a.phi[o] = ph;
}

// ---------------------------------------------------------------------------
// Mass / energy (src/diag_mod.F90:10-67): per-cell sums in the reference's
// order, then a compensated (Neumaier) sum over cells.
// ---------------------------------------------------------------------------
struct KSum {
  double s, c;
};
__device__ __forceinline__ void neumaier_add(KSum &a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
  else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void ksum_merge(KSum &a, const KSum &b) {
  neumaier_add(a, b.s);
  a.c += b.c;
}

template <int D>
__global__ void __launch_bounds__(256) mass_energy_kernel(const GridDesc g, const double *u, const double *v,
                                                          const double *phi, const double *sqrtG,
                                                          const double *ig11, const double *ig12,
                                                          const double *ig22, const double *phis, double w1d0,
                                                          double w1d1, double wden, double4 *partial) {
  constexpr int H = D - 1;
  const int Nc = g.Nc;
  const long long ncell = 6LL * Nc * Nc;
  KSum ms{0., 0.}, es{0., 0.};
  for (long long cidx = (long long)blockIdx.x * blockDim.x + threadIdx.x; cidx < ncell;
       cidx += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(cidx / ((long long)Nc * Nc));
    const int rem = (int)(cidx - (long long)p * Nc * Nc);
    const int jc = rem / Nc, ic = rem % Nc;
    double mc = 0., ec = 0.;
    for (int jd = 0; jd < D; ++jd)
      for (int id = 0; id < D; ++id) {
        // weightsOnPV (mesh_mod.F90:183-203): outer product of (1,4,1)/36 or (1,3,3,1)/80
        const double wi = (id == 0 || id == D - 1) ? w1d0 : w1d1;
        const double wj = (jd == 0 || jd == D - 1) ? w1d0 : w1d1;
        const double w = wi * wj / wden;
        const long long o = (long long)p * g.plane + (long long)(jc * (D - 1) + jd + H) * g.P + (ic * (D - 1) + id + H);
        const double sg = sqrtG[o], ph = phi[o], uu = u[o], vv = v[o];
        const double cu = ig11[o] * uu + ig12[o] * vv, cv = ig12[o] * uu + ig22[o] * vv;
        mc = mc + w * (ph * sg);
        const double KE = 0.5 * ph * (uu * cu + vv * cv);
        const double PE = 0.5 * ((ph + phis[o]) * (ph + phis[o]));
        ec = ec + w * sg * (KE + PE);
      }
    neumaier_add(ms, mc);
    neumaier_add(es, ec);
  }
  // block reduction of (sum, compensation) pairs
  __shared__ KSum red_m[256], red_e[256];
  red_m[threadIdx.x] = ms;
  red_e[threadIdx.x] = es;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      ksum_merge(red_m[threadIdx.x], red_m[threadIdx.x + s]);
      ksum_merge(red_e[threadIdx.x], red_e[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double4(red_m[0].s, red_m[0].c, red_e[0].s, red_e[0].c);
}

}  // namespace mcv
