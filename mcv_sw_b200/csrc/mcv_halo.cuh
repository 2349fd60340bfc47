// mcv_halo.cuh -- halo/boundary kernel (K2) and diagnostics of MCV_SW.
#pragma once
#include "mcv_ksum.cuh"
#include "mcv_stage.cuh"

namespace mcv {

struct HaloArgs {
  double *u, *v, *phi;        // state being completed [M][6][np][P]
  const double4 *bnd;         // raw boundary values written by the stage
  const double4 *Mtab;        // A*IG on inside strips [6][4][H+1][n]
  const double4 *Ntab;        // G*IA on outside strips [6][4][H+1][n]
  const int *giref;           // ghost%iref [H][n] (1-based cell)
  const double2 *gcoef;       // {ghost%coef, ghost%coef**3.} [H][n]
  double dx, dx2, dx3;        // dx, dx**2., dx**3.
  double rdx, rdx2, r2dx3;    // 1/dx, 1/dx**2., 1/(2 dx**3.)
  int members;                // active members in this launch
  const int *active;          // member index of each active slot [members]
  int ident;                  // 1 when active[k] == k for every slot: the slot is the member
  // split precision: the field completed is Y + increment; u/v/phi above are
  // Y (read only), the increment's halo and boundary are written instead
  float *du, *dv, *dp;
  const float4 *bnd32;
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
// K2: ghost fill + boundary unification for one (member, panel, edge, line, position).
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

// Index (edge * n + position) of the raw copy of boundary point (i, j).
__device__ __forceinline__ int boundary_slot(int i, int j, int n) {
  if (j == 0) return 2 * n + i;
  if (j == n - 1) return 3 * n + i;
  if (i == 0) return 0 * n + j;
  return 1 * n + j;
}

// linear_interp, src/ghost_mod.f90:183-227.  The divisions by dx, dx**2 and
// 2 dx**3 are multiplications by their reciprocals (one rounding away from
// the reference's quotients, as the stage kernel's cell widths are).
template <int D>
__device__ __forceinline__ double ghost_interp(const double *q, double coef, double coef3, const HaloArgs &a) {
  if constexpr (D == 3) {
    return q[0] - (3. * q[0] - 4. * q[1] + q[2]) * coef * a.rdx +
           2. * (q[0] - 2. * q[1] + q[2]) * (coef * coef) * a.rdx2;
  } else {
    return (2. * a.dx3 * q[0] + a.dx2 * (-(11. * q[0]) + 18. * q[1] - 9. * q[2] + 2. * q[3]) * coef +
            9. * a.dx * (2. * q[0] - 5. * q[1] + 4. * q[2] - q[3]) * (coef * coef) +
            9. * (-q[0] + 3. * q[1] - 3. * q[2] + q[3]) * coef3) *
           a.r2dx3;
  }
}

// The grids one halo launch completes: one, or the grids of a batched stage
// launch (each with its own threads, numbered from first[k]).
template <int NB>
struct HaloBatch {
  GridDesc g[NB];
  HaloArgs a[NB];
  int first[NB + 1];  // first member slot (blockIdx.z) of each grid
  int ngrids;
};

// Positions along an edge per block, and the window of neighbour positions a
// block stages per halo line.  The interpolation stencil of the ghost point at
// position k starts at neighbour position (iref - 1)(D - 1), within [k - 6,
// k + 2] on every line of the equiangular grids (checked for Nc = 8 to 1024,
// both orders), so the window
// [k0 - kHaloLead, k0 - kHaloLead + kHaloWin) of a segment starting at k0
// holds all of its stencils without reading iref first; a stencil point
// outside the window is read from global memory instead.
constexpr int kHaloSeg = 64, kHaloLead = 8, kHaloWin = kHaloSeg + 16;

// MIXED: the field completed is Y + increment.  Raw values combine Y with the
// increment in FP64; the result minus Y at the destination is stored as the
// new FP32 increment, so the next stage's input halo is the FP64 correction
// of its own interior.
//
// One block per (segment of kHaloSeg positions: x; panel and edge: y; grid and
// active member: z), one thread per (position, line h = 0..H), positions
// fastest so that a warp shares its line.  The block first stages the
// neighbour's lines 1..H over the segment's window -- each point loaded once,
// completed and rotated to the sphere once, with the loads coalesced along
// the neighbour's rows (lines fastest on a W/E neighbour edge, whose lines are
// columns) -- then interpolates the ghost points from shared memory.
template <int D, bool MIXED, int NB>
__global__ void __launch_bounds__(kHaloSeg * D) halo_kernel(const __grid_constant__ HaloBatch<NB> hb) {
  constexpr int H = D - 1;
  constexpr int NT = kHaloSeg * (H + 1);
  // the staged neighbour lines 1..H: {zonal, meridional, phi} on the sphere
  __shared__ double wz[H][kHaloWin], wm[H][kHaloWin], wp[H][kHaloWin];
  const int z = blockIdx.z;
  int kg = 0;
#pragma unroll
  for (int j = 1; j < NB; ++j)
    if (j < hb.ngrids && z >= hb.first[j]) kg = j;
  const GridDesc &g = hb.g[kg];
  const HaloArgs &a = hb.a[kg];
  const int n = g.n;
  const int k0 = blockIdx.x * kHaloSeg;
  if (k0 >= n) return;  // block-uniform: the grid is sized for the batch's largest grid
  const int slot = z - hb.first[kg];
  const int mem = active_member(a.active, a.ident, slot);
  const int p = blockIdx.y >> 2, e = blockIdx.y & 3;
  const EdgeLink L = c_links[p][e];
  const int q = L.q, e2 = L.e2;
  const long long mb = (long long)mem * g.mstride;
  const long long bb = (long long)mem * 24 * n;
  const int h = threadIdx.x / kHaloSeg;      // this thread's line
  const int k = k0 + threadIdx.x % kHaloSeg;  // and position
  const bool live = k < n;

  // raw (pre-unification) value of boundary point (i, j) of panel pp
  auto raw_boundary = [&](int pp, int i, int j, double &su, double &sv, double &sp) {
    const int slot = boundary_slot(i, j, n);
    if constexpr (!MIXED) {
      const double4 b = a.bnd[bb + pp * 4 * n + slot];
      su = b.x; sv = b.y; sp = b.z;
    } else {
      const float4 b = a.bnd32[bb + pp * 4 * n + slot];
      const long long o = mb + pp * g.plane + (long long)(j + H) * g.P + (i + H);
      su = a.u[o] + (double)b.x; sv = a.v[o] + (double)b.y; sp = a.phi[o] + (double)b.z;
    }
  };
  // the completed field at position kk of the neighbour's line hh (1..H),
  // rotated to the sphere (covProjPlane2Sphere, projection_mod.F90:79-96).  A
  // point at an end of the line is a boundary point and takes its raw copy;
  // the FP64 form, whose boundary this kernel rewrites, reads no state there.
  auto neighbour = [&](int hh, int kk, double &zq, double &mq, double &pq) {
    const int ks = L.rev ? n - 1 - kk : kk;
    const bool isb = (ks == 0 || ks == n - 1);
    int si, sj;
    strip_point(e2, hh, ks, n, si, sj);
    const double4 M = a.Mtab[((q * 4 + e2) * (H + 1) + hh) * n + ks];
    double su, sv, sp;
    if constexpr (MIXED) {
      const long long os = mb + q * g.plane + (long long)(sj + H) * g.P + (si + H);
      const double yu = a.u[os], yv = a.v[os], yp = a.phi[os];
      float du, dv, dp;
      if (isb) {
        const float4 b = a.bnd32[bb + q * 4 * n + boundary_slot(si, sj, n)];
        du = b.x; dv = b.y; dp = b.z;
      } else {
        du = a.du[os]; dv = a.dv[os]; dp = a.dp[os];
      }
      su = yu + (double)du;
      sv = yv + (double)dv;
      sp = yp + (double)dp;
    } else if (isb) {
      const double4 b = a.bnd[bb + q * 4 * n + boundary_slot(si, sj, n)];
      su = b.x; sv = b.y; sp = b.z;
    } else {
      const long long os = mb + q * g.plane + (long long)(sj + H) * g.P + (si + H);
      su = a.u[os]; sv = a.v[os]; sp = a.phi[os];
    }
    zq = M.x * su + M.z * sv;
    mq = M.y * su + M.w * sv;
    pq = sp;
  };

  // this thread's destination, its rotation back and (split precision) the Y
  // it corrects; the interpolation weights of a ghost line
  int di = 0, dj = 0;
  long long o = 0;
  double4 N{};
  double yu_d = 0., yv_d = 0., yp_d = 0.;
  int iref = 1;
  double2 cc{};
  if (live) {
    strip_point(e, -h, k, n, di, dj);
    o = mb + p * g.plane + (long long)(dj + H) * g.P + (di + H);
    N = a.Ntab[((p * 4 + e) * (H + 1) + h) * n + k];
    if constexpr (MIXED) {
      yu_d = a.u[o];
      yv_d = a.v[o];
      yp_d = a.phi[o];
    }
    if (h > 0) {
      iref = a.giref[(h - 1) * n + k];
      cc = a.gcoef[(h - 1) * n + k];
    }
  }
  // Launched with programmatic dependent launch, the blocks may be resident
  // before the stage kernel that writes the increments, boundary copies and
  // (FP64 form) the state has completed: everything above reads only what it
  // leaves alone (the strip tables, the active list and, split precision, Y).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // the next stage kernel may launch now (the stage kernel before this one
  // has completed): its items clear of the panel edges read nothing this
  // kernel writes, the others wait for its completion
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  // the boundary line (h = 0) needs no staged values
  bool store = live;
  double zw = 0., mw = 0., ph = 0.;
  if (live && h == 0) {
    if (k > 0 && k < n - 1) {
      // edge average (spatial_operators_mod.F90:298-345)
      const int ks = L.rev ? n - 1 - k : k;
      int oi, oj, ni, nj;
      strip_point(e, 0, k, n, oi, oj);
      strip_point(e2, 0, ks, n, ni, nj);
      double ou, ov, op, nu, nv, np_;
      raw_boundary(p, oi, oj, ou, ov, op);
      raw_boundary(q, ni, nj, nu, nv, np_);
      const double4 Mo = a.Mtab[((p * 4 + e) * (H + 1) + 0) * n + k];
      const double4 Mn = a.Mtab[((q * 4 + e2) * (H + 1) + 0) * n + ks];
      zw = 0.5 * ((Mo.x * ou + Mo.z * ov) + (Mn.x * nu + Mn.z * nv));
      mw = 0.5 * ((Mo.y * ou + Mo.w * ov) + (Mn.y * nu + Mn.w * nv));
      ph = 0.5 * (op + np_);
    } else if (e <= 1) {
      // cube vertex (:347-386), owned by the W/E edge threads
      const int corner = (e == 0) ? (k == 0 ? 0 : 2) : (k == 0 ? 1 : 3);
      const VertexRef V = c_vertex[p][corner];
      double zz[3], mm[3], pp[3];
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const int pt = V.panel[t], ct = V.corner[t];
        const int et = (ct == 0 || ct == 2) ? 0 : 1;  // W or E column holds the corner
        const int kt = (ct <= 1) ? 0 : n - 1;
        double bu, bv, bp;
        raw_boundary(pt, et == 0 ? 0 : n - 1, kt, bu, bv, bp);
        const double4 M = a.Mtab[((pt * 4 + et) * (H + 1) + 0) * n + kt];
        zz[t] = M.x * bu + M.z * bv;
        mm[t] = M.y * bu + M.w * bv;
        pp[t] = bp;
      }
      zw = (zz[0] + zz[1] + zz[2]) / 3.;
      mw = (mm[0] + mm[1] + mm[2]) / 3.;
      ph = (pp[0] + pp[1] + pp[2]) / 3.;
    } else {
      store = false;  // an S/N edge's end: the vertex, written by the W/E threads
    }
  }

  // stage the neighbour's lines 1..H over the window [lo, lo + kHaloWin)
  const int lo = max(k0 - kHaloLead, 0);
  for (int s = threadIdx.x; s < H * kHaloWin; s += NT) {
    const int hh = (e2 <= 1) ? 1 + s % H : 1 + s / kHaloWin;
    const int t = (e2 <= 1) ? s / H : s % kHaloWin;
    const int kk = lo + t;
    if (kk <= n - 1) neighbour(hh, kk, wz[hh - 1][t], wm[hh - 1][t], wp[hh - 1][t]);
  }
  __syncthreads();

  if (live && h > 0) {
    // halo line h: the neighbour's line h on the sphere, interpolated along
    // the edge (ghost_mod.f90:154-181)
    double qz[D], qm[D], qp[D];
#pragma unroll
    for (int m = 0; m < D; ++m) {
      const int kk = (iref - 1) * (D - 1) + m;
      const int t = kk - lo;
      if (t >= 0 && t < kHaloWin) {
        qz[m] = wz[h - 1][t];
        qm[m] = wm[h - 1][t];
        qp[m] = wp[h - 1][t];
      } else {
        neighbour(h, kk, qz[m], qm[m], qp[m]);
      }
    }
    zw = ghost_interp<D>(qz, cc.x, cc.y, a);
    mw = ghost_interp<D>(qm, cc.x, cc.y, a);
    ph = ghost_interp<D>(qp, cc.x, cc.y, a);
  }
  if (!store) return;
  // back to this panel's covariant winds (covProjSphere2Plane, :459-492)
  const double uo = N.x * zw + N.z * mw, vo = N.y * zw + N.w * mw;
  if constexpr (!MIXED) {
    a.u[o] = uo;
    a.v[o] = vo;
    a.phi[o] = ph;
  } else {
    a.du[o] = (float)(uo - yu_d);
    a.dv[o] = (float)(vo - yv_d);
    a.dp[o] = (float)(ph - yp_d);
  }
}

// ---------------------------------------------------------------------------
// Mass / energy (src/diag_mod.F90:10-67): per-cell sums in the reference's
// order, then a compensated (Neumaier) sum over cells.
// ---------------------------------------------------------------------------

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
        const double wgt = wi * wj / wden;
        const long long o = (long long)p * g.plane + (long long)(jc * (D - 1) + jd + H) * g.P + (ic * (D - 1) + id + H);
        const double sg = sqrtG[o], ph = phi[o], uu = u[o], vv = v[o];
        const double cu = ig11[o] * uu + ig12[o] * vv, cv = ig12[o] * uu + ig22[o] * vv;
        mc = mc + wgt * (ph * sg);
        const double KE = 0.5 * ph * (uu * cu + vv * cv);
        const double PE = 0.5 * ((ph + phis[o]) * (ph + phis[o]));
        ec = ec + wgt * sg * (KE + PE);
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

// Failure detection: flags[m] = 1 if an interior u, v or phi of member m is
// NaN or Inf (flags cleared by the caller; racing stores write the same value).
__global__ void __launch_bounds__(256) finite_check_kernel(const GridDesc g, int H, const double *u, const double *v,
                                                           const double *phi, int *flags) {
  const int m = blockIdx.y;
  const int n = g.n;
  const long long per = 6LL * n * n;
  bool bad = false;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < per;
       k += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(k / ((long long)n * n));
    const int rem = (int)(k - (long long)p * n * n);
    const int j = rem / n, i = rem - j * n;
    const long long o = (long long)m * g.mstride + p * g.plane + (long long)(j + H) * g.P + (i + H);
    bad |= !isfinite(u[o]) || !isfinite(v[o]) || !isfinite(phi[o]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) flags[m] = 1;
}

}  // namespace mcv
