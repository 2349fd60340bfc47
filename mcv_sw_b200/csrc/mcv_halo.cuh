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

// MIXED: the field completed is Y + increment.  Raw values combine Y with the
// increment in FP64; the result minus Y at the destination is stored as the
// new FP32 increment, so the next stage's input halo is the FP64 correction
// of its own interior.
template <int D, bool MIXED, int NB>
__global__ void __launch_bounds__(128) halo_kernel(const __grid_constant__ HaloBatch<NB> hb) {
  constexpr int H = D - 1;
  // the next stage kernel may launch now: its items clear of the panel edges
  // read nothing this kernel writes, the others wait for its completion
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // one thread per (position k along the edge: x; panel, edge and halo line
  // h = 0..H: y; grid and active member: z) -- no runtime divisions before
  // the first loads
  const int z = blockIdx.z;
  int kg = 0;
#pragma unroll
  for (int j = 1; j < NB; ++j)
    if (j < hb.ngrids && z >= hb.first[j]) kg = j;
  const GridDesc &g = hb.g[kg];
  const HaloArgs &a = hb.a[kg];
  const int n = g.n;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int slot = z - hb.first[kg];
  const int mem = __ldg(a.active + slot);
  const int h = blockIdx.y % (H + 1);
  const int pe = blockIdx.y / (H + 1);
  const int p = pe >> 2, e = pe & 3;
  const EdgeLink L = c_links[p][e];
  const int q = L.q, e2 = L.e2;
  const long long mb = (long long)mem * g.mstride;
  const long long bb = (long long)mem * 24 * n;

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

  // destination point and its rotation, loaded ahead of the dependent loads
  int di, dj;
  strip_point(e, -h, k, n, di, dj);
  const long long o = mb + p * g.plane + (long long)(dj + H) * g.P + (di + H);
  const double4 N = a.Ntab[((p * 4 + e) * (H + 1) + h) * n + k];
  double yu_d = 0., yv_d = 0., yp_d = 0.;
  if constexpr (MIXED) {
    yu_d = a.u[o];
    yv_d = a.v[o];
    yp_d = a.phi[o];
  }

  double zw, mw, ph;
  if (h > 0) {
    // halo line h: neighbour line h rotated to the sphere, interpolated along
    // the edge, rotated back to this panel (ghost_mod.f90:154-181).  The D
    // neighbour points' loads are all issued before any is used: a point at an
    // end of the line is a boundary point and takes its raw copy; the state
    // load of such a point goes to its inner neighbour instead (FP64 form: the
    // boundary itself is rewritten by this kernel) and is not used.
    const int iref = a.giref[(h - 1) * n + k];
    const double2 cc = a.gcoef[(h - 1) * n + k];
    double yu[D], yv[D], yp[D];
    double4 M[D], bv[D];
    float4 b32[D];
    float du[D], dv[D], dp[D];
    bool isb[D];
#pragma unroll
    for (int m = 0; m < D; ++m) {
      const int kk = (iref - 1) * (D - 1) + m;
      const int ks = L.rev ? n - 1 - kk : kk;
      isb[m] = (ks == 0 || ks == n - 1);
      int si, sj;
      strip_point(e2, h, ks, n, si, sj);
      const int bslot = boundary_slot(si, sj, n);
      const int kc = MIXED ? ks : min(max(ks, 1), n - 2);
      strip_point(e2, h, kc, n, si, sj);
      const long long os = mb + q * g.plane + (long long)(sj + H) * g.P + (si + H);
      yu[m] = a.u[os];
      yv[m] = a.v[os];
      yp[m] = a.phi[os];
      if constexpr (MIXED) {
        b32[m] = a.bnd32[bb + q * 4 * n + bslot];
        du[m] = a.du[os];
        dv[m] = a.dv[os];
        dp[m] = a.dp[os];
      } else {
        bv[m] = a.bnd[bb + q * 4 * n + bslot];
      }
      M[m] = a.Mtab[((q * 4 + e2) * (H + 1) + h) * n + ks];
    }
    double qz[D], qm[D], qp[D];
#pragma unroll
    for (int m = 0; m < D; ++m) {
      double su, sv, sp;
      if constexpr (MIXED) {
        su = yu[m] + (double)(isb[m] ? b32[m].x : du[m]);
        sv = yv[m] + (double)(isb[m] ? b32[m].y : dv[m]);
        sp = yp[m] + (double)(isb[m] ? b32[m].z : dp[m]);
      } else {
        su = isb[m] ? bv[m].x : yu[m];
        sv = isb[m] ? bv[m].y : yv[m];
        sp = isb[m] ? bv[m].z : yp[m];
      }
      qz[m] = M[m].x * su + M[m].z * sv;  // covProjPlane2Sphere, projection_mod.F90:79-96
      qm[m] = M[m].y * su + M[m].w * sv;
      qp[m] = sp;
    }
    zw = ghost_interp<D>(qz, cc.x, cc.y, a);
    mw = ghost_interp<D>(qm, cc.x, cc.y, a);
    ph = ghost_interp<D>(qp, cc.x, cc.y, a);
  } else if (k > 0 && k < n - 1) {
    // boundary line: edge average (spatial_operators_mod.F90:298-345)
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
    double z[3], mm[3], pp[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      const int pt = V.panel[t], ct = V.corner[t];
      const int et = (ct == 0 || ct == 2) ? 0 : 1;  // W or E column holds the corner
      const int kt = (ct <= 1) ? 0 : n - 1;
      double bu, bv, bp;
      raw_boundary(pt, et == 0 ? 0 : n - 1, kt, bu, bv, bp);
      const double4 M = a.Mtab[((pt * 4 + et) * (H + 1) + 0) * n + kt];
      z[t] = M.x * bu + M.z * bv;
      mm[t] = M.y * bu + M.w * bv;
      pp[t] = bp;
    }
    zw = (z[0] + z[1] + z[2]) / 3.;
    mw = (mm[0] + mm[1] + mm[2]) / 3.;
    ph = (pp[0] + pp[1] + pp[2]) / 3.;
  } else {
    return;
  }
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
