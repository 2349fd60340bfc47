// mcv_diag.cu -- device diagnostics of the history output: calc_VIA cell
// averages and the normalized error norms of doc/orderCheck.m, on states that
// stay in HBM (only the results cross PCIe).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mcv_internal.h"

namespace mcv {
namespace {

// weightsOnPV(iDOF, jDOF) (src/mesh_mod.F90:183-203): the outer product of
// {1, 4, 1} (MCV3) or {1, 3, 3, 1} (MCV4) divided by 36 or 80.  The products
// are small integers, so a*b/den is the reference's value bit for bit.
template <int D>
__device__ __forceinline__ double pv_weight(int id, int jd) {
  const double a = (id == 0 || id == D - 1) ? 1. : (D == 3 ? 4. : 3.);
  const double b = (jd == 0 || jd == D - 1) ? 1. : (D == 3 ? 4. : 3.);
  return (a * b) / (D == 3 ? 36. : 80.);
}

// calc_VIA of cell (ic, jc) (0-based) of panel p: the jDOF, iDOF loop of
// src/diag_mod.F90:79-90 with explicit roundings (no FMA contraction)
template <int D>
__device__ __forceinline__ double cell_via(const double *f, int npx, int P, int p, int ic, int jc) {
  constexpr int H = D - 1;
  double s = 0.;
#pragma unroll
  for (int jd = 0; jd < D; ++jd)
#pragma unroll
    for (int id = 0; id < D; ++id) {
      const long long o = ((long long)p * npx + (jc * (D - 1) + jd + H)) * P + (ic * (D - 1) + id + H);
      s = __dadd_rn(s, __dmul_rn(pv_weight<D>(id, jd), f[o]));
    }
  return s;
}

template <int D>
__global__ void via_kernel(int nc, int npx, int P, const double *f, double *out) {
  const int nce = nc + 2;  // ics:ice = 0..nc+1
  const long long total = 6LL * nce * nce;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(k / ((long long)nce * nce));
    const int r = (int)(k - (long long)p * nce * nce);
    const int jc = r / nce - 1, ic = r % nce - 1;  // cell indices 0..nc-1 inside
    out[k] = (ic < 0 || ic >= nc || jc < 0 || jc >= nc) ? 0. : cell_via<D>(f, npx, P, p, ic, jc);
  }
}

template <int D>
__global__ void __launch_bounds__(256) norms_kernel(int nc, int npx, int P, const double *a, const double *b,
                                                    const double *area, double4 *partial) {
  const long long total = 6LL * nc * nc;
  double l1 = 0., r1 = 0., l2 = 0., r2 = 0., md = 0., mb = 0.;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(k / ((long long)nc * nc));
    const int r = (int)(k - (long long)p * nc * nc);
    const int jc = r / nc, ic = r % nc;
    const double va = cell_via<D>(a, npx, P, p, ic, jc), vb = cell_via<D>(b, npx, P, p, ic, jc);
    const double w = area[r], d = va - vb;
    l1 += fabs(d) * w;
    r1 += fabs(vb) * w;
    l2 += d * d * w;
    r2 += vb * vb * w;
    md = fmax(md, fabs(d) * w);
    mb = fmax(mb, fabs(vb) * w);
  }
  __shared__ double sh[6][256];
  sh[0][threadIdx.x] = l1;
  sh[1][threadIdx.x] = r1;
  sh[2][threadIdx.x] = l2;
  sh[3][threadIdx.x] = r2;
  sh[4][threadIdx.x] = md;
  sh[5][threadIdx.x] = mb;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      for (int q = 0; q < 4; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
      for (int q = 4; q < 6; ++q) sh[q][threadIdx.x] = fmax(sh[q][threadIdx.x], sh[q][threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = make_double4(sh[0][0], sh[1][0], sh[2][0], sh[3][0]);
    partial[2 * blockIdx.x + 1] = make_double4(sh[4][0], sh[5][0], 0., 0.);
  }
}

}  // namespace

int via_device(int order, int nc, int npx, int P, const double *f, double *out, cudaStream_t s) {
  const int blocks = 296, threads = 256;
  if (order == 3) via_kernel<3><<<blocks, threads, 0, s>>>(nc, npx, P, f, out);
  else via_kernel<4><<<blocks, threads, 0, s>>>(nc, npx, P, f, out);
  return (int)cudaGetLastError();
}

int norms_device(int order, int nc, int npx, int P, const double *a, const double *b, const double *area,
                 double4 *partial, int blocks, cudaStream_t s) {
  if (order == 3) norms_kernel<3><<<blocks, 256, 0, s>>>(nc, npx, P, a, b, area, partial);
  else norms_kernel<4><<<blocks, 256, 0, s>>>(nc, npx, P, a, b, area, partial);
  return (int)cudaGetLastError();
}

// EquiangularAllAreas (src/mesh_mod.F90:240-276): the spherical excess of
// each cell, from the angles between the grid lines at its four corners,
// times radius^2 (mesh_mod.F90:205-208).
void equiangular_cell_areas(int nc, double radius, double *area) {
  const double pi = 2.0 * std::asin(1.0);
  const int m = nc + 1;
  std::vector<double> gp(m), ang((size_t)m * m);
  for (int k = 0; k < m; ++k) gp[k] = -0.25 * pi + (pi / (double)(2 * nc)) * (double)k;
  for (int k2 = 0; k2 < m; ++k2)
    for (int k1 = 0; k1 < m; ++k1) ang[k1 + (size_t)m * k2] = std::acos(-std::sin(gp[k1]) * std::sin(gp[k2]));
  auto A = [&](int k1, int k2) { return ang[k1 + (size_t)m * k2]; };
  for (int k2 = 0; k2 < nc; ++k2)
    for (int k1 = 0; k1 < nc; ++k1) {
      const double a1 = A(k1, k2), a2 = pi - A(k1 + 1, k2), a3 = pi - A(k1, k2 + 1), a4 = A(k1 + 1, k2 + 1);
      area[k1 + (size_t)nc * k2] = (-2.0 * pi + a1 + a2 + a3 + a4) * (radius * radius);
    }
}

}  // namespace mcv
