// mcv_geometry.cu -- a handle's grid geometry and a member's initial state
// computed on the device.
//
// Geometry: the equiangular metric planes, the sphere<->panel matrices on the
// edge strips, the 1-D metric table of split precision and the ghost
// interpolation weights, with the formulas and evaluation order of the host
// builder (mcv_build_geometry: src/projection_mod.F90:8-322,
// src/mesh_mod.F90:132-163, src/ghost_mod.f90:21-79).
// Initial state: the seeded balanced flow of the host init chain (tilted
// solid-body flow, src/test_case_mod.F90:118-120; real spherical harmonics;
// Gaussian mountain; sphere -> covariant winds), as mcv_ic_tilted_zonal,
// mcv_ic_add_harmonics, mcv_ic_add_mountain and mcv_sphere_to_cov compute it.
// This file is compiled without FMA contraction, like the host code; what
// differs from the host's numbers is the device math library (tan, cos, sin,
// atan2, acos, exp, sqrt, pow, within a few ulp) and the order of the sums.
#include <cuda_runtime.h>

#include "mcv_ksum.cuh"
#include "mcv_internal.h"

namespace mcv {
namespace {

constexpr double kOmegaDev = 7.292E-5;  // src/constants_mod.F90

__device__ void plane_to_sphere_dev(int panel, double x, double y, double pi, double &lambda, double &theta) {
  // src/projection_mod.F90:8-38
  if (panel <= 4) {
    lambda = x + (double)(panel - 1) * pi / 2.;
    theta = atan2(tan(y) * cos(x), 1.);
  } else {
    const double a = tan(x), b = tan(y);
    if (panel == 5) {
      lambda = atan2(a, -b);
      theta = atan2(1., sqrt(a * a + b * b));
    } else {
      lambda = atan2(a, b);
      theta = -atan2(1., sqrt(a * a + b * b));
    }
  }
}

__device__ void sphere_to_plane_dev(int panel, double lambda, double theta, double pi, double &x, double &y) {
  // src/projection_mod.F90:40-58
  if (panel <= 4) {
    const double l = lambda - (double)(panel - 1) * pi / 2.;
    x = atan(tan(l));
    y = atan(tan(theta) / cos(l));
  } else {
    const double s = (panel == 5) ? 1. : -1.;
    x = atan(s * sin(lambda) / tan(theta));
    y = atan(-cos(lambda) / tan(theta));
  }
}

struct PointGeo {
  double lon, lat, sqrtG, f;
  double G[4], IG[4], A[4], IA[4];  // 2x2, column-major
};

// The metric and the vector bases at panel coordinates (x, y)
// (src/projection_mod.F90:150-322), as point_geometry in host_setup.cpp.
template <typename A>
__device__ void point_geo(int panel, double x, double y, const A &a, PointGeo &g) {
  plane_to_sphere_dev(panel, x, y, a.pi, g.lon, g.lat);
  const double lon = g.lon;
  const double tx = tan(x), ty = tan(y), cx = cos(x), cy = cos(y);
  const double R2 = a.radius * a.radius;
  const double rho = sqrt(1. + tx * tx + ty * ty);
  const double fG = R2 / (pow(rho, 4.) * (cx * cx) * (cy * cy));
  const double gxx = 1. + tx * tx, gyy = 1. + ty * ty, gxy = -(tx * ty);
  g.G[0] = fG * gxx;
  g.G[1] = fG * gxy;
  g.G[2] = fG * gxy;
  g.G[3] = fG * gyy;
  const double fIG = (rho * rho * (cx * cx) * (cy * cy)) / R2;
  g.IG[0] = fIG * gyy;
  g.IG[1] = fIG * (tx * ty);
  g.IG[2] = fIG * (tx * ty);
  g.IG[3] = fIG * gxx;
  g.sqrtG = 1. / ((cx * cx) * (cy * cy) * (rho * rho * rho)) * R2;
  const double al = (panel <= 4) ? lon - (double)(panel - 1) * a.pi / 2. : lon;
  const double sa = sin(al), ca = cos(al), c = sin(g.lat), d = cos(g.lat);
  if (panel <= 4) {
    const double t = d * d * ca * ca + c * c;
    g.IA[0] = 1. / d;
    g.IA[2] = 0.;
    g.IA[1] = sa * c / t;
    g.IA[3] = ca / t;
    g.A[0] = d;
    g.A[2] = 0.;
    g.A[1] = -(c * d * sa / ca);
    g.A[3] = ca * d * d + c * c / ca;
  } else {
    const double sgn = (panel == 5) ? 1. : -1.;
    const double t1 = c + sa * sa * d * d / c, t2 = c + ca * ca * d * d / c;
    g.IA[0] = sgn * (ca / t1);
    g.IA[2] = -sgn * (sa / c / t1);
    g.IA[1] = sa / t2;
    g.IA[3] = ca / c / t2;
    const double u1 = 1. + sa * sa * d * d / c / c, u2 = 1. + ca * ca * d * d / c / c;
    g.A[0] = sgn * (ca * c * u1);
    g.A[1] = -sgn * (c * c * sa * u1);
    g.A[2] = sa * c * u2;
    g.A[3] = ca * c * c * u2;
  }
  for (int k = 0; k < 4; ++k) {
    g.IA[k] = g.IA[k] / a.radius;
    g.A[k] = g.A[k] * a.radius;
  }
  g.f = 2. * kOmegaDev * sin(g.lat);
}

// panel coordinate of padded index i (0-based): x_i = (i + ips - 1) dx/(D-1) + x_min
template <typename A>
__device__ __forceinline__ double coord(const A &a, int i) {
  return (double)(i + (1 - a.H) - 1) * a.dx / (double)(a.order - 1) + a.x_min;
}

// metric planes of the FP64 policy over the padded points, [6][npx][P]
__global__ void planes_kernel(const GeomArgs a) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y, p = blockIdx.z;
  if (ii >= a.npx) return;
  PointGeo g;
  point_geo(p + 1, coord(a, ii), coord(a, jj), a, g);
  const long long o = ((long long)p * a.npx + jj) * a.P + ii;
  a.sqrtG[o] = g.sqrtG;
  a.ig11[o] = g.IG[0];
  a.ig12[o] = g.IG[2];  // IG(1,2) == IG(2,1)
  a.ig22[o] = g.IG[3];
  a.fcor[o] = g.f;
}

// convert_ghost_wind_P2SP / SP2P matrices on the H+1 lines along each panel
// edge: Mt = A IG at the strip point, Nt = G IA at its mirror outside the edge
__global__ void strips_kernel(const GeomArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = blockIdx.y, pe = blockIdx.z, p = pe / 4, e = pe % 4;
  if (k >= a.n) return;
  auto pidx = [&](int dd, int &i, int &j) {
    switch (e) {
      case 0: i = dd; j = k; break;
      case 1: i = a.n - 1 - dd; j = k; break;
      case 2: i = k; j = dd; break;
      default: i = k; j = a.n - 1 - dd; break;
    }
  };
  int i, j;
  PointGeo g;
  double m[4];
  pidx(d, i, j);
  point_geo(p + 1, coord(a, i + a.H), coord(a, j + a.H), a, g);
  matmul22(m, g.A, g.IG);
  const long long o = ((long long)pe * (a.H + 1) + d) * a.n + k;
  a.Mtab[o] = make_double4(m[0], m[1], m[2], m[3]);
  pidx(-d, i, j);
  point_geo(p + 1, coord(a, i + a.H), coord(a, j + a.H), a, g);
  matmul22(m, g.G, g.IA);
  a.Ntab[o] = make_double4(m[0], m[1], m[2], m[3]);
}

// split precision's 1-D table {tan, cos^2/R^2, sin cos/R, R/cos^2} per padded index
__global__ void met1d_kernel(const GeomArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.npx) return;
  const double x = coord(a, i), t = tan(x), c = cos(x), s = sin(x), R = a.radius;
  a.met1d[i] = make_double4(t, c * c / (R * R), s * c / R, R / (c * c));
}

// ghost weights (src/ghost_mod.f90:21-79): halo line hh of panel 1's top edge
// located on panel 5's x axis; iref = the cell whose x range holds the point
__global__ void ghost_kernel(const GeomArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, hh = blockIdx.y + 1;
  if (i > a.n) return;
  const int D = a.order;
  auto xraw = [&](int c) { return (double)((c - 1) * (D - 1) + 1 - 1) * a.dx / (double)(D - 1) + a.x_min; };
  const double y = (double)(a.n + hh - 1) * a.dx / (double)(D - 1) + a.x_min;
  const double x = (double)(i - 1) * a.dx / (double)(D - 1) + a.x_min;
  double lam, th, X, Y;
  plane_to_sphere_dev(1, x, y, a.pi, lam, th);
  sphere_to_plane_dev(5, lam, th, a.pi, X, Y);
  // smallest iref in 1..nc+1 with X <= xraw(iref), as the host's forward scan.
  // A ghost point on a cell boundary (the panel corners map onto one) takes
  // the lower cell as the host does; kTieEps absorbs the few-ulp difference
  // between the device's and the host's tan/atan there (either cell's
  // polynomial gives the shared point's value).
  constexpr double kTieEps = 4e-15;
  int lo = 1, hi = a.nc + 1;
  if (X > xraw(hi) + kTieEps) {
    atomicExch(a.err, 1);
    return;
  }
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (X > xraw(mid) + kTieEps) lo = mid + 1;
    else hi = mid;
  }
  const int iref = lo;
  if (iref < 2 || !(X >= xraw(iref - 1) - kTieEps && X <= xraw(iref) + kTieEps)) {
    atomicExch(a.err, 1);
    return;
  }
  const long long k = (i - 1) + (long long)a.n * (hh - 1);
  const double c = X - xraw(iref - 1);
  a.giref[k] = iref - 1;
  a.gcoef[k] = make_double2(c, pow(c, 3.));
}

// ---------------------------------------------------------------------------
// Initial state of one member
// ---------------------------------------------------------------------------
constexpr double kGravityDev = 9.80616;  // src/constants_mod.F90

// weightsOnPV summed over the cells sharing padded index i (mesh_mod.F90:183-203),
// zero in the halo: (1,4,1)/6 or (1,3,3,1)/8 per cell
__device__ double pv_weight(const IcArgs &a, int i) {
  const int D = a.order, l = i - a.H;
  if (l < 0 || l >= a.n) return 0.;
  const double e = (D == 3) ? 1. / 6. : 1. / 8., mid = (D == 3) ? 4. / 6. : 3. / 8.;
  const int r = l % (D - 1);
  if (r != 0) return mid;
  return (l == 0 || l == a.n - 1) ? e : e + e;
}

// unit-scale harmonic height at (lon, lat): sum over l = 1..L, m = 0..l of
// coef[l^2 + l +- m] times the orthonormal real spherical harmonics, with the
// normalised associated Legendre functions of mcv_ic_add_harmonics
// (recurrence along the diagonal, then up each column m)
__device__ double harmonic_sum(const IcArgs &a, double lon, double lat) {
  const int L = a.lmax;
  const double x = sin(lat), s = cos(lat);
  const double r2pi = sqrt(2. * a.pi), rpi = sqrt(a.pi);
  double acc = 0., pmm = sqrt(0.5);
  for (int m = 0; m <= L; ++m) {
    if (m > 0) pmm = -sqrt((2. * m + 1.) / (2. * m)) * s * pmm;
    const double cm = cos(m * lon), sm = sin(m * lon);
    double p1 = 0., p2 = 0.;  // P_{l-1}, P_{l-2} of column m
    for (int l = m; l <= L; ++l) {
      double p;
      if (l == m) p = pmm;
      else if (l == m + 1) p = sqrt(2. * m + 3.) * x * pmm;
      else {
        const double aa = sqrt((4. * l * l - 1.) / ((double)l * l - (double)m * m));
        const double bb = sqrt(((l - 1.) * (l - 1.) - (double)m * m) / (4. * (l - 1.) * (l - 1.) - 1.));
        p = aa * (x * p1 - bb * p2);
      }
      if (l >= 1) {
        if (m == 0) acc += a.coef[l * l + l] * p / r2pi;
        else {
          const double pl = p / rpi;
          acc += a.coef[l * l + l + m] * pl * cm + a.coef[l * l + l - m] * pl * sm;
        }
      }
      p2 = p1;
      p1 = p;
    }
  }
  return acc;
}

// pass 1: the unit-scale harmonic height into the member's phi_s slot
__global__ void ic_harmonics_kernel(const IcArgs a) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y, p = blockIdx.z;
  if (ii >= a.npx) return;
  double lon, lat;
  plane_to_sphere_dev(p + 1, coord(a, ii), coord(a, jj), a.pi, lon, lat);
  a.phis[((long long)p * a.npx + jj) * a.P + ii] = harmonic_sum(a, lon, lat);
}

// Neumaier-compensated per-block sums over the interior points: mode 0
// (w x^2, w) with w = weightsOnPV sqrtG (the area-weighted RMS), mode 1
// (sqrtG x, sqrtG) (the mean depth); partial[block] = {s1, c1, s2, c2}
__global__ void __launch_bounds__(256) ic_sums_kernel(const IcArgs a, int mode, const double *x, double4 *partial) {
  const long long per = 6LL * a.n * a.n;
  KSum s1{0., 0.}, s2{0., 0.};
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < per; k += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(k / ((long long)a.n * a.n));
    const int rem = (int)(k - (long long)p * a.n * a.n);
    const int j = rem / a.n + a.H, i = rem % a.n + a.H;
    const long long o = ((long long)p * a.npx + j) * a.P + i;
    const double sg = a.sqrtG[o], v = x[o];
    if (mode == 0) {
      const double w = pv_weight(a, i) * pv_weight(a, j) * sg;
      neumaier_add(s1, w * v * v);
      neumaier_add(s2, w);
    } else {
      neumaier_add(s1, sg * v);
      neumaier_add(s2, sg);
    }
  }
  __shared__ KSum r1[256], r2[256];
  r1[threadIdx.x] = s1;
  r2[threadIdx.x] = s2;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      ksum_merge(r1[threadIdx.x], r1[threadIdx.x + st]);
      ksum_merge(r2[threadIdx.x], r2[threadIdx.x + st]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = make_double4(r1[0].s, r1[0].c, r2[0].s, r2[0].c);
}

// pass 2: u, v, phi, phi_s of the member
__global__ void ic_fields_kernel(const IcArgs a) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y, p = blockIdx.z;
  if (ii >= a.npx) return;
  PointGeo g;
  point_geo(p + 1, coord(a, ii), coord(a, jj), a, g);
  const double lon = g.lon, lat = g.lat;
  const long long o = ((long long)p * a.npx + jj) * a.P + ii;
  // tilted solid-body flow (mcv_ic_tilted_zonal)
  const double zw = a.u0 * (cos(lat) * cos(a.alpha) + cos(lon) * sin(lat) * sin(a.alpha));
  const double mw = -a.u0 * sin(lon) * sin(a.alpha);
  const double t = -cos(lon) * cos(lat) * sin(a.alpha) + sin(lat) * cos(a.alpha);
  double phi = a.gh0 - (a.radius * kOmegaDev * a.u0 + (a.u0 * a.u0) / 2.) * (t * t);
  // + g times the rescaled harmonic height (cases.harmonic_height)
  if (a.lmax > 0) phi = phi + kGravityDev * (a.phis[o] * a.ratio);
  // Gaussian mountain (mcv_ic_add_mountain): phi_s = hs, phi -= hs
  double phs = 0.;
  if (a.mountain) {
    const double cang = sin(a.lat_c) * sin(lat) + cos(a.lat_c) * cos(lat) * cos(lon - a.lon_c);
    const double d = a.radius * acos(fmax(-1., fmin(1., cang)));
    const double q = d / a.efold;
    const double hs = kGravityDev * a.h0 * exp(-(q * q));
    phs = phs + hs;
    phi = phi - hs;
  }
  // covariant winds (mcv_sphere_to_cov): (G IA) (zonal, meridional)
  double m[4];
  matmul22(m, g.G, g.IA);
  a.u[o] = m[0] * zw + m[2] * mw;
  a.v[o] = m[1] * zw + m[3] * mw;
  a.phi[o] = phi;
  a.phis[o] = phs;
  if (a.phis32) a.phis32[o] = (float)phs;
}

// convert_wind_P2SP (src/spatial_operators_mod.F90:391-405) over the padded
// points after addFillValue (src/output_mod.F90:230-248): the halo corner
// squares of u and v hold FillValue, and every point gets
// (zonal, meridional) = (A IG)(u, v) with matmul's k = 1, 2 order
// (covProjPlane2Sphere, src/projection_mod.F90:79-96).
__global__ void history_p2sp_kernel(const GeomArgs a, const double *u, const double *v, int which, double *out) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y, p = blockIdx.z;
  if (ii >= a.npx) return;
  PointGeo g;
  point_geo(p + 1, coord(a, ii), coord(a, jj), a, g);
  const bool corner = (ii < a.H || ii >= a.npx - a.H) && (jj < a.H || jj >= a.npx - a.H);
  const long long o = ((long long)p * a.npx + jj) * a.P + ii;
  const double fill = -9999999999999999.;  // FillValue, src/constants_mod.F90:20
  const double cu = corner ? fill : u[o], cv = corner ? fill : v[o];
  double m[4];
  matmul22(m, g.A, g.IG);
  out[((long long)p * a.npx + jj) * a.npx + ii] = which == 0 ? m[0] * cu + m[2] * cv : m[1] * cu + m[3] * cv;
}

}  // namespace

int history_p2sp_device(const GeomArgs &a, const double *u, const double *v, int which, double *out,
                        cudaStream_t s) {
  history_p2sp_kernel<<<dim3((a.npx + 127) / 128, a.npx, 6), 128, 0, s>>>(a, u, v, which, out);
  return (int)cudaGetLastError();
}

int ic_harmonics_device(const IcArgs &a, cudaStream_t s) {
  const int T = 128;
  ic_harmonics_kernel<<<dim3((a.npx + T - 1) / T, a.npx, 6), T, 0, s>>>(a);
  return (int)cudaGetLastError();
}

int ic_sums_device(const IcArgs &a, int mode, const double *x, double4 *partial, int blocks, cudaStream_t s) {
  ic_sums_kernel<<<blocks, 256, 0, s>>>(a, mode, x, partial);
  return (int)cudaGetLastError();
}

int ic_fields_device(const IcArgs &a, cudaStream_t s) {
  const int T = 128;
  ic_fields_kernel<<<dim3((a.npx + T - 1) / T, a.npx, 6), T, 0, s>>>(a);
  return (int)cudaGetLastError();
}

int build_geometry_device(const GeomArgs &a, cudaStream_t s) {
  const int T = 128;
  planes_kernel<<<dim3((a.npx + T - 1) / T, a.npx, 6), T, 0, s>>>(a);
  strips_kernel<<<dim3((a.n + T - 1) / T, a.H + 1, 24), T, 0, s>>>(a);
  if (a.met1d) met1d_kernel<<<(a.npx + T - 1) / T, T, 0, s>>>(a);
  ghost_kernel<<<dim3((a.n + T - 1) / T, a.H), T, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

}  // namespace mcv
