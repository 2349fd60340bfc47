// host_setup.cpp -- the caller's side of the C ABI: grid geometry and initial
// conditions on the host, in FP64.
//
// The metric, the sphere<->panel matrices and the ghost weights are inputs of
// the GPU step; they must be the numbers the reference's own setup produces,
// so every formula keeps the reference's evaluation order
// (src/projection_mod.F90:8-322, src/mesh_mod.F90:57-214,
// src/ghost_mod.f90:21-79, src/test_case_mod.F90:13-191).  Fortran's x**2. is
// the product x*x and x**3., x**4. are pow() calls, which is how GCC lowers
// them without -ffast-math.  Build without FMA contraction.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/mcv_gpu.h"
#include "mcv_internal.h"

namespace {

const double kPi = 2.0 * std::asin(1.0);
constexpr double kOmega = 7.292E-5;
constexpr double kGravity = 9.80616;

inline double sq(double x) { return x * x; }

// Cubed-sphere panel coordinates (x, y) of one panel -> (lambda, theta).
// src/projection_mod.F90:8-38
void plane_to_sphere(int panel, double x, double y, double &lambda, double &theta) {
  if (panel <= 4) {
    lambda = x + (double)(panel - 1) * kPi / 2.;
    theta = std::atan2(std::tan(y) * std::cos(x), 1.);
  } else {
    double a = std::tan(x), b = std::tan(y);
    if (panel == 5) {
      lambda = std::atan2(a, -b);
      theta = std::atan2(1., std::sqrt(a * a + b * b));
    } else {
      lambda = std::atan2(a, b);
      theta = -std::atan2(1., std::sqrt(a * a + b * b));
    }
  }
}

// src/projection_mod.F90:40-58
void sphere_to_plane(int panel, double lambda, double theta, double &x, double &y) {
  if (panel <= 4) {
    double l = lambda - (double)(panel - 1) * kPi / 2.;
    x = std::atan(std::tan(l));
    y = std::atan(std::tan(theta) / std::cos(l));
  } else {
    double s = (panel == 5) ? 1. : -1.;  // (-1.)**(panel+1)
    x = std::atan(s * std::sin(lambda) / std::tan(theta));
    y = std::atan(-std::cos(lambda) / std::tan(theta));
  }
}

// Everything the step needs at one point, 2x2 matrices column-major.
struct PointGeometry {
  double lon, lat, sqrtG, f;
  double G[4], IG[4], A[4], IA[4];
};

void point_geometry(int panel, double x, double y, double radius, PointGeometry &g) {
  plane_to_sphere(panel, x, y, g.lon, g.lat);
  const double tx = std::tan(x), ty = std::tan(y), cx = std::cos(x), cy = std::cos(y);
  const double R2 = sq(radius);
  // covariant metric G and its inverse IG (projection_mod.F90:150-192)
  const double rho = std::sqrt(1. + tx * tx + ty * ty);
  const double fG = R2 / (std::pow(rho, 4.) * (cx * cx) * (cy * cy));
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
  // Jacobian (projection_mod.F90:194-211)
  g.sqrtG = 1. / (sq(cx) * sq(cy) * (rho * rho * rho)) * R2;
  // sphere <-> panel vector bases (projection_mod.F90:213-322)
  const double al = (panel <= 4) ? g.lon - (double)(panel - 1) * kPi / 2. : g.lon;
  const double a = std::sin(al), b = std::cos(al), c = std::sin(g.lat), d = std::cos(g.lat);
  if (panel <= 4) {
    const double t = d * d * b * b + c * c;
    g.IA[0] = 1. / d;
    g.IA[2] = 0.;
    g.IA[1] = a * c / t;
    g.IA[3] = b / t;
    g.A[0] = d;
    g.A[2] = 0.;
    g.A[1] = -(c * d * a / b);
    g.A[3] = b * d * d + c * c / b;
  } else {
    const double sgn = (panel == 5) ? 1. : -1.;
    const double t1 = c + a * a * d * d / c, t2 = c + b * b * d * d / c;
    g.IA[0] = sgn * (b / t1);
    g.IA[2] = -sgn * (a / c / t1);
    g.IA[1] = a / t2;
    g.IA[3] = b / c / t2;
    const double u1 = 1. + a * a * d * d / c / c, u2 = 1. + b * b * d * d / c / c;
    g.A[0] = sgn * (b * c * u1);
    g.A[1] = -sgn * (c * c * a * u1);
    g.A[2] = a * c * u2;
    g.A[3] = b * c * c * u2;
  }
  for (int k = 0; k < 4; ++k) {
    g.IA[k] = g.IA[k] / radius;
    g.A[k] = g.A[k] * radius;
  }
  g.f = 2. * kOmega * std::sin(g.lat);
}

}  // namespace

extern "C" int mcv_grid_sizes(int order, int nc, int *npx, int *n, int *halo) {
  if ((order != 3 && order != 4) || nc < 2) return mcv::fail(MCV_ERR_ARG, "order must be 3 or 4 and nc >= 2");
  const int H = order - 1, nn = nc * (order - 1) + 1;
  if (npx) *npx = nn + 2 * H;
  if (n) *n = nn;
  if (halo) *halo = H;
  return MCV_OK;
}

extern "C" int mcv_build_geometry(int order, int nc, double radius, double *lonP, double *latP, double *sqrtG,
                                  double *matrixG, double *matrixIG, double *matrixA, double *matrixIA, double *f,
                                  int *ghost_iref, double *ghost_coef) {
  int npx, n, H;
  if (int rc = mcv_grid_sizes(order, nc, &npx, &n, &H)) return rc;
  const int D = order;
  // parameters_mod.F90:134-239: dx in degrees = 90/nc, then radians
  const double D2R = kPi / 180.;
  const double dx = (90. / nc) * D2R;
  const double x_min = -45. * D2R;
  const int ips = 1 - H;
  const long long plane = (long long)npx * npx;
  // per-point geometry (mesh_mod.F90:132-163); x, y depend on i resp. j only
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 1; p <= 6; ++p)
    for (int jj = 0; jj < npx; ++jj) {
      const double y = (double)(jj + ips - 1) * dx / (double)(D - 1) + x_min;
      for (int ii = 0; ii < npx; ++ii) {
        const double x = (double)(ii + ips - 1) * dx / (double)(D - 1) + x_min;
        PointGeometry g;
        point_geometry(p, x, y, radius, g);
        const long long k = ii + (long long)npx * jj + plane * (p - 1);
        if (lonP) lonP[k] = g.lon;
        if (latP) latP[k] = g.lat;
        if (sqrtG) sqrtG[k] = g.sqrtG;
        if (f) f[k] = g.f;
        for (int e = 0; e < 4; ++e) {
          if (matrixG) matrixG[4 * k + e] = g.G[e];
          if (matrixIG) matrixIG[4 * k + e] = g.IG[e];
          if (matrixA) matrixA[4 * k + e] = g.A[e];
          if (matrixIA) matrixIA[4 * k + e] = g.IA[e];
        }
      }
    }
  if (!ghost_iref && !ghost_coef) return MCV_OK;
  // ghost_mod.f90:21-79: panel-1 top halo points located on panel 5's x axis
  std::vector<double> xraw(nc + 2);
  for (int c = 1; c <= nc + 1; ++c) xraw[c] = (double)((c - 1) * (D - 1) + 1 - 1) * dx / (double)(D - 1) + x_min;
  for (int hh = 1; hh <= H; ++hh) {
    const double y = (double)(n + hh - 1) * dx / (double)(D - 1) + x_min;
    int iref = 1;
    for (int i = 1; i <= n; ++i) {
      const double x = (double)(i - 1) * dx / (double)(D - 1) + x_min;
      double lam, th, X, Y;
      plane_to_sphere(1, x, y, lam, th);
      sphere_to_plane(5, lam, th, X, Y);
      while (X > xraw[iref]) {
        ++iref;
        if (iref > nc + 1) return mcv::fail(MCV_ERR_ARG, "ghost cell location error");
      }
      if (iref < 2 || !(X >= xraw[iref - 1] && X <= xraw[iref])) return mcv::fail(MCV_ERR_ARG, "ghost cell location error");
      const long long k = (i - 1) + (long long)n * (hh - 1);
      if (ghost_coef) ghost_coef[k] = X - xraw[iref - 1];
      if (ghost_iref) ghost_iref[k] = iref - 1;
    }
  }
  return MCV_OK;
}

// ---------------------------------------------------------------------------
// Initial conditions (src/test_case_mod.F90) and seeded synthetic fields.
// ---------------------------------------------------------------------------

extern "C" int mcv_ic_williamson(int case_num, long long npts, const double *lonP, const double *latP, double radius,
                                 double *zonal, double *merid, double *phi, double *phi_s) {
  if (!lonP || !latP || !zonal || !merid || !phi || !phi_s || npts <= 0) return mcv::fail(MCV_ERR_ARG, "null array");
  if (case_num == 2) {  // test_case_mod.F90:52-81
    const double u0 = 2. * kPi * radius / (12. * 86400.), gh0 = 29400.;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < npts; ++k) {
      phi[k] = gh0 - (radius * kOmega * u0 + sq(u0) / 2.) * sq(std::sin(latP[k]));
      zonal[k] = u0 * std::cos(latP[k]);
      merid[k] = 0.;
      phi_s[k] = 0.;
    }
    return MCV_OK;
  }
  if (case_num == 5) {  // test_case_mod.F90:84-130
    const double hs0 = 2000., u0 = 20., alpha = 0., gh0 = 5960. * kGravity;
    const double rr = kPi / 9., lc = 1.5 * kPi, tc = kPi / 6.;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < npts; ++k) {
      double lon = lonP[k];
      const double lat = latP[k];
      if (lon < 0) lon = 2. * kPi + lon;
      const double r = std::sqrt(std::fmin(sq(rr), sq(lon - lc) + sq(lat - tc)));
      const double hs = kGravity * hs0 * (1. - r / rr);
      zonal[k] = u0 * (std::cos(lat) * std::cos(alpha) + std::cos(lon) * std::sin(lat) * std::sin(alpha));
      merid[k] = -u0 * std::sin(lon) * std::sin(alpha);
      phi[k] = gh0 -
               (radius * kOmega * u0 + sq(u0) / 2.) *
                   sq(-std::cos(lon) * std::cos(lat) * std::sin(alpha) + std::sin(lat) * std::cos(alpha)) -
               hs;
      phi_s[k] = hs;
    }
    return MCV_OK;
  }
  if (case_num == 6) {  // test_case_mod.F90:133-191 (R = 4)
    for (long long k = 0; k < npts; ++k) zonal[k] = merid[k] = phi[k] = phi_s[k] = 0.;
    int rc = mcv_ic_add_rossby_haurwitz(npts, lonP, latP, radius, 4, 7.848e-6, zonal, merid, phi);
    if (rc) return rc;
    // phi = gravity*h0 + radius**2*(...) with h0 = 8000 m
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < npts; ++k) phi[k] = kGravity * 8000. + phi[k];
    return MCV_OK;
  }
  return mcv::fail(MCV_ERR_ARG, "case_num must be 2, 5 or 6");
}

extern "C" int mcv_ic_tilted_zonal(long long npts, const double *lonP, const double *latP, double radius, double gh0,
                                   double u0, double alpha, double *zonal, double *merid, double *phi) {
  if (!lonP || !latP || !zonal || !merid || !phi || npts <= 0) return mcv::fail(MCV_ERR_ARG, "null array");
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npts; ++k) {
    const double lon = lonP[k], lat = latP[k];
    zonal[k] = u0 * (std::cos(lat) * std::cos(alpha) + std::cos(lon) * std::sin(lat) * std::sin(alpha));
    merid[k] = -u0 * std::sin(lon) * std::sin(alpha);
    phi[k] = gh0 - (radius * kOmega * u0 + sq(u0) / 2.) *
                       sq(-std::cos(lon) * std::cos(lat) * std::sin(alpha) + std::sin(lat) * std::cos(alpha));
  }
  return MCV_OK;
}

extern "C" int mcv_ic_add_harmonics(long long npts, const double *lonP, const double *latP, int lmax,
                                    const double *coef, double scale, double *phi) {
  if (!lonP || !latP || !coef || !phi || lmax < 1 || lmax > 200) return mcv::fail(MCV_ERR_ARG, "bad harmonic arguments");
  const int L = lmax;
#pragma omp parallel
  {
    // normalized associated Legendre functions by the standard stable
    // recurrences in m (diagonal) and l (column)
    std::vector<double> P((L + 1) * (L + 1));
    std::vector<double> cm(L + 1), sm(L + 1);
#pragma omp for schedule(static)
    for (long long k = 0; k < npts; ++k) {
      const double x = std::sin(latP[k]), s = std::cos(latP[k]);
      // \bar P_l^m with \int_{-1}^{1} \bar P^2 dx = 1 over m-normalisation below
      P[0] = std::sqrt(0.5);
      for (int m = 1; m <= L; ++m) P[m * (L + 1) + m] = -std::sqrt((2. * m + 1.) / (2. * m)) * s * P[(m - 1) * (L + 1) + m - 1];
      for (int m = 0; m < L; ++m) P[m * (L + 1) + m + 1] = std::sqrt(2. * m + 3.) * x * P[m * (L + 1) + m];
      for (int m = 0; m <= L; ++m)
        for (int l = m + 2; l <= L; ++l) {
          const double a = std::sqrt((4. * l * l - 1.) / ((double)l * l - (double)m * m));
          const double b = std::sqrt(((l - 1.) * (l - 1.) - (double)m * m) / (4. * (l - 1.) * (l - 1.) - 1.));
          P[m * (L + 1) + l] = a * (x * P[m * (L + 1) + l - 1] - b * P[m * (L + 1) + l - 2]);
        }
      for (int m = 0; m <= L; ++m) {
        cm[m] = std::cos(m * lonP[k]);
        sm[m] = std::sin(m * lonP[k]);
      }
      double acc = 0.;
      for (int l = 1; l <= L; ++l) {
        // orthonormal on the unit sphere: Y_l0 = Pbar/sqrt(2 pi), Y_lm = Pbar cos|sin / sqrt(pi)
        acc += coef[l * l + l] * P[l] / std::sqrt(2. * kPi);
        for (int m = 1; m <= l; ++m) {
          const double pl = P[m * (L + 1) + l] / std::sqrt(kPi);
          acc += coef[l * l + l + m] * pl * cm[m] + coef[l * l + l - m] * pl * sm[m];
        }
      }
      phi[k] += scale * acc;
    }
  }
  return MCV_OK;
}

extern "C" int mcv_ic_add_mountain(long long npts, const double *lonP, const double *latP, double radius,
                                   double lon_c, double lat_c, double h0, double efold, double *phi, double *phi_s) {
  if (!lonP || !latP || !phi || !phi_s || efold <= 0) return mcv::fail(MCV_ERR_ARG, "bad mountain arguments");
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npts; ++k) {
    const double cang = std::sin(lat_c) * std::sin(latP[k]) + std::cos(lat_c) * std::cos(latP[k]) * std::cos(lonP[k] - lon_c);
    const double d = radius * std::acos(std::fmax(-1., std::fmin(1., cang)));
    const double hs = kGravity * h0 * std::exp(-sq(d / efold));
    phi_s[k] += hs;
    phi[k] -= hs;
  }
  return MCV_OK;
}

extern "C" int mcv_ic_add_rossby_haurwitz(long long npts, const double *lonP, const double *latP, double radius,
                                          int Ri, double omg, double *zonal, double *merid, double *phi) {
  if (!lonP || !latP || !zonal || !merid || !phi || Ri < 1) return mcv::fail(MCV_ERR_ARG, "bad Rossby-Haurwitz arguments");
  const double R = Ri;
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npts; ++k) {
    const double sl = std::sin(latP[k]), cl = std::cos(latP[k]), lon = lonP[k];
    const double u1 = cl, u2 = R * std::pow(cl, R - 1) * sq(sl) * std::cos(R * lon),
                 u3 = std::pow(cl, R + 1) * std::cos(R * lon);
    zonal[k] += radius * omg * (u1 + u2 - u3);
    merid[k] += -radius * omg * R * std::pow(cl, R - 1) * sl * std::sin(R * lon);
    const double AA1 = omg * 0.5 * (2. * kOmega + omg) * sq(cl), Ac = 0.25 * sq(omg);
    const double A21 = (R + 1.) * std::pow(cl, 2. * R + 2.), A22 = (2. * sq(R) - R - 2.) * std::pow(cl, 2. * R),
                 A23 = 2. * sq(R) * std::pow(cl, 2. * R - 2);
    const double Ah = AA1 + Ac * (A21 + A22 - A23);
    const double Bc = 2. * (kOmega + omg) * omg / ((R + 1) * (R + 2)) * std::pow(cl, R);
    const double Bh = Bc * ((sq(R) + 2. * R + 2.) - std::pow(R + 1., 2.) * std::pow(cl, 2.));
    const double Ch = 0.25 * sq(omg) * std::pow(cl, 2. * R) * ((R + 1.) * sq(cl) - (R + 2.));
    phi[k] += sq(radius) * (Ah + Bh * std::cos(R * lon) + Ch * std::cos(2.0 * R * lon));
  }
  return MCV_OK;
}

extern "C" int mcv_ic_add_rossby_wave(long long npts, const double *lonP, const double *latP, double radius,
                                      int Ri, double K, double *zonal, double *merid, double *phi) {
  if (!lonP || !latP || !zonal || !merid || !phi || Ri < 1) return mcv::fail(MCV_ERR_ARG, "bad Rossby wave arguments");
  const double R = Ri;
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npts; ++k) {
    const double sl = std::sin(latP[k]), cl = std::cos(latP[k]), lon = lonP[k];
    const double cR1 = std::pow(cl, R - 1), cR = cR1 * cl;
    // the wave part of the case-6 velocity, without the solid-body rotation
    zonal[k] += radius * K * cR1 * (R * sq(sl) - sq(cl)) * std::cos(R * lon);
    merid[k] += -radius * K * R * cR1 * sl * std::sin(R * lon);
    // its cos(R lon) height term at linear order in K (Coriolis balance)
    const double B = 2. * kOmega * K / ((R + 1.) * (R + 2.)) * cR * ((sq(R) + 2. * R + 2.) - sq(R + 1.) * sq(cl));
    phi[k] += sq(radius) * B * std::cos(R * lon);
  }
  return MCV_OK;
}

extern "C" int mcv_sphere_to_cov(long long npts, const double *matrixG, const double *matrixIA, const double *zonal,
                                 const double *merid, double *u, double *v) {
  if (!matrixG || !matrixIA || !zonal || !merid || !u || !v) return mcv::fail(MCV_ERR_ARG, "null array");
#pragma omp parallel for schedule(static)
  for (long long k = 0; k < npts; ++k) {
    const double *G = matrixG + 4 * k, *IA = matrixIA + 4 * k;
    double m[4];
    mcv::matmul22(m, G, IA);
    u[k] = m[0] * zonal[k] + m[2] * merid[k];
    v[k] = m[1] * zonal[k] + m[3] * merid[k];
  }
  return MCV_OK;
}
