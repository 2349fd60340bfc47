/* orc_cases.c -- seeded initial states on the oracle's own mesh.
 *
 * TEST INFRASTRUCTURE ONLY (part of liborc.so): the CPU reference arm of the
 * benchmark builds its workloads with these routines and the oracle's mesh
 * (orc_get_mesh lonP / latP), so that it runs none of the GPU library's code.
 * They evaluate the same formulas as the library's host init chain:
 *   - the balanced solid-body zonal flow with a tilted axis: the case-5
 *     formulas of src/test_case_mod.F90:118-120 without the mountain;
 *   - real spherical harmonics, orthonormal on the unit sphere (normalised
 *     associated Legendre functions by the standard stable recurrences);
 *   - the Gaussian mountain hs = h0 exp(-(d/efold)^2): phi_s += g hs,
 *     phi -= g hs (test_case_mod.F90:117-128);
 *   - linear Rossby waves of zonal wavenumber R: the wave part of the case-6
 *     velocity (test_case_mod.F90:144-149) and its cos(R lon) height term at
 *     linear order.
 * Arrays are padded fields of npts points (any layout; point-wise).
 */
#include <math.h>
#include <stdlib.h>

static const double kOmegaC = 7.292E-5;      /* constants_mod.F90:18 */
static const double kGravityC = 9.80616;     /* constants_mod.F90:16 */

static double sqc(double x) { return x * x; }

void orc_ic_tilted_zonal(long npts, const double *lon, const double *lat, double radius, double gh0, double u0,
                         double alpha, double *zonal, double *merid, double *phi) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < npts; k++) {
    const double lo = lon[k], la = lat[k];
    zonal[k] = u0 * (cos(la) * cos(alpha) + cos(lo) * sin(la) * sin(alpha));
    merid[k] = -u0 * sin(lo) * sin(alpha);
    phi[k] = gh0 - (radius * kOmegaC * u0 + sqc(u0) / 2.) * sqc(-cos(lo) * cos(la) * sin(alpha) + sin(la) * cos(alpha));
  }
}

/* phi += scale * sum_{l=1..lmax} sum_{m=-l..l} coef[l*l + l + m] Y_lm(lon, lat) */
int orc_ic_add_harmonics(long npts, const double *lon, const double *lat, int lmax, const double *coef, double scale,
                         double *phi) {
  if (lmax < 1 || lmax > 200) return -1;
  const int L = lmax, S = L + 1;
  const double pi = 2.0 * asin(1.0);
  int bad = 0;
#pragma omp parallel
  {
    double *P = malloc(sizeof(double) * (size_t)S * S);
    double *cm = malloc(sizeof(double) * (size_t)S), *sm = malloc(sizeof(double) * (size_t)S);
    if (!P || !cm || !sm) {
#pragma omp atomic write
      bad = 1;
    }
#pragma omp for schedule(static)
    for (long k = 0; k < npts; k++) {
      if (!P || !cm || !sm) continue;
      const double x = sin(lat[k]), s = cos(lat[k]);
      /* P[m*S + l]: normalised so that the integral over [-1, 1] of P^2 is 1 */
      P[0] = sqrt(0.5);
      for (int m = 1; m <= L; m++) P[m * S + m] = -sqrt((2. * m + 1.) / (2. * m)) * s * P[(m - 1) * S + m - 1];
      for (int m = 0; m < L; m++) P[m * S + m + 1] = sqrt(2. * m + 3.) * x * P[m * S + m];
      for (int m = 0; m <= L; m++)
        for (int l = m + 2; l <= L; l++) {
          const double a = sqrt((4. * l * l - 1.) / ((double)l * l - (double)m * m));
          const double b = sqrt(((l - 1.) * (l - 1.) - (double)m * m) / (4. * (l - 1.) * (l - 1.) - 1.));
          P[m * S + l] = a * (x * P[m * S + l - 1] - b * P[m * S + l - 2]);
        }
      for (int m = 0; m <= L; m++) {
        cm[m] = cos(m * lon[k]);
        sm[m] = sin(m * lon[k]);
      }
      double acc = 0.;
      for (int l = 1; l <= L; l++) {
        /* Y_l0 = P / sqrt(2 pi); Y_l,+-m = P cos|sin(m lon) / sqrt(pi) */
        acc += coef[l * l + l] * P[l] / sqrt(2. * pi);
        for (int m = 1; m <= l; m++) {
          const double pl = P[m * S + l] / sqrt(pi);
          acc += coef[l * l + l + m] * pl * cm[m] + coef[l * l + l - m] * pl * sm[m];
        }
      }
      phi[k] += scale * acc;
    }
    free(P);
    free(cm);
    free(sm);
  }
  return bad ? -3 : 0;
}

void orc_ic_add_mountain(long npts, const double *lon, const double *lat, double radius, double lon_c, double lat_c,
                         double h0, double efold, double *phi, double *phi_s) {
#pragma omp parallel for schedule(static)
  for (long k = 0; k < npts; k++) {
    const double cang = sin(lat_c) * sin(lat[k]) + cos(lat_c) * cos(lat[k]) * cos(lon[k] - lon_c);
    const double d = radius * acos(fmax(-1., fmin(1., cang)));
    const double hs = kGravityC * h0 * exp(-sqc(d / efold));
    phi_s[k] += hs;
    phi[k] -= hs;
  }
}

void orc_ic_add_rossby_wave(long npts, const double *lon, const double *lat, double radius, int Ri, double K,
                            double *zonal, double *merid, double *phi) {
  const double R = Ri;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < npts; k++) {
    const double sl = sin(lat[k]), cl = cos(lat[k]), lo = lon[k];
    const double cR1 = pow(cl, R - 1), cR = cR1 * cl;
    zonal[k] += radius * K * cR1 * (R * sqc(sl) - sqc(cl)) * cos(R * lo);
    merid[k] += -radius * K * R * cR1 * sl * sin(R * lo);
    const double B = 2. * kOmegaC * K / ((R + 1.) * (R + 2.)) * cR * ((sqc(R) + 2. * R + 2.) - sqc(R + 1.) * sqc(cl));
    phi[k] += sqc(radius) * B * cos(R * lo);
  }
}
