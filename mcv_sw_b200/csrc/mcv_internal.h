// mcv_internal.h -- helpers shared by the host-side sources of libmcv_gpu.
#pragma once
#include <cuda_runtime.h>

#ifdef __CUDACC__
#define MCV_HD __host__ __device__
#else
#define MCV_HD
#endif

namespace mcv {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const char *msg);

// matmul(A, B) of two 2x2 column-major matrices, summing k = 1, 2 in order as
// the Fortran intrinsic does (used by covProjSphere2Plane / covProjPlane2Sphere,
// src/projection_mod.F90:60-96).
MCV_HD inline void matmul22(double out[4], const double *A, const double *B) {
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) out[i + 2 * j] = A[i] * B[2 * j] + A[i + 2] * B[1 + 2 * j];
}

// Inputs and device outputs of build_geometry_device (mcv_geometry.cu).
struct GeomArgs {
  int order, nc, npx, n, H, P;  // P: row pitch of the padded planes
  double radius, dx, x_min, pi;
  double *sqrtG, *ig11, *ig12, *ig22, *fcor;  // padded planes [6][npx][P]
  double4 *Mtab, *Ntab;                       // edge-strip matrices [24][H+1][n]
  int *giref;                                 // ghost cell index [H][n], 1..nc
  double2 *gcoef;                             // ghost offset and its cube [H][n]
  double4 *met1d;                             // 1-D metric table [npx] (split precision) or NULL
  int *err;                                   // set to 1 if a ghost point lies outside panel 5
};

// Enqueues the geometry kernels on stream s; 0 or a CUDA error code.
int build_geometry_device(const GeomArgs &a, cudaStream_t s);

// One member's seeded balanced-flow initial state on the device
// (mcv_set_member_balanced_flow).  Field pointers are the member's slices.
struct IcArgs {
  int order, nc, npx, n, H, P;
  double radius, dx, x_min, pi;
  double gh0, u0, alpha;  // tilted solid-body flow
  int lmax;               // harmonic degrees 1..lmax (0: none)
  const double *coef;     // device copy of the (lmax+1)^2 coefficients
  double ratio;           // target RMS / RMS of the unit-scale harmonic height
  int mountain;
  double h0, lon_c, lat_c, efold;
  double *u, *v, *phi, *phis;  // padded [6][npx][P]; phis holds the unit height between the passes
  float *phis32;               // split precision: FP32 phi_s, or NULL
  const double *sqrtG;
};
int ic_harmonics_device(const IcArgs &a, cudaStream_t s);
int ic_sums_device(const IcArgs &a, int mode, const double *x, double4 *partial, int blocks, cudaStream_t s);
int ic_fields_device(const IcArgs &a, cudaStream_t s);

}  // namespace mcv
