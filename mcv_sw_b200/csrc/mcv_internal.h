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

// History-output staging (mcv_get_history): convert_wind_P2SP over the whole
// padded array of one member (src/spatial_operators_mod.F90:391-405) after
// addFillValue (src/output_mod.F90:230-248), with A IG evaluated per point from
// the equiangular formulas.  Writes component `which` (0 zonal, 1 meridional)
// in the caller's dense layout [6][npx][npx].  u, v: the member's pitched
// fields [6][npx][P].
int history_p2sp_device(const GeomArgs &a, const double *u, const double *v, int which, double *out,
                        cudaStream_t s);

// calc_VIA (src/diag_mod.F90:69-93) of a member's pitched field [6][npx][P]:
// cell averages with the reference's weightsOnPV (mesh_mod.F90:183-203,
// MCV4's /80 included), summed in its jDOF, iDOF order without FMA
// contraction, into (ics:ice, jcs:jce, 6) = [6][nc+2][nc+2] with zero halo
// cells (the layout of stat%uC).
int via_device(int order, int nc, int npx, int P, const double *f, double *out, cudaStream_t s);

// The normalized L1 / L2 / Linf of doc/orderCheck.m:63-81 between the cell
// averages (calc_VIA) of two members' pitched fields a and b of one grid,
// weighted by areaCell ([nc][nc], the same on every panel): per block
// partial[2 b] = {sum |a-b| w, sum |b| w, sum (a-b)^2 w, sum b^2 w} and
// partial[2 b + 1] = {max |a-b| w, max |b| w, 0, 0} over `blocks` blocks.
int norms_device(int order, int nc, int npx, int P, const double *a, const double *b, const double *area,
                 double4 *partial, int blocks, cudaStream_t s);

// areaCell of one panel (src/mesh_mod.F90:205-212 with EquiangularAllAreas,
// :240-276): [nc][nc] spherical-excess areas times radius^2.
void equiangular_cell_areas(int nc, double radius, double *area);

}  // namespace mcv
