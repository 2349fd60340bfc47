// mcv_internal.h -- helpers shared by the host-side sources of libmcv_gpu.
#pragma once

namespace mcv {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const char *msg);

// matmul(A, B) of two 2x2 column-major matrices, summing k = 1, 2 in order as
// the Fortran intrinsic does (used by covProjSphere2Plane / covProjPlane2Sphere,
// src/projection_mod.F90:60-96).
inline void matmul22(double out[4], const double *A, const double *B) {
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 2; ++i) out[i + 2 * j] = A[i] * B[2 * j] + A[i + 2] * B[1 + 2 * j];
}

}  // namespace mcv
