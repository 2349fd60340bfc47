// mcv_ksum.cuh -- Neumaier-compensated sums for the device reductions
// (mass / energy diagnostics, initial-state normalisation).
#pragma once
#include <cuda_runtime.h>

namespace mcv {

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

}  // namespace mcv
