// mcv_noalloc.cu -- total mass and energy of caller-owned device states
// without allocating any memory.
//
// mcv_mass_energy (mcv_gpu.cu) needs a handle, which owns a device pool made
// with cudaMalloc.  Some callers cannot allocate device memory when they need
// these diagnostics: code whose device memory belongs to a framework's own
// caching allocator (PyTorch and similar), which must account for every byte
// and cannot have a library grab memory behind its back; time-critical loops
// that must not pay for cudaMalloc/cudaFree, which can block and synchronise
// the whole device; and processes running close to their memory budget, where
// an allocation in the middle of a forecast could fail.  For them,
// mcv_mass_energy_noalloc reads states that already live in the caller's device
// memory and keeps its scratch (one partial sum per block and member, and the
// per-member results) in a fixed static device array.
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents.  Each call overwrites every slot it later reads, so nothing
// has to start at zero; two calls that overlap on the GPU (different host
// threads or streams at the same time) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/mcv_gpu.h"
#include "mcv_internal.h"

namespace mcv {
namespace {

constexpr int kNoallocMaxMembers = 64;  // members per call
constexpr int kNoallocBlocks = 148;     // partial sums per member (one block per SM of a B200)
constexpr int kNoallocThreads = 256;
constexpr int kNoallocMaxDevices = 64;

// [member][block] partial sums {mass, mass compensation, energy, energy
// compensation}, then [member] final {mass, energy}: 64 x 148 x 32 B + 1 KiB.
constexpr size_t kPartialDoubles = (size_t)kNoallocMaxMembers * kNoallocBlocks * 4;
constexpr size_t kResultDoubles = (size_t)kNoallocMaxMembers * 2;
static __device__ __align__(256) double g_noalloc_scratch[kPartialDoubles + kResultDoubles];

struct Comp {
  double s, c;
};
__device__ __forceinline__ void comp_add(Comp &a, double x) {
  // Neumaier's compensated summation
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
  else a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ void comp_merge(Comp &a, const Comp &b) {
  comp_add(a, b.s);
  a.c += b.c;
}

// calc_total_mass / calc_total_energy (src/diag_mod.F90:10-67) on states in the
// reference's layout: fields (npx, npx, 6[, member]) and matrixIG
// (2, 2, npx, npx, 6), column-major, halo included.  Block (b, m) sums the cells
// b, b + blocks, ... of member m: per-cell sums in the reference's jDOF/iDOF
// order, Neumaier-compensated over cells and across the block.
template <int D>
__global__ void __launch_bounds__(kNoallocThreads) noalloc_partials_kernel(
    int nc, int npx, const double *u, const double *v, const double *phi, const double *phis, const double *sqrtG,
    const double *IG, double *scratch) {
  constexpr int H = D - 1;
  const int m = blockIdx.y;
  const long long plane6 = 6LL * npx * npx;
  const double *um = u + m * plane6, *vm = v + m * plane6, *pm = phi + m * plane6, *sm_ = phis + m * plane6;
  const double w1[2] = {1., D == 3 ? 4. : 3.};
  const double wden = D == 3 ? 36. : 80.;
  const long long ncell = 6LL * nc * nc;
  Comp ms{0., 0.}, es{0., 0.};
  for (long long cidx = (long long)blockIdx.x * blockDim.x + threadIdx.x; cidx < ncell;
       cidx += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(cidx / ((long long)nc * nc));
    const int rem = (int)(cidx - (long long)p * nc * nc);
    const int jc = rem / nc, ic = rem % nc;
    double mc = 0., ec = 0.;
    for (int jd = 0; jd < D; ++jd)
      for (int id = 0; id < D; ++id) {
        const double wgt = w1[(id == 0 || id == D - 1) ? 0 : 1] * w1[(jd == 0 || jd == D - 1) ? 0 : 1] / wden;
        const long long o = (long long)(ic * (D - 1) + id + H) + (long long)npx * ((jc * (D - 1) + jd + H) + (long long)npx * p);
        const double sg = sqrtG[o], ph = pm[o], uu = um[o], vv = vm[o];
        const double g11 = IG[4 * o], g12 = IG[4 * o + 2], g22 = IG[4 * o + 3];
        const double cu = g11 * uu + g12 * vv, cv = g12 * uu + g22 * vv;
        mc = mc + wgt * (ph * sg);
        const double KE = 0.5 * ph * (uu * cu + vv * cv);
        const double PE = 0.5 * ((ph + sm_[o]) * (ph + sm_[o]));
        ec = ec + wgt * sg * (KE + PE);
      }
    comp_add(ms, mc);
    comp_add(es, ec);
  }
  __shared__ Comp rm[kNoallocThreads], re[kNoallocThreads];
  rm[threadIdx.x] = ms;
  re[threadIdx.x] = es;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      comp_merge(rm[threadIdx.x], rm[threadIdx.x + s]);
      comp_merge(re[threadIdx.x], re[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double *slot = scratch + ((size_t)m * kNoallocBlocks + blockIdx.x) * 4;
    slot[0] = rm[0].s;
    slot[1] = rm[0].c;
    slot[2] = re[0].s;
    slot[3] = re[0].c;
  }
}

// One thread per member folds that member's block partials (written by the
// kernel above in the same call) into {mass, energy}.
__global__ void noalloc_final_kernel(int members, double *scratch) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= members) return;
  Comp ms{0., 0.}, es{0., 0.};
  for (int b = 0; b < kNoallocBlocks; ++b) {
    const double *slot = scratch + ((size_t)m * kNoallocBlocks + b) * 4;
    comp_merge(ms, Comp{slot[0], slot[1]});
    comp_merge(es, Comp{slot[2], slot[3]});
  }
  double *res = scratch + kPartialDoubles + 2 * (size_t)m;
  res[0] = ms.s + ms.c;
  res[1] = es.s + es.c;
}

// Device address of the scratch array for the current device and context,
// looked up with that device current (the array's name in host code is only a
// stand-in for it and must never reach a kernel).  The address belongs to the
// module loaded into one context: after cudaDeviceReset (or anything else that
// destroys and recreates the device's primary context) the module is loaded
// again, possibly elsewhere.  So the cache is keyed on the context's unique id
// (cuCtxGetId: unique over the process's lifetime, unlike the CUcontext
// handle, which a recreated primary context may reuse) and the address is
// looked up again when the current context's id has changed.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

void *driver_fn(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

// id of the calling thread's current context; 0 if there is none yet
bool current_ctx_id(unsigned long long *id) {
  static CtxGetCurrentFn get_ctx = (CtxGetCurrentFn)driver_fn("cuCtxGetCurrent");
  static CtxGetIdFn get_id = (CtxGetIdFn)driver_fn("cuCtxGetId");
  *id = 0;
  if (!get_ctx || !get_id) return false;
  CUcontext ctx = nullptr;
  if (get_ctx(&ctx) != CUDA_SUCCESS) return false;
  if (!ctx) return true;
  return get_id(ctx, id) == CUDA_SUCCESS;
}

struct ScratchAddr {
  unsigned long long ctx_id;
  double *ptr;
};
std::mutex g_noalloc_mutex;
ScratchAddr g_noalloc_addr[kNoallocMaxDevices] = {};

int noalloc_scratch(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MCV_ERR_CUDA, "mcv_mass_energy_noalloc: no current CUDA device");
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(MCV_ERR_CUDA, "mcv_mass_energy_noalloc: device index too large");
  // id 0 before the runtime has bound a context to this thread; the symbol
  // lookup below binds the device's primary context
  unsigned long long id = 0;
  if (!current_ctx_id(&id)) return fail(MCV_ERR_CUDA, "mcv_mass_energy_noalloc: cannot read the current CUDA context");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  ScratchAddr &a = g_noalloc_addr[dev];
  if (id == 0 || !a.ptr || a.ctx_id != id) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return fail(MCV_ERR_CUDA, "mcv_mass_energy_noalloc: cannot resolve the scratch array's device address");
    }
    if (!current_ctx_id(&id) || id == 0)
      return fail(MCV_ERR_CUDA, "mcv_mass_energy_noalloc: cannot read the current CUDA context");
    a.ctx_id = id;
    a.ptr = (double *)p;
  }
  *out = a.ptr;
  return MCV_OK;
}

}  // namespace
}  // namespace mcv

extern "C" int mcv_mass_energy_noalloc(int order, int nc, int members, const double *u, const double *v,
                                       const double *phi, const double *phi_s, const double *sqrtG,
                                       const double *matrixIG, void *stream, double *mass, double *energy) {
  using namespace mcv;
  if (order != 3 && order != 4) return fail(MCV_ERR_ARG, "mcv_mass_energy_noalloc: order must be 3 or 4");
  if (nc < 2 || nc > 4096) return fail(MCV_ERR_ARG, "mcv_mass_energy_noalloc: nc out of range [2, 4096]");
  if (members < 1 || members > kNoallocMaxMembers)
    return fail(MCV_ERR_ARG, "mcv_mass_energy_noalloc: members must be 1..64 (the fixed scratch holds 64)");
  if (!u || !v || !phi || !phi_s || !sqrtG || !matrixIG || !mass || !energy)
    return fail(MCV_ERR_ARG, "mcv_mass_energy_noalloc: NULL pointer");
  double *scratch = nullptr;
  if (int rc = noalloc_scratch(&scratch)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const int npx = nc * (order - 1) + 1 + 2 * (order - 1);
  const dim3 grid(kNoallocBlocks, members);
  if (order == 3)
    noalloc_partials_kernel<3><<<grid, kNoallocThreads, 0, s>>>(nc, npx, u, v, phi, phi_s, sqrtG, matrixIG, scratch);
  else
    noalloc_partials_kernel<4><<<grid, kNoallocThreads, 0, s>>>(nc, npx, u, v, phi, phi_s, sqrtG, matrixIG, scratch);
  noalloc_final_kernel<<<1, kNoallocMaxMembers, 0, s>>>(members, scratch);
  double res[2 * kNoallocMaxMembers];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(res, scratch + kPartialDoubles, sizeof(double) * 2 * members, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    fail(MCV_ERR_CUDA, cudaGetErrorString(e));
    return MCV_ERR_CUDA;
  }
  for (int m = 0; m < members; ++m) {
    mass[m] = res[2 * m];
    energy[m] = res[2 * m + 1];
  }
  return MCV_OK;
}
