// mcv_tma.cuh -- tensor-memory-accelerator (TMA) staging of stage-kernel tiles
// on sm_100a: mbarrier and bulk-copy wrappers (inline PTX) and the tensor
// maps a stage kernel reads its input fields through.
//
// A tile's input fields are copied from HBM into shared memory by one thread
// with cp.async.bulk.tensor (one 2-D box per field: the tile with its halo
// cross, [LY rows][BX columns]); completion is counted in bytes on one
// mbarrier.  Rules kept here: every box starts at an x coordinate whose byte
// offset is a multiple of 16 (tile origins are multiples of 4 elements), boxes
// are 16-byte multiples wide, shared destinations are 128-byte aligned, loads
// only (no multicast), and every wait is bounded.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mcv {

// Input fields of one stage launch, in the order the kernel stages them.
// FP64 policy: us, vs, ps, phis, sqrtG, ig11, ig12, ig22.
// Split precision: yu, yv, yp (FP64), phis32, du, dv, dp (FP32).
struct TileMaps {
  CUtensorMap f[8];
  int total;  // work items of the launch: tiles x 6 panels x active members
  int pad[15];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes an initialised mbarrier visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// orders this thread's generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// one 2-D box of a tensor map, element coordinates (x fastest)
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// contiguous bytes (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for phase `parity` of the barrier: gives up after limit_ns of
// wall time (default about one second, far beyond the microseconds a tile's
// copies take) and at most 2^24 polls.  Returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = 1000000000ull) {
  const uint64_t t0 = global_ns();
  for (int it = 0; it < (1 << 24); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

}  // namespace mcv
