// Bulk copies from global to shared memory with the Tensor Memory Accelerator, completed on
// shared-memory mbarriers (sm_90+ PTX, used here on sm_100a).
//
// Rules kept by every caller:
//   - addresses 16-byte aligned and sizes multiples of 16 bytes (untiled cp.async.bulk);
//   - for tiled copies, the innermost coordinate times the element size a multiple of 16 bytes;
//   - no multicast: every copy lands in the issuing CTA's own shared memory;
//   - every wait is bounded: a wait that runs out reports it, and the kernel records an error
//     and returns instead of spinning.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace shz {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// An mbarrier expecting `count` arrivals per phase.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Makes mbarrier initialisation visible to the async proxy (before the first copy on it).
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Orders this thread's earlier generic-proxy accesses to shared memory before later async-proxy
// (TMA) accesses: issued before a copy overwrites memory that threads have read.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One arrival that also announces `bytes` of transfers the phase must see complete.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Untiled bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) into this CTA's
// shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Tiled 3D copy of the tensor map's box at (x, y, z) into this CTA's shared memory.
__device__ __forceinline__ void tile3d_g2s(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of parity `parity` to complete, at most `limit` tries (each try may suspend
// the thread for a short hardware-chosen time). False if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Tries of a wait for a copy before the kernel gives up (far above any copy's latency).
constexpr uint32_t WAIT_LIMIT = 1u << 22;

// Error codes a kernel records in its error word.
constexpr int ERR_TMA_TIMEOUT = 1;

}  // namespace tma
}  // namespace shz
