// bulk.cuh -- asynchronous bulk copies from global to shared memory (the
// sm_90+/sm_100 copy engine behind cp.async.bulk) completing on shared-memory
// mbarriers, with bounded waits.
//
// Used by the per-step gathers: a tile's packed records are one contiguous
// range of the record array, so one elected thread asks the copy engine for
// the whole range (in chunks, one mbarrier each) before the block stages its
// neighbour data; the records stream in while the threads gather, and no
// register or load slot is held for them.  Sources are this GPU's own
// memory, never a peer's, and no copy is multicast.
#pragma once
#include <cstdint>

namespace mega {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t arrivals) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals) : "memory");
}

// make the initialised barriers visible to the copy engine (async proxy)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of transfers completing on the barrier
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of the barrier, giving up after `limit` polls
// (each try_wait itself blocks for a bounded, implementation-defined time).
// Returns false on time-out; the caller records it in the status word.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int limit) {
  for (int k = 0; k < limit; ++k)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace mega
