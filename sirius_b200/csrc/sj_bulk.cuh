// Bulk copies global -> shared memory on the TMA engine (cp.async.bulk, no tensor map, no
// multicast), completed on a shared-memory mbarrier, with a bounded wait.
//
// Rules the callers follow: source and destination 16-byte aligned, sizes multiples of 16 bytes;
// one thread issues the copies of a stage after arming the stage's mbarrier with the byte count
// (arrive.expect_tx); consumers wait for the stage's phase parity; a stage is refilled only after
// a CTA barrier that every reader of its previous contents has passed.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sj {

// Polls of a stage's mbarrier before a wait gives up (each try_wait may suspend for a while, so
// this bounds a wait to roughly a second); a copy lands in microseconds.
constexpr uint32_t kBulkWaitPolls = 1u << 20;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Waits until the phase with parity `parity` of `bar` has completed; false after `polls` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t polls) {
  for (uint32_t i = 0; i < polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace sj
