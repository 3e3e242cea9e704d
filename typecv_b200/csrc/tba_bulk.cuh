// Bulk copies (cp.async.bulk, the copy engine of sm_90+) between global and shared memory, with
// completion on shared-memory mbarriers.  Every wait is bounded: a wait that runs out returns
// false, and the caller records an error and stops instead of hanging.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace tba {

constexpr uint32_t kBulkWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t bulk_smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One expected arrival per phase (the producer's).
__device__ __forceinline__ void bulk_bar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

// Makes the barriers' initialisation visible to the copy engine.
__device__ __forceinline__ void bulk_bar_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// The producer's arrival announcing `bytes` of copies that complete this phase.
__device__ __forceinline__ void bulk_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// The producer's arrival for a phase with no copies.
__device__ __forceinline__ void bulk_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// A global-to-shared copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) that
// completes its bytes on `bar`.
__device__ __forceinline__ void bulk_load(uint32_t bar, uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Waits, a bounded number of times, for the phase of `bar` with the given parity to complete.
__device__ __forceinline__ bool bulk_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t k = 0; k < kBulkWaitLimit; k++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace tba
