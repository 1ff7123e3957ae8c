// Bulk asynchronous copies global → shared memory (the Blackwell/Hopper copy engine behind TMA,
// `cp.async.bulk`) completed on an mbarrier, with a bounded wait.
//
// Only this GPU's own memory is ever the source (no multicast). Addresses must be 16-byte
// aligned and sizes multiples of 16 bytes; the callers check that before choosing these paths.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace bwpm {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bulk_mbar_init(std::uint64_t* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
}

// makes mbarrier initialisation visible to the asynchronous proxy (before the first copy)
__device__ __forceinline__ void bulk_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// this thread's arrival, announcing `bytes` of copies that complete on the barrier
__device__ __forceinline__ void bulk_expect(std::uint64_t* mbar, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}"
               ::"r"(smem_addr(mbar)), "r"(bytes) : "memory");
}

// `bytes` from global `src` to shared `dst`, counted on `mbar`
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, std::uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(mbar)) : "memory");
}

__device__ __forceinline__ bool bulk_try(std::uint64_t* mbar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok) : "r"(smem_addr(mbar)), "r"(parity) : "memory");
  return ok != 0;
}

// Waits for phase `parity` of `mbar` for at most about 2 s; on giving up sets *status = 1 and
// returns false (the caller's results are then invalid and the host reports the error).
__device__ __forceinline__ bool bulk_wait(std::uint64_t* mbar, unsigned parity, int* status) {
  if (bulk_try(mbar, parity)) return true;
  long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    if (bulk_try(mbar, parity)) return true;
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 2000000000LL) {
      atomicExch(status, 1);
      return false;
    }
  }
}

}  // namespace bwpm
