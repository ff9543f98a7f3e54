// Bulk asynchronous copies (TMA, cp.async.bulk) global -> shared with
// mbarrier completion, for sm_100a. No multicast anywhere: every copy reads
// this GPU's own memory into the issuing CTA's shared memory.
//
// Every wait is bounded: after MBAR_SPIN_LIMIT polls (each try_wait already
// suspends for a while) the waiting thread records an error word and
// returns false; kernels then stop taking work and exit, and the host turns
// the error word into an error status.
#pragma once

#include <cstdint>

namespace ddm {

constexpr long long MBAR_SPIN_LIMIT = 1ll << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy accesses (a TMA write into a buffer just read).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// 1D bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return done != 0;
}

// Bounded wait for the given phase parity; false (and *err set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, int* err, int code) {
  for (long long i = 0; i < MBAR_SPIN_LIMIT; i++)
    if (mbar_try_wait(bar, phase)) return true;
  if (err) atomicExch(err, code);
  return false;
}

}  // namespace ddm
