// mbarrier and 1-D bulk-copy helpers (inline PTX, sm_100a) shared by the
// kernels that stage data with the Tensor Memory Accelerator's bulk copies.
// Every wait is bounded: a wait that runs out returns false and the caller
// records an error instead of spinning on.
#pragma once
#include <stdint.h>

namespace mm {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase: false after ~2^22 polls (well over a
// second), which the caller turns into an error.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++) {
    if (mbar_try_wait(mbar, parity)) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// One arrival that also announces `bytes` of bulk copies completing on the barrier.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completing on `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory
// before async-proxy accesses (bulk copies, tensor-core reads) issued after it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 bytes global -> shared through L2 only (cp.async.cg; both addresses
// 16-byte aligned), no registers held while in flight.  A thread's copies are
// grouped by cp_async_commit; cp_async_wait<N> returns once at most N of its
// groups are still in flight (the hardware completes them: no polling).
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace mm
