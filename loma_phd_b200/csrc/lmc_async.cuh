// lmc_async.cuh -- asynchronous global -> shared copies for the
// persistent transform kernels: 1-D bulk copies through the TMA unit
// (cp.async.bulk with an mbarrier) and per-thread 16-byte cp.async.
//
// Every wait is bounded: after LMC_WAIT_LIMIT polls the kernel records
// LMC_ETIMEOUT in the handle's status word and gives up.  No copy here ever
// reads another GPU's memory and none uses cluster multicast.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lmcd {

constexpr uint32_t LMC_WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// one arrival that also announces `bytes` of incoming transactions
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait on phase `parity` (at most `limit` polls); false on
// time-out (status word set)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *status,
                                          uint32_t limit = LMC_WAIT_LIMIT) {
  for (uint32_t it = 0; it < limit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicExch(status, -4 /* LMC_ETIMEOUT */);
  return false;
}
// order this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy (bulk copy) writes to it
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size % 16 == 0)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// per-thread 16-byte asynchronous copy (L1 bypass) and its groups
__device__ __forceinline__ void cp16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace lmcd
