// bulk.cuh -- 1-D bulk copies global -> shared memory (cp.async.bulk, the
// non-tensor TMA path of sm_90+/sm_100a) completed on an mbarrier, with
// bounded waits.
//
// A bulk copy needs 16-byte aligned source and destination and a size that
// is a multiple of 16 bytes; callers check this on the host and fall back to
// plain loads otherwise.  Waits give up after kBulkSpin polls (each poll may
// suspend the thread for a short hardware-defined time) so a lost completion
// can never hang the GPU: the caller then reports CANOE_EBIT_TIMEOUT.
#pragma once

#include <cstdint>

namespace cb {

constexpr int kBulkSpin = 1 << 18;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count)
               : "memory");
}

// make mbarrier initialisation visible to the async proxy
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses of the same memory
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one plain arrival on mbarrier m
__device__ __forceinline__ void mbar_arrive(uint64_t *m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(m)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *m) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(m))
      : "memory");
}

// start moving [src, src + bytes) into L2 (no completion to wait for; the
// data is then read by ordinary loads); 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for phase `parity` of mbarrier m: false after `spins` polls
__device__ __forceinline__ bool mbar_wait(uint64_t *m, uint32_t parity, int spins = kBulkSpin) {
  for (int it = 0; it < spins; ++it)
    if (mbar_try_wait(m, parity)) return true;
  return false;
}

}  // namespace cb
