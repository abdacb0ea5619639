// Bulk-async (TMA engine) copies global -> shared with an mbarrier, written as
// inline PTX for sm_100a.  No multicast form is used anywhere: every copy reads
// this GPU's own HBM into the issuing CTA's shared memory.
//
// Rules the callers follow:
//   - source and destination 16-byte aligned, size a multiple of 16 bytes
//     (the padded adjacency layout guarantees both);
//   - one elected thread arms the barrier (arrive.expect_tx) and issues the
//     copies; every thread waits on the phase parity;
//   - waits are bounded: after kSpinLimit polls the wait reports failure and
//     the kernel records GARY_ERR_TIMEOUT instead of hanging.
#pragma once
#include <cstdint>

namespace gary {

constexpr uint32_t kSpinLimit = 1u << 24;   // polls of mbarrier.try_wait
constexpr uint32_t kBulkChunk = 32768;      // bytes per cp.async.bulk

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
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

// Bounded wait for the phase with the given parity: at most `polls` polls
// of try_wait (0 gives up at once).  Returns false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint32_t polls = kSpinLimit) {
  for (uint32_t i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Issue the copy of `bytes` (multiple of 16) in kBulkChunk pieces on one
// barrier phase.  Called by a single thread.
__device__ __forceinline__ void bulk_stage(void *dst, const void *src, uint32_t bytes,
                                           uint64_t *bar) {
  mbar_arrive_expect_tx(bar, bytes);
  const char *s = static_cast<const char *>(src);
  char *d = static_cast<char *>(dst);
  for (uint32_t off = 0; off < bytes; off += kBulkChunk) {
    uint32_t b = bytes - off < kBulkChunk ? bytes - off : kBulkChunk;
    bulk_copy_g2s(d + off, s + off, b, bar);
  }
}

}  // namespace gary
