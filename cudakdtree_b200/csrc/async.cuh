// Bulk asynchronous copies (the TMA engine's cp.async.bulk) from global into
// shared memory, completed through a shared-memory mbarrier, and a bounded
// wait on that barrier.  sm_90 and later; used by the builder's partition
// pass to stage each CTA's chunk with one instruction per array.
#pragma once

#include <cstdint>

namespace ckb {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return uint32_t(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t arrivals)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals)
               : "memory");
  // make the initialised barrier visible to the async (bulk copy) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of incoming bulk-copy data
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

// global -> shared bulk copy; dst, src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity` of the barrier to complete; gives up after
// `polls` unsuccessful polls (each poll may suspend the thread for a
// hardware-defined while) and returns false, so that a barrier that never
// completes ends the kernel with an error instead of a hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t polls)
{
  for (uint32_t i = 0; i < polls; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace ckb
