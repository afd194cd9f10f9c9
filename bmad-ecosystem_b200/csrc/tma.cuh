// tma.cuh -- shared-memory staging of the element table with the bulk-copy engine.
//
// One thread arms an mbarrier with the byte count and issues cp.async.bulk copies (global ->
// this CTA's shared memory, no multicast) in chunks; every thread then waits on the barrier's
// phase with a bounded number of try_wait polls, so a copy that never completes turns into an
// error flag instead of a hang.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "table.h"

namespace bmadgpu {

constexpr uint32_t kBulkChunk = 32768;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
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

// Bounded wait for the given phase of the barrier; false if it did not complete in time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < kSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// 1-D bulk copy global -> this CTA's shared memory (no multicast), completion on an mbarrier.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Issued by one thread: arm the barrier for `bytes` and copy the table (16-byte multiple, 16-byte
// aligned source and destination) in kBulkChunk pieces.
__device__ __forceinline__ void stage_table_issue(uint8_t* dst, const uint8_t* src, uint32_t bytes, uint64_t* bar) {
  mbar_arrive_expect_tx(bar, bytes);
  for (uint32_t off = 0; off < bytes; off += kBulkChunk) {
    uint32_t n = bytes - off < kBulkChunk ? bytes - off : kBulkChunk;
    bulk_g2s(dst + off, src + off, n, bar);
  }
}

}  // namespace bmadgpu
