// bulk.cuh — Hopper/Blackwell bulk-copy (TMA, non-tensor) and mbarrier
// helpers, written as inline PTX.
//
// A contiguous global range is copied into shared memory by one
// cp.async.bulk issued from one thread and completed on an mbarrier the
// whole CTA waits on; shared memory is written back with one bulk store.
// No multicast anywhere. Every wait is bounded: after kMaxWaitIters
// unsuccessful try_wait polls the kernel records a timeout in the caller's
// device status word and gives up instead of spinning forever.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace aw {

constexpr int kMaxWaitIters = 1 << 22;
// status word codes
constexpr int kStatusOk = 0;
constexpr int kStatusWaitTimeout = 1;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gmem_src, uint32_t bytes,
                                          uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(mbar))
      : "memory");
}

// Waits for phase `parity` of the mbarrier; false (and *status set) after
// max_iters unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, int *status,
                                          int max_iters = kMaxWaitIters) {
  for (int it = 0; it < max_iters; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  if (status) atomicExch(status, kStatusWaitTimeout);
  return false;
}

// shared -> global; the caller fences (fence_async_smem) and synchronises
// the CTA before one thread issues this, then that thread calls
// bulk_wait_read before the CTA may exit
__device__ __forceinline__ void bulk_store(void *gmem_dst, const void *smem_src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmem_dst),
               "r"(smem_u32(smem_src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// 3D tensor tile load through a TMA descriptor (no multicast); OOB box
// elements read as zero and still count toward the transaction bytes
__device__ __forceinline__ void tma_load_3d(void *smem_dst, const void *tmap, int x, int y, int z,
                                            uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(mbar))
      : "memory");
}

// 5D tensor tile load (no multicast): coordinates innermost first; a box
// reaching outside the tensor reads zeros there (the innermost coordinate
// must stay a multiple of 16 bytes; the others may be negative)
__device__ __forceinline__ void tma_load_5d(void *smem_dst, const void *tmap, int c0, int c1, int c2,
                                            int c3, int c4, uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(mbar))
      : "memory");
}

// 3D tensor tile store; out-of-bounds box elements are not written
__device__ __forceinline__ void tma_store_3d(const void *tmap, int x, int y, int z,
                                             const void *smem_src) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::
          "l"(tmap),
      "r"(x), "r"(y), "r"(z), "r"(smem_u32(smem_src))
      : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// makes this thread's generic-proxy shared-memory writes visible to the
// async proxy (bulk stores)
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace aw
