// umma.cuh — Blackwell 5th-generation tensor-core (tcgen05) building blocks
// as inline PTX: TMEM allocation, shared-memory matrix descriptors, the
// BF16 x BF16 -> FP32 MMA issued by one thread, its commit to an mbarrier,
// and the TMEM -> register loads of the epilogue.
//
// Shared-memory operand layout (no swizzle, "interleaved" core matrices):
// a core matrix is 8 rows x 16 bytes stored contiguously (128 B). For a
// stage tile of R rows (M or N) the 16-byte chunk (r, j) of a K-major
// operand — elements K = 8j..8j+7 of row r — sits at
//     j * (R * 16) + (r / 8) * 128 + (r % 8) * 16,
// and the chunk (k, c) of an MN-major operand — elements MN = 8c..8c+7 at
// K index k — at
//     (k / 8) * (R * 16) + c * 128 + (k % 8) * 16.
// Both are the canonical layouts with stride-byte-offset 128 B (adjacent
// core matrices along MN) and leading-byte-offset R * 16 B (along K).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "aw_common.cuh"
#include "bulk.cuh"

namespace aw {

// smem matrix descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4
// [32,46), version 1 [46,48), base offset 0, no swizzle [61,64) = 0
__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_addr, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// instruction descriptor of kind::f16: D F32, A and B BF16, M x N, majors
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N, int a_mn_major,
                                                       int b_mn_major) {
  return (1u << 4)                          // D format F32
         | (1u << 7)                        // A format BF16
         | (1u << 10)                       // B format BF16
         | ((uint32_t)a_mn_major << 15)     // A major
         | ((uint32_t)b_mn_major << 16)     // B major
         | ((uint32_t)(N >> 3) << 17)       // N / 8
         | ((uint32_t)(M >> 4) << 24);      // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive on `mbar` once every tcgen05 op this thread issued has completed
__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// one full warp: allocate `cols` TMEM columns (power of two >= 32), address
// to *dst in shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace aw
