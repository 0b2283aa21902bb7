// Inline-PTX helpers for the 5th-generation tensor cores (tcgen05, sm_100a):
// tensor-memory allocation, shared-memory matrix descriptors, the BF16 MMA
// with FP32 accumulation in tensor memory, commit to an mbarrier and the
// tensor-memory -> register load of the epilogue.  One CTA group (no pairs),
// operands in the canonical K-major layout without swizzle:
//   core matrix = 8 rows x 16 bytes stored contiguously (128 B);
//   LBO = byte distance between the two 8-element K halves of a K=16 step;
//   SBO = byte distance between consecutive 8-row groups along M (or N).
#pragma once

#include <stdint.h>

namespace fs {

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// and stride byte offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo,
                                              uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // version
  return d;                // base offset 0, layout type 0 = no swizzle
}

// Instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4)                         // D format F32
         | (1u << 7)                       // A format BF16
         | (1u << 10)                      // B format BF16
         | ((uint32_t)(N >> 3) << 17)      // N / 8
         | ((uint32_t)(M >> 4) << 24);     // M / 16
}

// The same with both operands MN-major (the M or N index contiguous in 16-byte
// groups of 8 elements, K the strided index): bits 15 and 16 of the
// instruction descriptor.  With no swizzle a core matrix is then 8 K-rows of
// 16 bytes; LBO = byte distance between 8-row K groups, SBO = byte distance
// between 8-element M (or N) groups.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int M, int N) {
  return umma_idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}

// Make this thread's generic-proxy shared-memory writes visible to the async
// proxy (tensor-core operand reads, TMA) before a barrier.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(dst_smem)),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T ; accumulate != 0 adds to D.
__device__ __forceinline__ void tc_mma_bf16(uint32_t d_tmem, uint64_t adesc,
                                            uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrive once on `bar` when every MMA issued so far by this thread is done.
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          (uint32_t)__cvta_generic_to_shared(bar))
      : "memory");
}

// 32 lanes x 32 bit, 16 consecutive columns per thread (thread = lane).
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
        "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
        "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace fs
