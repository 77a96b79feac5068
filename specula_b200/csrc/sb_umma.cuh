// Fifth-generation tensor-core (tcgen05) helpers for sm_100a: tensor-memory
// allocation, the single-CTA BF16 MMA with FP32 accumulation in tensor
// memory, its commit to an mbarrier, tensor-memory loads and the fences that
// order them against thread barriers; plus the split of FP32 values into
// bf16 hi + lo pairs.
//
// Shared-memory operands use the no-swizzle K-major layout: one 16-byte
// segment holds 8 consecutive bf16 of K for one row; the segments of 8
// consecutive rows are contiguous (128 bytes) and consecutive 8-row groups
// follow at SBO = 128 bytes, so row m of a K-segment sits at m * 16 bytes;
// the two K-segments of one K=16 MMA step sit LBO bytes apart.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "sb_tma.cuh"

namespace sb {

// --- tensor memory ---------------------------------------------------------
// warp-collective: the allocating warp writes the base address to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// shared-memory writes of this thread -> visible to the tensor cores (async proxy)
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// --- MMA -------------------------------------------------------------------
// shared-memory matrix descriptor, no swizzle, K-major, SBO = 128 bytes
__device__ __forceinline__ uint64_t umma_desc_kmajor(const void *p, uint32_t lbo_bytes) {
    return (uint64_t)((smem_u32(p) & 0x3FFFFu) >> 4) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(128u >> 4) << 32) | ((uint64_t)1 << 46);   // bits 46-47: descriptor version 1
}

// instruction descriptor: A, B bf16 K-major, D f32, dense, M x N
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int m, int n) {
    return (1u << 4)                            // D format f32
           | (1u << 7)                          // A format bf16
           | (1u << 10)                         // B format bf16
           | ((uint32_t)(n >> 3) << 17)         // N / 8
           | ((uint32_t)(m >> 4) << 24);        // M / 16
}

// D[tmem] (+)= A * B^T, issued by one thread
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// the mbarrier completes one arrival once every MMA this thread issued before has finished
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// --- tensor-memory loads ---------------------------------------------------
// 32 lanes x 16 columns: thread l of the warp receives row (lane base + l)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
// wait for this thread's tensor-memory loads; the registers pass through the
// statement so that no use of them is scheduled before it
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                   "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                   "+r"(r[14]), "+r"(r[15])
                 :
                 : "memory");
}

// --- split BF16 --------------------------------------------------------------
// x = hi + lo + e with hi = bf16(x), lo = bf16(x - hi) (x - hi is exact in
// float32), |e| <= 2^-8 |x - hi| <= 2^-16 |x| up to underflow
__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}
__device__ __forceinline__ void split_bf16x8(const float (&x)[8], uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * q]), h1 = __float2bfloat16_rn(x[2 * q + 1]);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * q] - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * q + 1] - __bfloat162float(h1));
        h[q] = bf16x2_bits(h0, h1);
        l[q] = bf16x2_bits(l0, l1);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

}  // namespace sb
