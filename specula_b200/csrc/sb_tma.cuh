// Tensor-memory-accelerator (TMA) helpers for sm_100a: mbarrier waits with an
// iteration bound, 2-D tiled bulk loads into shared memory with an L2
// eviction hint, and the host-side tensor-map encoding.  Every load goes to
// the issuing CTA's own shared memory and only ever reads this GPU's own
// memory.
#pragma once

#include <cuda.h>

#include "sb_common.cuh"

namespace sb {

// about one second of SM clock cycles: the bound of every mbarrier wait
constexpr long long kMbarWaitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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

// Wait for the phase of `bar` with the given parity to complete; false after
// kMbarWaitCycles (the caller records the timeout and stops).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > kMbarWaitCycles) return false;
    return true;
}

// try_wait with a suspend-time hint: the thread may sleep in the barrier
// (up to `ns` nanoseconds, or until the phase completes) instead of spinning
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

// mbar_wait for many waiting warps: they sleep in the barrier between polls
// (same bound, false after kMbarWaitCycles)
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t *bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait_sleep(bar, parity, 20000u))
        if (clock64() - t0 > kMbarWaitCycles) return false;
    return true;
}

// L2 policy for data read exactly once (lines evicted first, so the working
// set of concurrently running kernels stays in L2)
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// 2-D tiled TMA load of the box at element coordinates (x, y) into shared
// memory, completing on `bar`.  x * element size must be a multiple of 16.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar,
                                            uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// L2 policy for data read by many CTAs (lines kept over streamed data)
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// 1-D bulk copy (no tensor map) of `bytes` contiguous bytes from this GPU's
// global memory into this CTA's shared memory, completing on `bar`.  Both
// addresses 16-byte aligned, `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_load_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                             uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// 3-D tiled TMA load of the box at element coordinates (x, y, z), completing
// on `bar`.  x * element size must be a multiple of 16.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar,
                                            uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// Host: encode a row-major float32 matrix (rows x cols, row stride
// `ld` elements) as a 2-D tensor map with box (box_rows x box_cols);
// out-of-range elements of a box read as zero.  Returns SB_OK or a status.
int tensor_map_2d_f32(CUtensorMap *map, const float *base, int rows, int cols, int ld, int box_rows, int box_cols);


// Streaming multiprocessors of the current device (cached per device).
int sm_count();

}  // namespace sb
