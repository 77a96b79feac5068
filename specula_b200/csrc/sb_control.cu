// Reconstructor, integrator and DM projection on the B200.
//
// All three are HBM-streaming: the reconstructor reads R once per step
// (n_modes x n_slopes), the DM projection reads the influence functions once
// per step (n_modes x n_valid, the largest array of the loop).  Both kernels
// issue 16-byte loads with several in flight per thread and reduce in a
// fixed order, so results are bit-reproducible run to run.
#include "sb_common.cuh"

namespace {

// modes[m] = sum_j R[m][j] * s[j]: one CTA per row (modalrec.py:159)
template <bool VEC>
__global__ void __launch_bounds__(256) gemv_rows_kernel(const float *__restrict__ R, int ncols, int ldr,
                                                        const float *__restrict__ s, float *__restrict__ y) {
    __shared__ float red[33];
    const int m = blockIdx.x;
    const float *row = R + (size_t)m * ldr;
    float acc = 0.f;
    if (VEC) {
        const int n4 = ncols >> 2;
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
        const float4 *s4 = reinterpret_cast<const float4 *>(s);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 4
        for (int j = threadIdx.x; j < n4; j += blockDim.x) {
            const float4 r = __ldg(r4 + j), v = __ldg(s4 + j);
            a0 = fmaf(r.x, v.x, a0);
            a1 = fmaf(r.y, v.y, a1);
            a2 = fmaf(r.z, v.z, a2);
            a3 = fmaf(r.w, v.w, a3);
        }
        acc = (a0 + a1) + (a2 + a3);
        for (int j = (n4 << 2) + threadIdx.x; j < ncols; j += blockDim.x) acc = fmaf(row[j], s[j], acc);
    } else {
        for (int j = threadIdx.x; j < ncols; j += blockDim.x) acc = fmaf(row[j], s[j], acc);
    }
    acc = sb::block_sum(acc, red);
    if (threadIdx.x == 0) y[m] = acc;
}

// 2-tap IIR per mode, operation order of iir_filter.py:100-211 (no FMA
// contraction, so float32 results match the reference bit for bit)
__global__ void integrator_kernel(sb_iir_plan p, const float *__restrict__ delta, float *__restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n) return;
    float *st = p.state + (size_t)e * p.total;
    if (p.shift)
        for (int k = p.total - 1; k >= 1; --k) st[k] = st[k - 1];
    float *ist = p.ist + 2 * e, *ost = p.ost + 2 * e;
    const float *num = p.num + 2 * e, *den = p.den + 2 * e;
    ost[0] = ost[1];
    ost[1] = 0.f;
    ist[0] = ist[1];
    ist[1] = 0.f;
    ist[1] = delta[e];
    const float factor = __fdiv_rn(1.0f, den[1]);
    const float num_c = __fadd_rn(__fmul_rn(num[0], ist[0]), __fmul_rn(num[1], ist[1]));
    const float den_c = __fmul_rn(den[0], ost[0]);
    const float y = __fmul_rn(factor, __fsub_rn(num_c, den_c));
    ost[1] = y;
    st[0] = y;
    float o;
    if (p.rem == 0.f) {
        o = st[p.k_out];
    } else {
        o = __fadd_rn(__fmul_rn(p.rem, st[p.k_out]), __fmul_rn(p.one_minus_rem, st[p.k_out - 1]));
    }
    out[e] = o;
    if (p.out_next) p.out_next[e] = st[p.k_out - 1];
}

// phase[idx[p]] = sum_m c[m] * IF[m][p].
// Persistent kernel: one 512-thread CTA per SM walks column tiles of
// 32*W pixels (tile += gridDim.x).  Inside a tile the 16 warps split the
// modes (warp w takes w, w+16, ...), each lane keeps W columns, and 8 rows
// are loaded back to back so 8 x 16 bytes are in flight per thread
// (~9.7 MB GPU-wide, enough to cover HBM latency).  Partial tiles are
// reduced across warps in shared memory in a fixed order.  Holding one CTA
// per SM leaves room on every SM for kernels running concurrently on other
// streams (the SH chain of the pipelined loop step).
constexpr int kDmWarps = 16;
constexpr int kDmUnroll = 8;

template <int W>
__global__ void __launch_bounds__(32 * kDmWarps, 2) dm_project_kernel(const float *__restrict__ IF, int nmodes,
                                                                      int nvalid, int ld,
                                                                      const float *__restrict__ cmd, int ncmd,
                                                                      float sign, const int32_t *__restrict__ idx,
                                                                      float *__restrict__ phase) {
    extern __shared__ float sm[];
    float *c = sm;                               // nmodes (sign applied)
    float *part = sm + ((nmodes + 3) & ~3);      // kDmWarps x 32*W
    for (int m = threadIdx.x; m < nmodes; m += blockDim.x) c[m] = m < ncmd ? sign * cmd[m] : 0.f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (nvalid + 32 * W - 1) / (32 * W);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int col0 = tile * 32 * W + lane * W;
        float acc[W];
#pragma unroll
        for (int k = 0; k < W; ++k) acc[k] = 0.f;
        if (W == 4 && col0 + 3 < nvalid) {
            const float *base = IF + col0;
            int m = warp;
            for (; m + (kDmUnroll - 1) * kDmWarps < nmodes; m += kDmUnroll * kDmWarps) {
                float4 v[kDmUnroll];
#pragma unroll
                for (int u = 0; u < kDmUnroll; ++u)
                    v[u] = __ldg(reinterpret_cast<const float4 *>(base + (size_t)(m + u * kDmWarps) * ld));
#pragma unroll
                for (int u = 0; u < kDmUnroll; ++u) {
                    const float cm = c[m + u * kDmWarps];
                    acc[0] = fmaf(cm, v[u].x, acc[0]);
                    acc[1] = fmaf(cm, v[u].y, acc[1]);
                    acc[2] = fmaf(cm, v[u].z, acc[2]);
                    acc[3] = fmaf(cm, v[u].w, acc[3]);
                }
            }
            for (; m < nmodes; m += kDmWarps) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(base + (size_t)m * ld));
                const float cm = c[m];
                acc[0] = fmaf(cm, v.x, acc[0]);
                acc[1] = fmaf(cm, v.y, acc[1]);
                acc[2] = fmaf(cm, v.z, acc[2]);
                acc[3] = fmaf(cm, v.w, acc[3]);
            }
        } else if (col0 < nvalid) {
            for (int m = warp; m < nmodes; m += kDmWarps) {
                const float cm = c[m];
#pragma unroll
                for (int k = 0; k < W; ++k)
                    if (col0 + k < nvalid) acc[k] = fmaf(cm, __ldg(IF + (size_t)m * ld + col0 + k), acc[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < W; ++k) part[warp * 32 * W + lane * W + k] = acc[k];
        __syncthreads();
        for (int t = threadIdx.x; t < 32 * W; t += blockDim.x) {
            const int col = tile * 32 * W + t;
            if (col < nvalid) {
                float s = 0.f;
#pragma unroll
                for (int w = 0; w < kDmWarps; ++w) s += part[w * 32 * W + t];
                phase[idx[col]] = s;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// DM projection streamed through shared memory by the bulk-copy (TMA) engine.
// One CTA per SM: warp 4 (one elected lane) issues cp.async.bulk row copies
// of a 256-column tile into a 6-stage ring (16 rows per stage, 96 KB) that
// completes on an mbarrier; warps 0-3 (128 threads, 2 columns each)
// accumulate sum_m c[m] * IF[m][col] from shared memory and release the
// stage.  The copy engine keeps ~14 MB in flight GPU-wide with 160 threads
// and no registers per byte in flight, which leaves every SM free for the
// kernels of the SH chain running concurrently on another stream.
// Every wait is bounded (about one second of clock cycles); on timeout the
// kernel records the stage in g_sb_timeout and returns.
// ---------------------------------------------------------------------------
constexpr int kTmaConsumers = 128;
constexpr int kTmaTileCols = 256;
constexpr int kTmaRows = 16;
constexpr int kTmaStages = 6;
constexpr long long kWaitCycles = 2000000000LL;

__device__ int g_sb_timeout = 0;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
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
// bounded wait: false (and the timeout flag set) after ~1 s
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int where) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            atomicExch(&g_sb_timeout, where);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__global__ void __launch_bounds__(kTmaConsumers + 32, 1)
    dm_project_tma_kernel(const float *__restrict__ IF, int nmodes, int nvalid, int ld, const float *__restrict__ cmd,
                          int ncmd, float sign, const int32_t *__restrict__ idx, float *__restrict__ phase) {
    extern __shared__ __align__(128) unsigned char smem[];
    float *ring = reinterpret_cast<float *>(smem);                       // [stages][rows][tile]
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)kTmaStages * kTmaRows * kTmaTileCols * 4);
    uint64_t *empty = full + kTmaStages;
    float *c = reinterpret_cast<float *>(empty + kTmaStages);
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int st = 0; st < kTmaStages; ++st) {
            mbar_init(&full[st], 1);
            mbar_init(&empty[st], kTmaConsumers);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    for (int m = tid; m < nmodes; m += blockDim.x) c[m] = m < ncmd ? sign * cmd[m] : 0.f;
    __syncthreads();
    const int ntiles = (nvalid + kTmaTileCols - 1) / kTmaTileCols;
    const int nst = (nmodes + kTmaRows - 1) / kTmaRows;
    if (tid >= kTmaConsumers) {
        // producer: one lane of the last warp
        if (tid != kTmaConsumers) return;
        uint32_t it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const int col0 = tile * kTmaTileCols;
            const int width = min(kTmaTileCols, ld - col0);
            for (int sg = 0; sg < nst; ++sg, ++it) {
                const int s = it % kTmaStages;
                // a fresh barrier counts as released for parity 1: the first
                // pass over the ring does not wait
                if (!mbar_wait(&empty[s], ((it / kTmaStages) & 1) ^ 1, 1)) {
                    abort_flag = 1;
                    return;
                }
                if (*((volatile int *)&abort_flag)) return;
                const int rows = min(kTmaRows, nmodes - sg * kTmaRows);
                mbar_arrive_expect_tx(&full[s], (uint32_t)(rows * width * 4));
                float *dst = ring + (size_t)s * kTmaRows * kTmaTileCols;
                const float *src = IF + (size_t)(sg * kTmaRows) * ld + col0;
                for (int r = 0; r < rows; ++r)
                    bulk_g2s(dst + r * kTmaTileCols, src + (size_t)r * ld, (uint32_t)(width * 4), &full[s]);
            }
        }
        // drain: wait (bounded) until the consumers released every stage, so
        // no copy issued by this CTA is still in flight when it exits
        for (uint32_t k = 0; k < kTmaStages && k < it; ++k) {
            const uint32_t j = it - 1 - k;
            if (!mbar_wait(&empty[j % kTmaStages], (j / kTmaStages) & 1, 3)) return;
        }
        return;
    }
    // consumers
    uint32_t it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int col0 = tile * kTmaTileCols;
        float a0 = 0.f, a1 = 0.f;
        for (int sg = 0; sg < nst; ++sg, ++it) {
            const int s = it % kTmaStages;
            if (!mbar_wait(&full[s], (it / kTmaStages) & 1, 2)) {
                abort_flag = 1;
                return;
            }
            const int rows = min(kTmaRows, nmodes - sg * kTmaRows);
            const float *buf = ring + (size_t)s * kTmaRows * kTmaTileCols + 2 * tid;
            const float *cm = c + sg * kTmaRows;
#pragma unroll 4
            for (int r = 0; r < rows; ++r) {
                const float2 v = *reinterpret_cast<const float2 *>(buf + r * kTmaTileCols);
                a0 = fmaf(cm[r], v.x, a0);
                a1 = fmaf(cm[r], v.y, a1);
            }
            mbar_arrive(&empty[s]);
        }
        const int col = col0 + 2 * tid;
        if (col < nvalid) phase[idx[col]] = a0;
        if (col + 1 < nvalid) phase[idx[col + 1]] = a1;
    }
}

size_t dm_tma_smem(int nmodes) {
    return (size_t)kTmaStages * kTmaRows * kTmaTileCols * 4 + 2 * kTmaStages * 8 + ((size_t)nmodes + 4) * 4;
}

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

}  // namespace

extern "C" int sb_modalrec(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes, float *modes,
                           void *stream) {
    sb::clear_error();
    if (!R || !slopes || !modes || n_modes < 0 || n_slopes < 0 || ldr < n_slopes)
        return sb::fail(SB_EINVAL, "sb_modalrec: bad args");
    if (n_modes == 0) return SB_OK;
    cudaStream_t st = sb::as_stream(stream);
    const bool vec = (ldr % 4 == 0) && ((uintptr_t)R % 16 == 0) && ((uintptr_t)slopes % 16 == 0);
    if (vec)
        gemv_rows_kernel<true><<<n_modes, 256, 0, st>>>(R, n_slopes, ldr, slopes, modes);
    else
        gemv_rows_kernel<false><<<n_modes, 256, 0, st>>>(R, n_slopes, ldr, slopes, modes);
    return sb::check_launch("gemv_rows_kernel");
}

extern "C" int sb_integrator(const sb_iir_plan *p, const float *delta, float *out, void *stream) {
    sb::clear_error();
    if (!p || !delta || !out || !p->num || !p->den || !p->ist || !p->ost || !p->state)
        return sb::fail(SB_EINVAL, "sb_integrator: null pointer");
    if (p->n < 0 || p->total < 1 || p->k_out < 0 || p->k_out >= p->total || (p->rem != 0.f && p->k_out < 1))
        return sb::fail(SB_EINVAL, "sb_integrator: bad state layout");
    if (p->out_next && (p->rem != 0.f || p->k_out < 1))
        return sb::fail(SB_EINVAL, "sb_integrator: out_next needs an integer delay >= 1");
    if (p->n == 0) return SB_OK;
    integrator_kernel<<<(p->n + 127) / 128, 128, 0, sb::as_stream(stream)>>>(*p, delta, out);
    return sb::check_launch("integrator_kernel");
}

extern "C" int sb_dm_project(const float *ifunc, int n_modes, int n_valid, int ld_if, const float *cmd, int n_cmd,
                             float sign, const int32_t *mask_idx, float *phase, void *stream) {
    sb::clear_error();
    if (!ifunc || !cmd || !mask_idx || !phase || n_modes < 1 || n_valid < 0 || ld_if < n_valid || n_cmd < 0)
        return sb::fail(SB_EINVAL, "sb_dm_project: bad args");
    if (n_cmd > n_modes) return sb::fail(SB_ESHAPE, "sb_dm_project: %d commands for %d modes", n_cmd, n_modes);
    if (n_valid == 0) return SB_OK;
    cudaStream_t st = sb::as_stream(stream);
    const bool vec = (ld_if % 4 == 0) && ((uintptr_t)ifunc % 16 == 0);
    const int W = vec ? 4 : 1;
    const size_t smem = (size_t)(((n_modes + 3) & ~3) + kDmWarps * 32 * W) * sizeof(float);
    if (smem > 200 * 1024) return sb::fail(SB_ESHAPE, "sb_dm_project: too many modes (%d)", n_modes);
    if (vec && ld_if % 32 == 0 && dm_tma_smem(n_modes) <= 200 * 1024) {
        static size_t tma_smem_set = 0;
        const size_t sm2 = dm_tma_smem(n_modes);
        if (sm2 > tma_smem_set) {
            cudaError_t e = cudaFuncSetAttribute(dm_project_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)sm2);
            if (e != cudaSuccess) return sb::fail(SB_ECUDA, "sb_dm_project: smem attribute: %s", cudaGetErrorString(e));
            tma_smem_set = sm2;
        }
        const int tiles = (n_valid + kTmaTileCols - 1) / kTmaTileCols;
        const int nb = tiles < sm_count() ? tiles : sm_count();
        dm_project_tma_kernel<<<nb, kTmaConsumers + 32, sm2, st>>>(ifunc, n_modes, n_valid, ld_if, cmd, n_cmd, sign,
                                                                 mask_idx, phase);
        return sb::check_launch("dm_project_tma_kernel");
    }
    const int ntiles = (n_valid + 32 * W - 1) / (32 * W);
    const int nblk = ntiles < sm_count() ? ntiles : sm_count();
    if (vec) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(dm_project_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dm_project_kernel<4><<<nblk, 32 * kDmWarps, smem, st>>>(ifunc, n_modes, n_valid, ld_if, cmd, n_cmd, sign,
                                                                mask_idx, phase);
    } else {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(dm_project_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dm_project_kernel<1><<<nblk, 32 * kDmWarps, smem, st>>>(ifunc, n_modes, n_valid, ld_if, cmd, n_cmd, sign,
                                                                mask_idx, phase);
    }
    return sb::check_launch("dm_project_kernel");
}

extern "C" int sb_device_timeout_flag(int *host_out) {
    sb::clear_error();
    if (!host_out) return sb::fail(SB_EINVAL, "sb_device_timeout_flag: null pointer");
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_sb_timeout, sizeof(int));
    if (e != cudaSuccess) return sb::fail(SB_ECUDA, "sb_device_timeout_flag: %s", cudaGetErrorString(e));
    *host_out = v;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_sb_timeout, &zero, sizeof(int));
    }
    return SB_OK;
}
