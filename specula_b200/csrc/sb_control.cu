// Reconstructor, integrator and DM projection on the B200.
//
// All three are HBM-streaming: the reconstructor reads R once per step
// (n_modes x n_slopes), the DM projection reads the influence functions once
// per step (n_modes x n_valid, the largest array of the loop).  The
// reconstructor issues 16-byte loads with several in flight per thread; the
// DM projection streams the influence functions through shared memory with
// 2-D TMA loads.  Sums run in a fixed order, so results are bit-reproducible
// run to run.
#include <new>
#include <vector>

#include "sb_common.cuh"
#include "sb_mc.cuh"
#include "sb_tma.cuh"

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

constexpr int kIirMaxTaps = 8;

// sum of t float32 terms in NumPy's order along a row: sequential below 8
// terms, the 8-accumulator pairwise tree at exactly 8
__device__ __forceinline__ float numpy_row_sum(const float (&v)[kIirMaxTaps], int t) {
    if (t == 8)
        return __fadd_rn(__fadd_rn(__fadd_rn(v[0], v[1]), __fadd_rn(v[2], v[3])),
                         __fadd_rn(__fadd_rn(v[4], v[5]), __fadd_rn(v[6], v[7])));
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k)
        if (k < t) acc = __fadd_rn(acc, v[k]);
    return acc;
}

// general IIR filter (n_num / n_den taps) for mode e: returns the new output
// and updates ist / ost in place (iir_filter.py:169-197)
__device__ __forceinline__ float iir_taps(const sb_iir_plan &p, int e, float delta) {
    const int ni = p.n_num, no = p.n_den;
    float *ist = p.ist + (size_t)ni * e, *ost = p.ost + (size_t)no * e;
    const float *num = p.num + (size_t)ni * e, *den = p.den + (size_t)no * e;
    float is[kIirMaxTaps], os[kIirMaxTaps], prod[kIirMaxTaps];
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k) {
        is[k] = (k + 1 < ni) ? ist[k + 1] : 0.f;       // delay the vectors (shift left, last column 0)
        os[k] = (k + 1 < no) ? ost[k + 1] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k)
        if (k == ni - 1) is[k] = delta;                // new input
    const float factor = __fdiv_rn(1.0f, den[no - 1]);
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k) prod[k] = k < ni ? __fmul_rn(num[k], is[k]) : 0.f;
    const float num_c = numpy_row_sum(prod, ni);
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k) prod[k] = k < no - 1 ? __fmul_rn(den[k], os[k]) : 0.f;
    const float den_c = numpy_row_sum(prod, no - 1);
    const float y = __fmul_rn(factor, __fsub_rn(num_c, den_c));
#pragma unroll
    for (int k = 0; k < kIirMaxTaps; ++k) {
        if (k < ni) ist[k] = is[k];
        if (k < no) ost[k] = (k == no - 1) ? y : os[k];
    }
    return y;
}

// IIR for mode e, operation order of iir_filter.py:100-211 (no FMA
// contraction, so float32 results match the reference bit for bit); the
// 2-tap integrator has its own straight-line path
__device__ __forceinline__ void iir_update(const sb_iir_plan &p, int e, float delta, float *__restrict__ out) {
    if (p.n_num != 2 || p.n_den != 2) {
        constexpr int kMaxTotal = 8;
        float *st = p.state + (size_t)e * p.total;
        float sv[kMaxTotal];
        const int total = p.total;
#pragma unroll
        for (int k = 0; k < kMaxTotal; ++k) sv[k] = k < total ? st[k] : 0.f;
        if (p.shift) {
#pragma unroll
            for (int k = kMaxTotal - 1; k >= 1; --k) sv[k] = sv[k - 1];
        }
        sv[0] = iir_taps(p, e, delta);
        float o;
        if (p.rem == 0.f) {
            o = sv[p.k_out];
        } else {
            o = __fadd_rn(__fmul_rn(p.rem, sv[p.k_out]), __fmul_rn(p.one_minus_rem, sv[p.k_out - 1]));
        }
#pragma unroll
        for (int k = 0; k < kMaxTotal; ++k)
            if (k < total) st[k] = sv[k];
        out[e] = o;
        if (p.out_next) p.out_next[e] = sv[p.k_out - 1];
        return;
    }
    // every load is issued before any store (the arrays may alias as far as
    // the compiler knows), so the update costs two memory round trips
    constexpr int kMaxTotal = 8;
    float *st = p.state + (size_t)e * p.total;
    float *ist = p.ist + 2 * e, *ost = p.ost + 2 * e;
    const float2 num = *reinterpret_cast<const float2 *>(p.num + 2 * e);
    const float2 den = *reinterpret_cast<const float2 *>(p.den + 2 * e);
    const float ist1 = ist[1], ost1 = ost[1];
    float sv[kMaxTotal];
    const int total = p.total;
#pragma unroll
    for (int k = 0; k < kMaxTotal; ++k) sv[k] = k < total ? st[k] : 0.f;
    // prepare_trigger: shift the state buffer
    if (p.shift) {
#pragma unroll
        for (int k = kMaxTotal - 1; k >= 1; --k) sv[k] = sv[k - 1];
    }
    // trigger_code: ost/ist shift left, new input in the last column
    const float ist0 = ist1, ost0 = ost1;
    const float factor = __fdiv_rn(1.0f, den.y);
    const float num_c = __fadd_rn(__fmul_rn(num.x, ist0), __fmul_rn(num.y, delta));
    const float den_c = __fmul_rn(den.x, ost0);
    const float y = __fmul_rn(factor, __fsub_rn(num_c, den_c));
    sv[0] = y;
    // post_trigger: delayed output
    float o;
    if (p.rem == 0.f) {
        o = sv[p.k_out];
    } else {
        o = __fadd_rn(__fmul_rn(p.rem, sv[p.k_out]), __fmul_rn(p.one_minus_rem, sv[p.k_out - 1]));
    }
    ist[0] = ist0;
    ist[1] = delta;
    ost[0] = ost0;
    ost[1] = y;
#pragma unroll
    for (int k = 0; k < kMaxTotal; ++k)
        if (k < total) st[k] = sv[k];
    out[e] = o;
    if (p.out_next) p.out_next[e] = sv[p.k_out - 1];
}

__global__ void integrator_kernel(sb_iir_plan p, const float *__restrict__ delta, float *__restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n) return;
    iir_update(p, e, delta[e], out);
}

// reconstructor row m (as gemv_rows_kernel) followed by the integrator update
// of mode m in the same CTA: one launch for Modalrec + Integrator
template <bool VEC>
__global__ void __launch_bounds__(256) gemv_iir_kernel(const float *__restrict__ R, int ncols, int ldr,
                                                       const float *__restrict__ s, float *__restrict__ y,
                                                       sb_iir_plan p, float *__restrict__ out) {
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
    if (threadIdx.x == 0) {
        y[m] = acc;
        if (m < p.n) iir_update(p, m, acc, out);
    }
}

// phase[idx[p]] = sum_m c[m] * IF[m][p]; CTA = 8 warps sharing a strip of
// 32*W columns, warp w takes modes w, w+8, ...; partial strips are reduced
// across warps in shared memory (fixed order).  W = 4 (float4) when the rows
// are 16-byte aligned, else 1.
template <int W>
__global__ void __launch_bounds__(256) dm_project_kernel(const float *__restrict__ IF, int nmodes, int nvalid,
                                                         int ld, const float *__restrict__ cmd, int ncmd, float sign,
                                                         const int32_t *__restrict__ idx,
                                                         float *__restrict__ phase) {
    extern __shared__ float sm[];
    float *c = sm;                     // nmodes
    float *part = sm + nmodes;         // 8 warps x 32*W
    for (int m = threadIdx.x; m < nmodes; m += blockDim.x) c[m] = m < ncmd ? sign * cmd[m] : 0.f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = blockIdx.x * 32 * W + lane * W;
    float acc[W];
#pragma unroll
    for (int k = 0; k < W; ++k) acc[k] = 0.f;
    if (col0 < nvalid) {
        if (W == 4 && col0 + 3 < nvalid) {
            const float *base = IF + col0;
            int m = warp;
            for (; m + 24 < nmodes; m += 32) {
                const float4 v0 = __ldg(reinterpret_cast<const float4 *>(base + (size_t)m * ld));
                const float4 v1 = __ldg(reinterpret_cast<const float4 *>(base + (size_t)(m + 8) * ld));
                const float4 v2 = __ldg(reinterpret_cast<const float4 *>(base + (size_t)(m + 16) * ld));
                const float4 v3 = __ldg(reinterpret_cast<const float4 *>(base + (size_t)(m + 24) * ld));
                const float c0 = c[m], c1 = c[m + 8], c2 = c[m + 16], c3 = c[m + 24];
                acc[0] = fmaf(c0, v0.x, acc[0]); acc[1] = fmaf(c0, v0.y, acc[1]);
                acc[2] = fmaf(c0, v0.z, acc[2]); acc[3] = fmaf(c0, v0.w, acc[3]);
                acc[0] = fmaf(c1, v1.x, acc[0]); acc[1] = fmaf(c1, v1.y, acc[1]);
                acc[2] = fmaf(c1, v1.z, acc[2]); acc[3] = fmaf(c1, v1.w, acc[3]);
                acc[0] = fmaf(c2, v2.x, acc[0]); acc[1] = fmaf(c2, v2.y, acc[1]);
                acc[2] = fmaf(c2, v2.z, acc[2]); acc[3] = fmaf(c2, v2.w, acc[3]);
                acc[0] = fmaf(c3, v3.x, acc[0]); acc[1] = fmaf(c3, v3.y, acc[1]);
                acc[2] = fmaf(c3, v3.z, acc[2]); acc[3] = fmaf(c3, v3.w, acc[3]);
            }
            for (; m < nmodes; m += 8) {
                const float4 v = __ldg(reinterpret_cast<const float4 *>(base + (size_t)m * ld));
                const float cm = c[m];
                acc[0] = fmaf(cm, v.x, acc[0]); acc[1] = fmaf(cm, v.y, acc[1]);
                acc[2] = fmaf(cm, v.z, acc[2]); acc[3] = fmaf(cm, v.w, acc[3]);
            }
        } else {
            for (int m = warp; m < nmodes; m += 8) {
                const float cm = c[m];
#pragma unroll
                for (int k = 0; k < W; ++k)
                    if (col0 + k < nvalid) acc[k] = fmaf(cm, __ldg(IF + (size_t)m * ld + col0 + k), acc[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < W; ++k) part[warp * 32 * W + lane * W + k] = acc[k];
    __syncthreads();
    for (int t = threadIdx.x; t < 32 * W; t += blockDim.x) {
        const int col = blockIdx.x * 32 * W + t;
        if (col < nvalid) {
            float s = 0.f;
#pragma unroll
            for (int w = 0; w < 8; ++w) s += part[w * 32 * W + t];
            phase[idx[col]] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// DM projection with TMA.  One CTA per SM.  A producer lane streams boxes of
// 32 IF rows x 256 columns (32 KB, one TMA load each) through a 3-stage ring
// in shared memory (L2 evict-first: each IF byte is read once per step);
// 2 consumer warps, four columns per thread, accumulate sum_m c[m] IF[m][col]
// in mode order and release each stage on an mbarrier.  The CTA keeps ~97 KB
// of shared memory, 96 threads and few registers, so the latency-bound
// kernels of the SH chain, running concurrently on another stream, find room
// on every SM while the copy engine keeps HBM busy.  Every wait is bounded:
// on timeout the kernel records it in g_dm_status, stops issuing, lets the
// copies already issued land (bounded as well) and returns.
// ---------------------------------------------------------------------------
constexpr int kDmRows = 32;            // IF rows per box (multiple of 4)
constexpr int kDmCols = 256;           // IF columns per box (four per consumer thread)
#ifndef SB_DM_STAGES
#define SB_DM_STAGES 3                 // ring depth (build-time: -DSB_DM_STAGES=n)
#endif
constexpr int kDmStages = SB_DM_STAGES;
constexpr int kDmConsumerWarps = kDmCols / 128;   // 4 columns per thread
constexpr int kDmMaxModes = 4096;      // command vector staged in shared memory

__device__ int g_dm_status = 0;        // nonzero: a bounded wait timed out

size_t dm_tma_smem_bytes(int nmodes) {
    const int nst = (nmodes + kDmRows - 1) / kDmRows;
    return 1024 + (size_t)kDmStages * kDmRows * kDmCols * 4 + 2 * kDmStages * 8 + (size_t)nst * kDmRows * 4;
}

__global__ void __launch_bounds__(32 * (kDmConsumerWarps + 1), 1)
    dm_project_tma_kernel(const __grid_constant__ CUtensorMap map, int nmodes, int nvalid,
                          const float *__restrict__ cmd, int ncmd, float sign, const int32_t *__restrict__ idx,
                          float *__restrict__ phase) {
    extern __shared__ unsigned char smem_raw[];
    // TMA destinations aligned to 1024 bytes
    unsigned char *base = smem_raw + ((1024 - (sb::smem_u32(smem_raw) & 1023)) & 1023);
    float *ring = reinterpret_cast<float *>(base);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + (size_t)kDmStages * kDmRows * kDmCols * 4);
    uint64_t *empty = full + kDmStages;
    float *c = reinterpret_cast<float *>(empty + kDmStages);
    __shared__ int abort_flag, issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nst = (nmodes + kDmRows - 1) / kDmRows;
    if (tid == 0) {
        for (int s = 0; s < kDmStages; ++s) {
            sb::mbar_init(&full[s], 1);
            sb::mbar_init(&empty[s], kDmConsumerWarps);
        }
        sb::mbar_init_fence();
        abort_flag = 0;
        issued = 0;
    }
    for (int m = tid; m < nst * kDmRows; m += blockDim.x) c[m] = (m < ncmd && m < nmodes) ? sign * cmd[m] : 0.f;
    __syncthreads();
    const int ntiles = (nvalid + kDmCols - 1) / kDmCols;
    const int bid = blockIdx.x, nblk = gridDim.x;
    const int my_tiles = bid < ntiles ? (ntiles - 1 - bid) / nblk + 1 : 0;
    const int total = my_tiles * nst;          // boxes this CTA streams
    if (warp == kDmConsumerWarps) {
        if (lane == 0) {
            const uint64_t pol = sb::l2_evict_first_policy();
            int q = 0;
            for (; q < total; ++q) {
                const int slot = q % kDmStages;
                // reuse a slot once all consumer warps released its last use
                if (q >= kDmStages && !sb::mbar_wait(&empty[slot], ((q / kDmStages) - 1) & 1)) {
                    atomicExch(&g_dm_status, 1);
                    abort_flag = 1;
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                const int tile = bid + (q / nst) * nblk;
                sb::mbar_arrive_expect_tx(&full[slot], kDmRows * kDmCols * 4);
                sb::tma_load_2d(ring + (size_t)slot * kDmRows * kDmCols, &map, tile * kDmCols, (q % nst) * kDmRows,
                                &full[slot], pol);
            }
            issued = q;
        }
    } else {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int q = 0; q < total; ++q) {
            const int slot = q % kDmStages;
            if (!sb::mbar_wait(&full[slot], (q / kDmStages) & 1)) {
                atomicExch(&g_dm_status, 2);
                abort_flag = 1;
                break;
            }
            if (*(volatile int *)&abort_flag) break;
            const int sg = q % nst;
            const float4 *buf = reinterpret_cast<const float4 *>(ring + (size_t)slot * kDmRows * kDmCols) + tid;
            const float4 *cm4 = reinterpret_cast<const float4 *>(c + sg * kDmRows);
#pragma unroll
            for (int r4 = 0; r4 < kDmRows / 4; ++r4) {
                const float4 cc = cm4[r4];
                const float cr[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float4 v = buf[(r4 * 4 + k) * (kDmCols / 4)];
                    acc.x = fmaf(cr[k], v.x, acc.x);
                    acc.y = fmaf(cr[k], v.y, acc.y);
                    acc.z = fmaf(cr[k], v.z, acc.z);
                    acc.w = fmaf(cr[k], v.w, acc.w);
                }
            }
            __syncwarp();
            if (lane == 0) sb::mbar_arrive(&empty[slot]);
            if (sg == nst - 1) {
                const int col = (bid + (q / nst) * nblk) * kDmCols + 4 * tid;
                if (col < nvalid) phase[idx[col]] = acc.x;
                if (col + 1 < nvalid) phase[idx[col + 1]] = acc.y;
                if (col + 2 < nvalid) phase[idx[col + 2]] = acc.z;
                if (col + 3 < nvalid) phase[idx[col + 3]] = acc.w;
                acc = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    }
    __syncthreads();
    if (abort_flag && tid == 0) {
        // let every issued copy land before the shared memory is released
        for (int q = 0; q < issued; ++q) sb::mbar_wait(&full[q % kDmStages], (q / kDmStages) & 1);
    }
}

// ---------------------------------------------------------------------------
// Batched (multi-right-hand-side) forms for Monte-Carlo realisations that
// share one mirror and one reconstructor: every influence-function and
// reconstructor element is read once per step for all realisations.
// ---------------------------------------------------------------------------

// phase_b[idx[p]] = sum_m c_b[m] IF[m][p] for b < NB.  Same TMA ring as
// dm_project_tma_kernel (32 x 256 boxes, evict-first), with NB accumulators
// per column and the NB command vectors staged in shared memory as
// [mode][NB].  RS = 1: 8 consumer warps, one column per thread.  RS = 2: 16
// consumer warps of 16 columns each; the two half-warps take the first and
// the second 16 mode rows of every stage and their partial sums meet by a
// shuffle at the end of the tile (twice the warps to hide shared-memory
// latency; another summation order, so not bit-identical to RS = 1).
constexpr int kDbWarps = 8;
// more stages than the single-vector kernel: the NB accumulators make each
// stage's consumption longer, and this kernel need not leave room for
// concurrent kernels
constexpr int kDbStages = 5;
constexpr int kDbMaxModes = 1024;
template <int NB>
size_t dm_batched_smem_bytes(int nmodes) {
    const int nst = (nmodes + kDmRows - 1) / kDmRows;
    return 1024 + (size_t)kDbStages * kDmRows * kDmCols * 4 + 2 * kDbStages * 8 + (size_t)nst * kDmRows * NB * 4;
}

template <int NB, int RS>
__global__ void __launch_bounds__(32 * (kDbWarps * RS + 1), 1)
    dm_project_batched_kernel(const __grid_constant__ CUtensorMap map, int nmodes, int nvalid,
                              const float *__restrict__ cmd, int ldc, int nb, float sign,
                              const int32_t *__restrict__ idx, float *__restrict__ phase, long long phase_stride) {
    static_assert(RS == 1 || RS == 2, "one or two mode-row groups");
    constexpr int NCW = kDbWarps * RS;            // consumer warps
    constexpr int RR = kDmRows / RS;              // mode rows per thread and stage
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = smem_raw + ((1024 - (sb::smem_u32(smem_raw) & 1023)) & 1023);
    float *ring = reinterpret_cast<float *>(base);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + (size_t)kDbStages * kDmRows * kDmCols * 4);
    uint64_t *empty = full + kDbStages;
    float *c = reinterpret_cast<float *>(empty + kDbStages);       // [mode][NB]
    __shared__ int abort_flag, issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nst = (nmodes + kDmRows - 1) / kDmRows;
    if (tid == 0) {
        for (int s = 0; s < kDbStages; ++s) {
            sb::mbar_init(&full[s], 1);
            sb::mbar_init(&empty[s], NCW);
        }
        sb::mbar_init_fence();
        abort_flag = 0;
        issued = 0;
    }
    for (int e = tid; e < nst * kDmRows * NB; e += blockDim.x) {
        const int m = e / NB, b = e - m * NB;
        c[e] = (m < nmodes && b < nb) ? sign * cmd[(size_t)b * ldc + m] : 0.f;
    }
    __syncthreads();
    const int ntiles = (nvalid + kDmCols - 1) / kDmCols;
    const int bid = blockIdx.x, nblk = gridDim.x;
    const int my_tiles = bid < ntiles ? (ntiles - 1 - bid) / nblk + 1 : 0;
    const int total = my_tiles * nst;
    if (warp == NCW) {
        if (lane == 0) {
            const uint64_t pol = sb::l2_evict_first_policy();
            int q = 0;
            for (; q < total; ++q) {
                const int slot = q % kDbStages;
                if (q >= kDbStages && !sb::mbar_wait(&empty[slot], ((q / kDbStages) - 1) & 1)) {
                    atomicExch(&g_dm_status, 3);
                    abort_flag = 1;
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                const int tile = bid + (q / nst) * nblk;
                sb::mbar_arrive_expect_tx(&full[slot], kDmRows * kDmCols * 4);
                sb::tma_load_2d(ring + (size_t)slot * kDmRows * kDmCols, &map, tile * kDmCols, (q % nst) * kDmRows,
                                &full[slot], pol);
            }
            issued = q;
        }
    } else {
        // this thread's column within the tile and first mode row within a stage
        const int col_l = RS == 1 ? warp * 32 + lane : warp * 16 + (lane & 15);
        const int r0 = RS == 1 ? 0 : (lane >> 4) * RR;
        float acc[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[b] = 0.f;
        for (int q = 0; q < total; ++q) {
            const int slot = q % kDbStages;
            // warp-uniform decisions: the lanes meet in shuffles below
            if (!__all_sync(0xffffffffu, sb::mbar_wait(&full[slot], (q / kDbStages) & 1))) {
                if (lane == 0) atomicExch(&g_dm_status, 4);
                abort_flag = 1;
                break;
            }
            if (__any_sync(0xffffffffu, *(volatile int *)&abort_flag)) break;
            const int sg = q % nst;
            const float *buf = ring + (size_t)slot * kDmRows * kDmCols + (size_t)r0 * kDmCols + col_l;
            const float4 *cm = reinterpret_cast<const float4 *>(c + ((size_t)sg * kDmRows + r0) * NB);
#pragma unroll 4
            for (int r = 0; r < RR; ++r) {
                const float v = buf[r * kDmCols];
#pragma unroll
                for (int b4 = 0; b4 < NB / 4; ++b4) {
                    const float4 cc = cm[r * (NB / 4) + b4];
                    acc[4 * b4 + 0] = fmaf(cc.x, v, acc[4 * b4 + 0]);
                    acc[4 * b4 + 1] = fmaf(cc.y, v, acc[4 * b4 + 1]);
                    acc[4 * b4 + 2] = fmaf(cc.z, v, acc[4 * b4 + 2]);
                    acc[4 * b4 + 3] = fmaf(cc.w, v, acc[4 * b4 + 3]);
                }
            }
            __syncwarp();
            if (lane == 0) sb::mbar_arrive(&empty[slot]);
            if (sg == nst - 1) {
                if constexpr (RS == 2) {
#pragma unroll
                    for (int b = 0; b < NB; ++b) acc[b] += __shfl_xor_sync(0xffffffffu, acc[b], 16);
                }
                const int col = (bid + (q / nst) * nblk) * kDmCols + col_l;
                if ((RS == 1 || lane < 16) && col < nvalid) {
                    const int pix = idx[col];
#pragma unroll
                    for (int b = 0; b < NB; ++b)
                        if (b < nb) phase[(size_t)b * phase_stride + pix] = acc[b];
                }
#pragma unroll
                for (int b = 0; b < NB; ++b) acc[b] = 0.f;
            }
        }
    }
    __syncthreads();
    if (abort_flag && tid == 0) {
        for (int q = 0; q < issued; ++q) sb::mbar_wait(&full[q % kDbStages], (q / kDbStages) & 1);
    }
}

// Register-blocked batched projection: every consumer thread keeps 4
// adjacent columns x NB realisations in registers.  Per mode row it does one
// 16-byte shared load of the box, NB/4 broadcast loads of the commands and
// 4*NB FMAs, so FMAs are ~90 % of the consumer instructions (the scalar form
// above spends a shared load per FMA group on one column).  A stage is NBX
// boxes of (32/NBX) mode rows x 256 columns side by side (32 KB), so a tile
// is 256*NBX columns with 2*NBX consumer warps, and every column still sums
// its modes in order from 0: the phases are bit-identical to the scalar
// form with one mode-row group.
template <int NBX, int ST = kDbStages>
size_t dm_c4_smem_bytes(int nmodes, int nb_max) {
    constexpr int rows = kDmRows / NBX;
    const int nst = (nmodes + rows - 1) / rows;
    return 1024 + (size_t)ST * kDmRows * kDmCols * 4 + 2 * ST * 8 + (size_t)nst * rows * nb_max * 4;
}

// the tiles bid, bid + nblk, ... of the columns; ST stages in the ring
template <int NB, int NBX, int ST = kDbStages>
__device__ __forceinline__ void dm_c4_body(const CUtensorMap &map, int nmodes, int nvalid, const float *__restrict__ cmd,
                                           int ldc, int nb, float sign, const int32_t *__restrict__ idx,
                                           float *__restrict__ phase, long long phase_stride, int bid, int nblk) {
    static_assert(NB % 4 == 0 && (NBX == 1 || NBX == 2 || NBX == 4), "NB multiple of 4, 1/2/4 boxes per stage");
    constexpr int NCW = 2 * NBX;                  // consumer warps: 128 columns each
    constexpr int ROWS = kDmRows / NBX;           // mode rows per stage
    constexpr int TW = kDmCols * NBX;             // columns per tile
    constexpr int BOX = ROWS * kDmCols;           // floats per box
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = smem_raw + ((1024 - (sb::smem_u32(smem_raw) & 1023)) & 1023);
    float *ring = reinterpret_cast<float *>(base);
    uint64_t *full = reinterpret_cast<uint64_t *>(base + (size_t)ST * kDmRows * kDmCols * 4);
    uint64_t *empty = full + ST;
    float *c = reinterpret_cast<float *>(empty + ST);       // [mode][NB]
    __shared__ int abort_flag, issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nst = (nmodes + ROWS - 1) / ROWS;
    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            sb::mbar_init(&full[s], 1);
            sb::mbar_init(&empty[s], NCW);
        }
        sb::mbar_init_fence();
        abort_flag = 0;
        issued = 0;
    }
    for (int e = tid; e < nst * ROWS * NB; e += blockDim.x) {
        const int m = e / NB, b = e - m * NB;
        c[e] = (m < nmodes && b < nb) ? sign * cmd[(size_t)b * ldc + m] : 0.f;
    }
    __syncthreads();
    const int ntiles = (nvalid + TW - 1) / TW;
    const int my_tiles = bid < ntiles ? (ntiles - 1 - bid) / nblk + 1 : 0;
    const int total = my_tiles * nst;
    if (warp == NCW) {
        if (lane == 0) {
            const uint64_t pol = sb::l2_evict_first_policy();
            int q = 0;
            for (; q < total; ++q) {
                const int slot = q % ST;
                if (q >= ST && !sb::mbar_wait(&empty[slot], ((q / ST) - 1) & 1)) {
                    atomicExch(&g_dm_status, 5);
                    abort_flag = 1;
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                const int tile = bid + (q / nst) * nblk;
                sb::mbar_arrive_expect_tx(&full[slot], kDmRows * kDmCols * 4);
                float *dst = ring + (size_t)slot * kDmRows * kDmCols;
#pragma unroll
                for (int x = 0; x < NBX; ++x)
                    sb::tma_load_2d(dst + x * BOX, &map, tile * TW + x * kDmCols, (q % nst) * ROWS, &full[slot], pol);
            }
            issued = q;
        }
    } else {
        // this thread's 4 columns: box tid / 64, columns 4 * (tid % 64) .. +3 of the box
        const int bx = tid >> 6, cb = 4 * (tid & 63);
        float acc[4][NB];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[j][b] = 0.f;
        for (int q = 0; q < total; ++q) {
            const int slot = q % ST;
            // warp-uniform decisions: the lanes meet in __syncwarp below
            if (!__all_sync(0xffffffffu, sb::mbar_wait(&full[slot], (q / ST) & 1))) {
                if (lane == 0) atomicExch(&g_dm_status, 6);
                abort_flag = 1;
                break;
            }
            if (__any_sync(0xffffffffu, *(volatile int *)&abort_flag)) break;
            const int sg = q % nst;
            const float4 *buf =
                reinterpret_cast<const float4 *>(ring + (size_t)slot * kDmRows * kDmCols + bx * BOX + cb);
            const float4 *cm = reinterpret_cast<const float4 *>(c + (size_t)sg * ROWS * NB);
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const float4 v = buf[r * (kDmCols / 4)];
#pragma unroll
                for (int b4 = 0; b4 < NB / 4; ++b4) {
                    const float4 cc = cm[r * (NB / 4) + b4];
                    const float cr[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        acc[0][4 * b4 + k] = fmaf(cr[k], v.x, acc[0][4 * b4 + k]);
                        acc[1][4 * b4 + k] = fmaf(cr[k], v.y, acc[1][4 * b4 + k]);
                        acc[2][4 * b4 + k] = fmaf(cr[k], v.z, acc[2][4 * b4 + k]);
                        acc[3][4 * b4 + k] = fmaf(cr[k], v.w, acc[3][4 * b4 + k]);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) sb::mbar_arrive(&empty[slot]);
            if (sg == nst - 1) {
                const int col0 = (bid + (q / nst) * nblk) * TW + bx * kDmCols + cb;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (col0 + j < nvalid) {
                        const int pix = idx[col0 + j];
#pragma unroll
                        for (int b = 0; b < NB; ++b)
                            if (b < nb) phase[(size_t)b * phase_stride + pix] = acc[j][b];
                    }
#pragma unroll
                    for (int b = 0; b < NB; ++b) acc[j][b] = 0.f;
                }
            }
        }
    }
    __syncthreads();
    if (abort_flag && tid == 0) {
        for (int q = 0; q < issued; ++q) sb::mbar_wait(&full[q % ST], (q / ST) & 1);
    }
}

template <int NB, int NBX>
__global__ void __launch_bounds__(32 * (2 * NBX + 1), 1)
    dm_project_batched_c4_kernel(const __grid_constant__ CUtensorMap map, int nmodes, int nvalid,
                                 const float *__restrict__ cmd, int ldc, int nb, float sign,
                                 const int32_t *__restrict__ idx, float *__restrict__ phase,
                                 long long phase_stride) {
    dm_c4_body<NB, NBX>(map, nmodes, nvalid, cmd, ldc, nb, sign, idx, phase, phase_stride, blockIdx.x, gridDim.x);
}


// modes_b[m] = sum_j R[m][j] s_b[j] for b < NB.  A CTA of 256 threads takes
// RB reconstructor rows; each thread walks the slope index in pairs (8-byte
// loads when the strides allow), loads the NB slope pairs once and uses them
// for all RB rows, so S is read from L2 once per RB rows and R streams from
// HBM once.  Per (row, vector): warp sums, then a fixed-order sum over the
// 8 warps (deterministic).  RB (1, 2, 4) is the SB_TUNE_MODALREC_BATCHED
// variant.
// rows m0 .. m0 + RB - 1; epi(m, b, t) receives each finished sum
template <int NB, int RB, class Epi>
__device__ __forceinline__ void gemv_rows_batched_body(const float *__restrict__ R, int nrows, int ncols, int ldr,
                                                       const float *__restrict__ S, int lds, int nb, int vec2, int m0,
                                                       Epi &&epi) {
    __shared__ float red[RB * NB][9];
    float acc[RB][NB];
#pragma unroll
    for (int r = 0; r < RB; ++r)
#pragma unroll
        for (int b = 0; b < NB; ++b) acc[r][b] = 0.f;
    const float *rows[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) rows[r] = R + (size_t)(m0 + r < nrows ? m0 + r : m0) * ldr;
    for (int k = 2 * threadIdx.x; k < ncols; k += 2 * blockDim.x) {
        const bool pair = k + 1 < ncols;
        float2 sv[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            sv[b] = make_float2(0.f, 0.f);
            if (b < nb) {
                const float *sp = S + (size_t)b * lds + k;
                if (vec2 && pair) sv[b] = __ldg(reinterpret_cast<const float2 *>(sp));
                else sv[b] = make_float2(__ldg(sp), pair ? __ldg(sp + 1) : 0.f);
            }
        }
#pragma unroll
        for (int r = 0; r < RB; ++r) {
            if (m0 + r >= nrows) break;
            float2 rv;
            if (vec2 && pair) rv = __ldg(reinterpret_cast<const float2 *>(rows[r] + k));
            else rv = make_float2(__ldg(rows[r] + k), pair ? __ldg(rows[r] + k + 1) : 0.f);
#pragma unroll
            for (int b = 0; b < NB; ++b) acc[r][b] = fmaf(rv.y, sv[b].y, fmaf(rv.x, sv[b].x, acc[r][b]));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < RB; ++r)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const float v = sb::warp_sum(acc[r][b]);
            if (lane == 0) red[r * NB + b][warp] = v;
        }
    __syncthreads();
    for (int e = threadIdx.x; e < RB * NB; e += blockDim.x) {
        const int r = e / NB, b = e - r * NB;
        if (m0 + r < nrows && b < nb) {
            float t = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[e][w];
            epi(m0 + r, b, t);
        }
    }
}

template <int NB, int RB>
__global__ void __launch_bounds__(256) gemv_rows_batched_kernel(const float *__restrict__ R, int nrows, int ncols,
                                                                int ldr, const float *__restrict__ S, int lds,
                                                                int nb, float *__restrict__ M, int ldm, int vec2) {
    gemv_rows_batched_body<NB, RB>(R, nrows, ncols, ldr, S, lds, nb, vec2, blockIdx.x * RB,
                                   [&](int m, int b, float t) { M[(size_t)b * ldm + m] = t; });
}

}  // namespace

// ---------------------------------------------------------------------------
// Monte-Carlo step, stages 6-7.  Realisations go in chunks of up to 16
// (a job): the reconstructor launch gives every job ceil(n_modes / 2) CTAs of
// gemv_rows_batched_body followed by the group's integrator update of each
// finished mode; the mirror launch shares the SMs among the jobs so that the
// busiest CTA streams the fewest influence-function rows, each CTA running
// the register-blocked TMA projection (4 boxes per stage) over its job's
// tiles.  The sums are those of sb_modalrec_batched, sb_integrator and
// sb_dm_project_batched with one mode-row group.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMcRecRows = 2;          // reconstructor rows per CTA
constexpr int kMcChunk = 16;           // realisations per job
constexpr int kMcDmNbx = 4;            // boxes per mirror stage
// ring stages of the mirror launch (measured on the 96-realisation mix,
// pipelined step: 3 stages 0.977, 4 0.967, 5 0.963 ms)
constexpr int kMcDmStages = 5;

struct McRecJob {
    const float *R, *S;
    float *M;
    int nrows, ncols, ldr, lds, ldm, nb, vec2, g, e0;
};

struct McRecArgs {
    const McRecJob *jobs;
    const int2 *blk;                   // per CTA: job, row block
    sb_iir_plan iir[sb::kMcMaxGroups];
    float *out[sb::kMcMaxGroups];
};

struct McDmJob {
    const float *cmd[2];               // commands, commands_next
    const int32_t *idx;
    float *phase[2];                   // dm_phase, dm_phase_alt
    long long phase_stride;
    int ldc, nb, nmodes, nvalid, g, cta0, ncta;
    float sign;
};

struct McDmArgs {
    CUtensorMap map[sb::kMcMaxGroups];
    const McDmJob *jobs;
    const int *cta_job;
    int cmd, sel;                      // command and phase buffers of this launch
};

struct McRecBlob {
    McRecArgs args;
    int blocks;
};

struct McDmBlob {
    McDmArgs args;
    int blocks, pipelined;
    size_t smem;
};

// realisations b0 .. b0 + nb - 1 of job J (nb <= NB)
template <int NB>
__device__ __forceinline__ void mc_rec_job(const McRecJob &J, int b0, int nb, int m0, const sb_iir_plan &p,
                                           float *out) {
    gemv_rows_batched_body<NB, kMcRecRows>(J.R, J.nrows, J.ncols, J.ldr, J.S + (size_t)b0 * J.lds, J.lds, nb,
                                           J.vec2, m0, [&](int m, int b, float t) {
                                               J.M[(size_t)(b0 + b) * J.ldm + m] = t;
                                               iir_update(p, J.e0 + (b0 + b) * J.nrows + m, t, out);
                                           });
}

// a job of more than 8 realisations in two passes of 8 over the reconstructor
// rows (the sums of each (row, realisation) do not depend on the pass)
__global__ void __launch_bounds__(256) mc_rec_kernel(McRecArgs m) {
    const int2 jb = m.blk[blockIdx.x];
    const McRecJob &J = m.jobs[jb.x];
    const int m0 = jb.y * kMcRecRows;
    const sb_iir_plan &p = m.iir[J.g];
    float *out = m.out[J.g];
    const int nb = J.nb;
    if (nb <= 4) {
        mc_rec_job<4>(J, 0, nb, m0, p, out);
        return;
    }
    mc_rec_job<8>(J, 0, nb < 8 ? nb : 8, m0, p, out);
    if (nb > 8) {
        __syncthreads();                  // the reduction buffer is reused
        mc_rec_job<8>(J, 8, nb - 8, m0, p, out);
    }
}

__global__ void __launch_bounds__(32 * (2 * kMcDmNbx + 1), 1) mc_dm_kernel(const __grid_constant__ McDmArgs m) {
    const McDmJob &J = m.jobs[m.cta_job[blockIdx.x]];
    const int bid = blockIdx.x - J.cta0;
    if (J.nb <= 8)
        dm_c4_body<8, kMcDmNbx, kMcDmStages>(m.map[J.g], J.nmodes, J.nvalid, J.cmd[m.cmd], J.ldc, J.nb, J.sign,
                                             J.idx, J.phase[m.sel], J.phase_stride, bid, J.ncta);
    else
        dm_c4_body<16, kMcDmNbx, kMcDmStages>(m.map[J.g], J.nmodes, J.nvalid, J.cmd[m.cmd], J.ldc, J.nb, J.sign,
                                              J.idx, J.phase[m.sel], J.phase_stride, bid, J.ncta);
}

int mc_jobs(const sb_mc_group *gs, int n) {
    int j = 0;
    for (int g = 0; g < n; ++g) j += (gs[g].n_batch + kMcChunk - 1) / kMcChunk;
    return j;
}

int mc_rec_blocks(const sb_mc_group *gs, int n) {
    int b = 0;
    for (int g = 0; g < n; ++g)
        b += ((gs[g].n_batch + kMcChunk - 1) / kMcChunk) * ((gs[g].n_modes + kMcRecRows - 1) / kMcRecRows);
    return b;
}

}  // namespace

namespace sb {

size_t mc_control_workspace(const sb_mc_group *gs, int n) {
    const size_t nj = mc_jobs(gs, n);
    return mc_align(nj * sizeof(McRecJob)) + mc_align((size_t)mc_rec_blocks(gs, n) * sizeof(int2)) +
           mc_align(nj * sizeof(McDmJob)) + mc_align((size_t)sm_count() * sizeof(int));
}

int mc_control_prepare(const sb_mc_group *gs, int n, void *ws, McBlob &rec, McBlob &dm, cudaStream_t st) {
    static_assert(sizeof(McRecBlob) <= sizeof(McBlob) && sizeof(McDmBlob) <= sizeof(McBlob),
                  "control stage arguments exceed the blob");
    static_assert(sizeof(McRecArgs) <= 4096 && sizeof(McDmArgs) <= 4096, "kernel arguments above 4 KB");
    const char *who = "sb_mc_create";
    McRecBlob *RB = new (rec.b) McRecBlob();
    McDmBlob *DB = new (dm.b) McDmBlob();
    const int nj = mc_jobs(gs, n), nblk_rec = mc_rec_blocks(gs, n), nsm = sm_count();
    if (nj > nsm) return fail(SB_ESHAPE, "%s: %d realisation chunks for %d SMs", who, nj, nsm);
    std::vector<McRecJob> rj(nj);
    std::vector<int2> rb(nblk_rec);
    std::vector<McDmJob> dj(nj);
    std::vector<int> tiles(nj), ncta(nj, 1);
    unsigned char *w = static_cast<unsigned char *>(ws);
    McRecJob *d_rj = reinterpret_cast<McRecJob *>(w);
    w += mc_align(nj * sizeof(McRecJob));
    int2 *d_rb = reinterpret_cast<int2 *>(w);
    w += mc_align((size_t)nblk_rec * sizeof(int2));
    McDmJob *d_dj = reinterpret_cast<McDmJob *>(w);
    w += mc_align(nj * sizeof(McDmJob));
    int *d_cta = reinterpret_cast<int *>(w);
    constexpr int TW = kDmCols * kMcDmNbx;
    int j = 0, blk = 0;
    size_t smem = 0;
    for (int g = 0; g < n; ++g) {
        const sb_mc_group &G = gs[g];
        const int nm = G.n_modes;
        if (!G.R || !G.modes || !G.commands || !G.ifunc || !G.mask_idx || nm < 1 || G.n_slopes < 1 ||
            G.ldr < G.n_slopes || G.n_slopes > G.slopes_stride || G.iir.n != G.n_batch * nm)
            return fail(SB_EINVAL, "%s: group %d: bad reconstructor / integrator", who, g);
        if (nm > kDbMaxModes) return fail(SB_ESHAPE, "%s: group %d: at most %d modes", who, g, kDbMaxModes);
        if (G.commands_next && G.iir.out_next != G.commands_next)
            return fail(SB_EINVAL, "%s: group %d: iir.out_next must be commands_next", who, g);
        if (!G.commands_next != !G.dm_phase_alt)
            return fail(SB_EINVAL, "%s: group %d: dm_phase_alt and commands_next go together", who, g);
        if (G.n_valid < 1 || G.ld_if < G.n_valid || G.ld_if % 4 || (uintptr_t)G.ifunc % 16)
            return fail(SB_EINVAL, "%s: group %d: influence functions need 16-byte aligned rows", who, g);
        RB->args.iir[g] = G.iir;
        RB->args.out[g] = G.commands;
        int rc = tensor_map_2d_f32(&DB->args.map[g], G.ifunc, nm, G.ld_if, G.ld_if, kDmRows / kMcDmNbx, kDmCols);
        if (rc) return rc;
        const int vec2 = (G.ldr % 2 == 0) && (G.slopes_stride % 2 == 0) && ((uintptr_t)G.R % 8 == 0) &&
                         ((uintptr_t)G.slopes % 8 == 0);
        for (int b0 = 0; b0 < G.n_batch; b0 += kMcChunk, ++j) {
            const int nb = G.n_batch - b0 < kMcChunk ? G.n_batch - b0 : kMcChunk;
            McRecJob &r = rj[j];
            r.R = G.R;
            r.S = G.slopes + (size_t)b0 * G.slopes_stride;
            r.M = G.modes + (size_t)b0 * nm;
            r.nrows = nm;
            r.ncols = G.n_slopes;
            r.ldr = G.ldr;
            r.lds = G.slopes_stride;
            r.ldm = nm;
            r.nb = nb;
            r.vec2 = vec2;
            r.g = g;
            r.e0 = b0 * nm;
            for (int k = 0; k < (nm + kMcRecRows - 1) / kMcRecRows; ++k) rb[blk++] = make_int2(j, k);
            McDmJob &d = dj[j];
            d.cmd[0] = G.commands + (size_t)b0 * nm;
            d.cmd[1] = G.commands_next ? G.commands_next + (size_t)b0 * nm : nullptr;
            d.idx = G.mask_idx;
            d.phase[0] = G.dm_phase + (size_t)b0 * G.dm_stride;
            d.phase[1] = G.dm_phase_alt ? G.dm_phase_alt + (size_t)b0 * G.dm_stride : nullptr;
            d.phase_stride = G.dm_stride;
            d.ldc = nm;
            d.nb = nb;
            d.nmodes = nm;
            d.nvalid = G.n_valid;
            d.g = g;
            d.sign = G.dm_sign;
            tiles[j] = (G.n_valid + TW - 1) / TW;
            const size_t sm = nb <= 8 ? dm_c4_smem_bytes<kMcDmNbx, kMcDmStages>(nm, 8)
                                      : dm_c4_smem_bytes<kMcDmNbx, kMcDmStages>(nm, 16);
            smem = sm > smem ? sm : smem;
        }
    }
    // SMs to jobs: each added CTA goes to the job whose busiest CTA has the
    // most work: tiles per CTA x modes, x 7/4 for 16 realisations per pass
    // (twice the FMAs per influence-function value: a CTA streams ~1.75x
    // slower than with 8)
    for (int left = nsm - nj; left > 0; --left) {
        int best = -1;
        long long worst = 0;
        for (int k = 0; k < nj; ++k) {
            if (ncta[k] >= tiles[k]) continue;
            const long long c =
                (long long)((tiles[k] + ncta[k] - 1) / ncta[k]) * dj[k].nmodes * (dj[k].nb > 8 ? 7 : 4);
            if (c > worst) {
                worst = c;
                best = k;
            }
        }
        if (best < 0) break;
        ++ncta[best];
    }
    std::vector<int> cta_job;
    for (int k = 0; k < nj; ++k) {
        dj[k].cta0 = (int)cta_job.size();
        dj[k].ncta = ncta[k];
        for (int c = 0; c < ncta[k]; ++c) cta_job.push_back(k);
    }
    RB->args.jobs = d_rj;
    RB->args.blk = d_rb;
    RB->blocks = nblk_rec;
    DB->args.jobs = d_dj;
    DB->args.cta_job = d_cta;
    DB->blocks = (int)cta_job.size();
    DB->pipelined = 1;
    for (int g = 0; g < n; ++g) DB->pipelined &= gs[g].commands_next != nullptr;
    DB->smem = smem;
    cudaError_t e = cudaMemcpyAsync(d_rj, rj.data(), nj * sizeof(McRecJob), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rb, rb.data(), nblk_rec * sizeof(int2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dj, dj.data(), nj * sizeof(McDmJob), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_cta, cta_job.data(), cta_job.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mc_dm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail(SB_ECUDA, "%s: control tables: %s", who, cudaGetErrorString(e));
    return SB_OK;
}

int mc_rec_launch(const McBlob &blob, cudaStream_t st) {
    const McRecBlob *B = reinterpret_cast<const McRecBlob *>(blob.b);
    mc_rec_kernel<<<B->blocks, 256, 0, st>>>(B->args);
    return check_launch("mc_rec_kernel");
}

int mc_dm_launch(const McBlob &blob, int cmd, int sel, cudaStream_t st) {
    const McDmBlob *B = reinterpret_cast<const McDmBlob *>(blob.b);
    if ((cmd || sel) && !B->pipelined)
        return fail(SB_EINVAL, "sb_mc_stage: the groups have no commands_next / dm_phase_alt");
    McDmArgs a = B->args;
    a.cmd = cmd;
    a.sel = sel;
    mc_dm_kernel<<<B->blocks, 32 * (2 * kMcDmNbx + 1), B->smem, st>>>(a);
    return check_launch("mc_dm_kernel");
}

}  // namespace sb

extern "C" int sb_device_status(void) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_dm_status, sizeof(int)) != cudaSuccess)
        return sb::fail(SB_ECUDA, "sb_device_status: %s", cudaGetErrorString(cudaGetLastError()));
    const int sh = sb::sh_tc_status_take();
    if (sh < 0) return sb::fail(SB_ECUDA, "sb_device_status: %s", cudaGetErrorString(cudaGetLastError()));
    const int ct = sb::contract_status_take();
    if (ct < 0) return sb::fail(SB_ECUDA, "sb_device_status: %s", cudaGetErrorString(cudaGetLastError()));
    const int pt = sb::psf_tc_status_take();
    if (pt < 0) return sb::fail(SB_ECUDA, "sb_device_status: %s", cudaGetErrorString(cudaGetLastError()));
    if (v == 0 && sh == 0 && ct == 0 && pt == 0) return SB_OK;
    if (v == 0 && sh == 0 && ct == 0)
        return sb::fail(SB_ETIMEOUT, "a tensor-core PSF wait timed out (%s)",
                        pt == 1 ? "copy ring" : (pt == 2 ? "MMA issue" : "epilogue"));
    if (v == 0 && sh == 0)
        return ct == 3 ? sb::fail(SB_EINVAL, "sb_intmat_contract_rows: a row segment does not cover its columns or "
                                             "is not 16-byte aligned (those rows were not contracted)")
                       : sb::fail(SB_ETIMEOUT, "an interaction-matrix contraction wait timed out (%s side)",
                                  ct == 1 ? "producer" : "consumer");
    if (v == 0)
        return sh == 9 ? sb::fail(SB_ETIMEOUT, "an SH field-tile (TMA) wait timed out")
                       : sb::fail(SB_ETIMEOUT, "a tensor-core SH wait timed out (stage %d)", sh);
    const int zero = 0;
    cudaMemcpyToSymbol(g_dm_status, &zero, sizeof(int));
    return sb::fail(SB_ETIMEOUT, "a DM projection wait timed out (%s side)", v == 1 ? "producer" : "consumer");
}

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

namespace {
// copy of the plan with the tap counts filled in (0 means the 2-tap integrator)
int iir_taps_checked(const sb_iir_plan *p, sb_iir_plan *q, const char *who) {
    *q = *p;
    if (q->n_num == 0) q->n_num = 2;
    if (q->n_den == 0) q->n_den = 2;
    if (q->n_num < 1 || q->n_num > kIirMaxTaps || q->n_den < 1 || q->n_den > kIirMaxTaps)
        return sb::fail(SB_EINVAL, "%s: filters of 1 to %d taps", who, kIirMaxTaps);
    return SB_OK;
}
}  // namespace

extern "C" int sb_modalrec_integrator(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes,
                                      float *modes, const sb_iir_plan *plan, float *out, void *stream) {
    sb::clear_error();
    if (!R || !slopes || !modes || !plan || !out || n_modes < 0 || n_slopes < 0 || ldr < n_slopes)
        return sb::fail(SB_EINVAL, "sb_modalrec_integrator: bad args");
    sb_iir_plan q;
    const int trc = iir_taps_checked(plan, &q, "sb_modalrec_integrator");
    if (trc) return trc;
    const sb_iir_plan *p = &q;
    if (!p->num || !p->den || !p->ist || !p->ost || !p->state)
        return sb::fail(SB_EINVAL, "sb_modalrec_integrator: null integrator state");
    if (p->n != n_modes) return sb::fail(SB_ESHAPE, "sb_modalrec_integrator: %d filters for %d modes", p->n, n_modes);
    if (p->total < 1 || p->total > 8 || p->k_out < 0 || p->k_out >= p->total || (p->rem != 0.f && p->k_out < 1))
        return sb::fail(SB_EINVAL, "sb_modalrec_integrator: bad state layout (delay up to 7 frames)");
    if (p->out_next && (p->rem != 0.f || p->k_out < 1))
        return sb::fail(SB_EINVAL, "sb_modalrec_integrator: out_next needs an integer delay >= 1");
    if (n_modes == 0) return SB_OK;
    cudaStream_t st = sb::as_stream(stream);
    const bool vec = (ldr % 4 == 0) && ((uintptr_t)R % 16 == 0) && ((uintptr_t)slopes % 16 == 0);
    if (vec)
        gemv_iir_kernel<true><<<n_modes, 256, 0, st>>>(R, n_slopes, ldr, slopes, modes, *p, out);
    else
        gemv_iir_kernel<false><<<n_modes, 256, 0, st>>>(R, n_slopes, ldr, slopes, modes, *p, out);
    return sb::check_launch("gemv_iir_kernel");
}

extern "C" int sb_integrator(const sb_iir_plan *plan, const float *delta, float *out, void *stream) {
    sb::clear_error();
    if (!plan || !delta || !out || !plan->num || !plan->den || !plan->ist || !plan->ost || !plan->state)
        return sb::fail(SB_EINVAL, "sb_integrator: null pointer");
    sb_iir_plan q;
    const int trc = iir_taps_checked(plan, &q, "sb_integrator");
    if (trc) return trc;
    const sb_iir_plan *p = &q;
    if (p->n < 0 || p->total < 1 || p->total > 8 || p->k_out < 0 || p->k_out >= p->total ||
        (p->rem != 0.f && p->k_out < 1))
        return sb::fail(SB_EINVAL, "sb_integrator: bad state layout (delay up to 7 frames)");
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
    if (vec && n_modes <= kDmMaxModes) {
        CUtensorMap map;
        const int nsm = sb::sm_count();
        if (nsm > 0 && sb::tensor_map_2d_f32(&map, ifunc, n_modes, ld_if, ld_if, kDmRows, kDmCols) == SB_OK) {
            const size_t smem = dm_tma_smem_bytes(n_modes);
            static bool attr_set[64] = {false};
            int dev = 0;
            cudaGetDevice(&dev);
            if (dev >= 0 && dev < 64 && !attr_set[dev]) {
                const size_t max_smem = dm_tma_smem_bytes(kDmMaxModes);
                if (cudaFuncSetAttribute(dm_project_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)max_smem) != cudaSuccess)
                    return sb::fail(SB_ECUDA, "sb_dm_project: %s", cudaGetErrorString(cudaGetLastError()));
                attr_set[dev] = true;
            }
            const int ntiles = (n_valid + kDmCols - 1) / kDmCols;
            dm_project_tma_kernel<<<ntiles < nsm ? ntiles : nsm, 32 * (kDmConsumerWarps + 1), smem, st>>>(
                map, n_modes, n_valid, cmd, n_cmd, sign, mask_idx, phase);
            return sb::check_launch("dm_project_tma_kernel");
        }
        sb::clear_error();    // no tensor map: the load/store kernel below
    }
    const int W = vec ? 4 : 1;
    const size_t smem = (size_t)(n_modes + 8 * 32 * W) * sizeof(float);
    if (smem > 200 * 1024) return sb::fail(SB_ESHAPE, "sb_dm_project: too many modes (%d)", n_modes);
    const int nblk = (n_valid + 32 * W - 1) / (32 * W);
    if (vec) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(dm_project_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dm_project_kernel<4><<<nblk, 256, smem, st>>>(ifunc, n_modes, n_valid, ld_if, cmd, n_cmd, sign, mask_idx, phase);
    } else {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(dm_project_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dm_project_kernel<1><<<nblk, 256, smem, st>>>(ifunc, n_modes, n_valid, ld_if, cmd, n_cmd, sign, mask_idx, phase);
    }
    return sb::check_launch("dm_project_kernel");
}

namespace {

template <int NB, int RS>
int launch_dm_batched(const CUtensorMap &map, int n_modes, int n_valid, const float *cmd, int ldc, int nb, float sign,
                      const int32_t *mask_idx, float *phase, long long phase_stride, cudaStream_t st) {
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = dm_batched_smem_bytes<NB>(n_modes);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        if (cudaFuncSetAttribute(dm_project_batched_kernel<NB, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dm_batched_smem_bytes<NB>(kDbMaxModes)) != cudaSuccess)
            return sb::fail(SB_ECUDA, "sb_dm_project_batched: %s", cudaGetErrorString(cudaGetLastError()));
        attr_set[dev] = true;
    }
    const int nsm = sb::sm_count();
    const int ntiles = (n_valid + kDmCols - 1) / kDmCols;
    dm_project_batched_kernel<NB, RS><<<ntiles < nsm ? ntiles : nsm, 32 * (kDbWarps * RS + 1), smem, st>>>(
        map, n_modes, n_valid, cmd, ldc, nb, sign, mask_idx, phase, phase_stride);
    return sb::check_launch("dm_project_batched_kernel");
}

template <int NB, int NBX>
int launch_dm_c4(const CUtensorMap &map, int n_modes, int n_valid, const float *cmd, int ldc, int nb, float sign,
                 const int32_t *mask_idx, float *phase, long long phase_stride, cudaStream_t st) {
    static bool attr_set[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        if (cudaFuncSetAttribute(dm_project_batched_c4_kernel<NB, NBX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dm_c4_smem_bytes<NBX>(kDbMaxModes, NB)) != cudaSuccess)
            return sb::fail(SB_ECUDA, "sb_dm_project_batched: %s", cudaGetErrorString(cudaGetLastError()));
        attr_set[dev] = true;
    }
    const int nsm = sb::sm_count();
    const int ntiles = (n_valid + kDmCols * NBX - 1) / (kDmCols * NBX);
    dm_project_batched_c4_kernel<NB, NBX><<<ntiles < nsm ? ntiles : nsm, 32 * (2 * NBX + 1),
                                            dm_c4_smem_bytes<NBX>(n_modes, NB), st>>>(
        map, n_modes, n_valid, cmd, ldc, nb, sign, mask_idx, phase, phase_stride);
    return sb::check_launch("dm_project_batched_c4_kernel");
}

template <int NBX>
int launch_dm_c4_nb(const CUtensorMap &map, int n_modes, int n_valid, const float *c, int ldc, int nb, float sign,
                    const int32_t *mask_idx, float *ph, long long phase_stride, cudaStream_t st) {
    if (nb <= 4) return launch_dm_c4<4, NBX>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
    if (nb <= 8) return launch_dm_c4<8, NBX>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
    return launch_dm_c4<16, NBX>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
}

template <int NB, int RB>
int launch_gemv_batched_rb(const float *R, int nrows, int ncols, int ldr, const float *S, int lds, int nb, float *M,
                           int ldm, int vec2, cudaStream_t st) {
    gemv_rows_batched_kernel<NB, RB><<<(nrows + RB - 1) / RB, 256, 0, st>>>(R, nrows, ncols, ldr, S, lds, nb, M, ldm,
                                                                           vec2);
    return sb::check_launch("gemv_rows_batched_kernel");
}

template <int NB>
int launch_gemv_batched(int rb, const float *R, int nrows, int ncols, int ldr, const float *S, int lds, int nb,
                        float *M, int ldm, int vec2, cudaStream_t st) {
    if (rb == 4) return launch_gemv_batched_rb<NB, 4>(R, nrows, ncols, ldr, S, lds, nb, M, ldm, vec2, st);
    if (rb == 1) return launch_gemv_batched_rb<NB, 1>(R, nrows, ncols, ldr, S, lds, nb, M, ldm, vec2, st);
    return launch_gemv_batched_rb<NB, 2>(R, nrows, ncols, ldr, S, lds, nb, M, ldm, vec2, st);
}

template <int RS>
int launch_dm_batched_rs(const CUtensorMap &map, int n_modes, int n_valid, const float *c, int ldc, int nb,
                         float sign, const int32_t *mask_idx, float *ph, long long phase_stride, cudaStream_t st) {
    if (nb <= 4) return launch_dm_batched<4, RS>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
    if (nb <= 8) return launch_dm_batched<8, RS>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
    return launch_dm_batched<16, RS>(map, n_modes, n_valid, c, ldc, nb, sign, mask_idx, ph, phase_stride, st);
}

}  // namespace

extern "C" int sb_dm_project_batched(const float *ifunc, int n_modes, int n_valid, int ld_if, const float *cmd,
                                     int ld_cmd, int n_batch, float sign, const int32_t *mask_idx, float *phase,
                                     long long phase_stride, void *stream) {
    sb::clear_error();
    if (!ifunc || !cmd || !mask_idx || !phase || n_modes < 1 || n_valid < 0 || ld_if < n_valid || n_batch < 1 ||
        ld_cmd < n_modes || phase_stride < 1)
        return sb::fail(SB_EINVAL, "sb_dm_project_batched: bad args");
    if (n_modes > kDbMaxModes)
        return sb::fail(SB_ESHAPE, "sb_dm_project_batched: at most %d modes", kDbMaxModes);
    if (ld_if % 4 || (uintptr_t)ifunc % 16)
        return sb::fail(SB_EINVAL, "sb_dm_project_batched: influence-function rows must be 16-byte aligned");
    if (n_valid == 0) return SB_OK;
    cudaStream_t st = sb::as_stream(stream);
    // tile variant: realisations per pass (every pass re-reads the IF once) and mode-row groups
    // (0-5), or the register-blocked form with 4, 2 or 1 boxes per stage and 8 (6-8) or 16 (9-11)
    // realisations per pass
    const int v = sb::tune_lookup(SB_TUNE_DM_BATCHED, sb_tune_key(n_modes, n_valid, n_batch));
    CUtensorMap map;
    if (v >= 6) {
        const int w = (v - 6) % 3, pass = v < 9 ? 8 : 16;
        const int nbx = w == 0 ? 4 : (w == 1 ? 2 : 1);
        int rc = sb::tensor_map_2d_f32(&map, ifunc, n_modes, ld_if, ld_if, kDmRows / nbx, kDmCols);
        if (rc) return rc;
        for (int b0 = 0; b0 < n_batch; b0 += pass) {
            const int nb = n_batch - b0 < pass ? n_batch - b0 : pass;
            const float *c = cmd + (size_t)b0 * ld_cmd;
            float *ph = phase + (size_t)b0 * phase_stride;
            rc = nbx == 4 ? launch_dm_c4_nb<4>(map, n_modes, n_valid, c, ld_cmd, nb, sign, mask_idx, ph, phase_stride, st)
               : nbx == 2 ? launch_dm_c4_nb<2>(map, n_modes, n_valid, c, ld_cmd, nb, sign, mask_idx, ph, phase_stride, st)
                          : launch_dm_c4_nb<1>(map, n_modes, n_valid, c, ld_cmd, nb, sign, mask_idx, ph, phase_stride, st);
            if (rc) return rc;
        }
        return SB_OK;
    }
    int rc = sb::tensor_map_2d_f32(&map, ifunc, n_modes, ld_if, ld_if, kDmRows, kDmCols);
    if (rc) return rc;
    const int pass = v < 2 ? 16 : (v < 4 ? 8 : 4);
    const bool rs2 = (v & 1) != 0;
    for (int b0 = 0; b0 < n_batch; b0 += pass) {
        const int nb = n_batch - b0 < pass ? n_batch - b0 : pass;
        const float *c = cmd + (size_t)b0 * ld_cmd;
        float *ph = phase + (size_t)b0 * phase_stride;
        rc = rs2 ? launch_dm_batched_rs<2>(map, n_modes, n_valid, c, ld_cmd, nb, sign, mask_idx, ph, phase_stride, st)
                 : launch_dm_batched_rs<1>(map, n_modes, n_valid, c, ld_cmd, nb, sign, mask_idx, ph, phase_stride, st);
        if (rc) return rc;
    }
    return SB_OK;
}

extern "C" int sb_modalrec_batched(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes, int lds,
                                   int n_batch, float *modes, int ldm, void *stream) {
    sb::clear_error();
    if (!R || !slopes || !modes || n_modes < 0 || n_slopes < 0 || ldr < n_slopes || n_batch < 1 ||
        lds < n_slopes || ldm < n_modes)
        return sb::fail(SB_EINVAL, "sb_modalrec_batched: bad args");
    if (n_modes == 0) return SB_OK;
    cudaStream_t st = sb::as_stream(stream);
    const int vec2 = (ldr % 2 == 0) && (lds % 2 == 0) && ((uintptr_t)R % 8 == 0) && ((uintptr_t)slopes % 8 == 0);
    // rows per CTA: the SB_TUNE_MODALREC_BATCHED variant (2, 1, 4)
    const int v = sb::tune_lookup(SB_TUNE_MODALREC_BATCHED, sb_tune_key(n_modes, n_slopes, n_batch));
    const int rb = v == 1 ? 1 : (v == 2 ? 4 : 2);
    for (int b0 = 0; b0 < n_batch; b0 += 16) {
        const int nb = n_batch - b0 < 16 ? n_batch - b0 : 16;
        const float *S = slopes + (size_t)b0 * lds;
        float *M = modes + (size_t)b0 * ldm;
        int rc;
        if (nb <= 4) rc = launch_gemv_batched<4>(rb, R, n_modes, n_slopes, ldr, S, lds, nb, M, ldm, vec2, st);
        else if (nb <= 8) rc = launch_gemv_batched<8>(rb, R, n_modes, n_slopes, ldr, S, lds, nb, M, ldm, vec2, st);
        else rc = launch_gemv_batched<16>(rb, R, n_modes, n_slopes, ldr, S, lds, nb, M, ldm, vec2, st);
        if (rc) return rc;
    }
    return SB_OK;
}
