// Shack-Hartmann forward model on the B200.
//
// One warp owns one sub-aperture; a CTA holds the sub-apertures of one chunk
// of a lenslet row.  Per sub-aperture (all in shared memory):
//   E[r][c]  = A * exp(i * k * phase) * tilt          (np x np, complex)
//   G[r][b]  = sum_c E[r][c] * W[b][c]                 (np x cutsize)
//   F[a][b]  = sum_r W[a][r] * G[r][b]                 (cutsize x cutsize)
//   I[a][b]  = |F|^2 * field_stop[a][b]
//   D[p][q]  = sum_ab R[p][a] R[q][b] I[a][b]           (subap_npx^2, LCM rebin)
// W holds only the DFT rows that survive the fftshift + FoV cut, so the
// zero-padded FFT of the reference (sh.py:376-405) is evaluated on exactly
// the samples that reach the detector.  Row/column sums of D and of the
// input amplitude go to per-CTA partials; a second kernel turns them into
// the photon normalisation of sh.py:425-427 in a fixed (deterministic) order.
#include <new>

#include "sb_common.cuh"
#include "sb_dft.cuh"
#include "sb_mc.cuh"
#include "sb_umma.cuh"

namespace {

struct ShArgs {
    int n, p, cs, npx, ld, spc;
    float k;
    const float2 *tw;
    const float2 *tilt;
    const float *mask;
    const float *rebin;
    const float *A;
    const float *ph;
    const float *A_norm;
    int n_norm;
    float *out;
    float *part_I;
    float *part_A;
    // batched launches: blockIdx.z selects the realisation (strides in
    // elements; 0 and gridDim.z = 1 for a single field)
    long long sA, sph, sAn, sout;
    int nbp;                       // partial sums per realisation
    int vec;                       // field rows may be read as float4 (16-byte aligned rows and strides)
    // the mirror term of the on-axis propagation applied while the field is
    // read (single field, FP32 forms): amplitude A * A2, phase ph + ph2, the
    // normalising amplitude A_norm * A2; the resulting field is written to
    // A_out / P_out when they are given.  NULL A2: the field is A, ph.
    const float *A2, *ph2;
    float *A_out, *P_out;
    // a band of lenslet rows (sb_sh_forward_rows): grid row y is lenslet row
    // row0 + y, and the partial sums are indexed as in the whole grid of
    // grid_rows rows (0: the launch grid itself)
    int row0, grid_rows;
};

// amplitude and phase (nm) of field element g, with the mirror term when present
__device__ __forceinline__ void field_at(const ShArgs &a, size_t g, float &amp, float &phn) {
    amp = a.A[g];
    phn = a.ph[g];
    if (a.A2) {
        amp = __fmul_rn(amp, a.A2[g]);      // the order of the on-axis propagation: layers, stop, mirror
        phn = __fadd_rn(phn, a.ph2[g]);
        if (a.A_out) {
            a.A_out[g] = amp;
            a.P_out[g] = phn;
        }
    }
}

__device__ __forceinline__ float norm_amp(const ShArgs &a, int e) {
    return a.A2 ? __fmul_rn(a.A_norm[e], a.A2[e]) : a.A_norm[e];
}

// realisation z's slice of a batched launch
__device__ __forceinline__ void slice_to(ShArgs &a, long long z) {
    a.A += z * a.sA;
    a.ph += z * a.sph;
    a.A_norm += z * a.sAn;
    a.out += z * a.sout;
    a.part_I += z * a.nbp;
    a.part_A += z * a.nbp;
}

__device__ __forceinline__ void batch_slice(ShArgs &a) { slice_to(a, blockIdx.z); }

struct ShSmem {
    int tw, tilt, mask, rebin, per_warp_E, per_warp_G, per_warp_I, per_warp_H, tables, per_warp;
};

// Shared-memory layout.  The twiddles are stored transposed, twT[c][b], so
// the lanes of a warp (consecutive output frequencies b) read consecutive
// words; the field rows are padded to np+1 to keep rows in distinct banks.
__host__ __device__ inline ShSmem sh_smem_layout(int p, int cs, int npx) {
    ShSmem s;
    s.tw = 0;
    s.tilt = s.tw + cs * p * 8;
    s.mask = s.tilt + p * p * 8;
    s.rebin = s.mask + cs * cs * 4;
    s.tables = ((s.rebin + npx * cs * 4) + 15) & ~15;
    s.per_warp_E = 0;
    s.per_warp_G = s.per_warp_E + p * (p + 1) * 8;
    s.per_warp_I = s.per_warp_G + p * cs * 8;
    s.per_warp_H = s.per_warp_I + cs * cs * 4;
    s.per_warp = ((s.per_warp_H + cs * npx * 4) + 15) & ~15;
    return s;
}

constexpr int kU = 4;   // independent accumulators per lane

__global__ void __launch_bounds__(256, 4) sh_forward_kernel(ShArgs a) {
    batch_slice(a);
    extern __shared__ __align__(16) unsigned char smem[];
    const ShSmem L = sh_smem_layout(a.p, a.cs, a.npx);
    float2 *twT = reinterpret_cast<float2 *>(smem + L.tw);
    float2 *tilt = reinterpret_cast<float2 *>(smem + L.tilt);
    float *mask = reinterpret_cast<float *>(smem + L.mask);
    float *R = reinterpret_cast<float *>(smem + L.rebin);
    __shared__ float red[33];

    const int p = a.p, cs = a.cs, npx = a.npx;
    for (int e = threadIdx.x; e < cs * p; e += blockDim.x) {
        const int b = e / p, c = e - b * p;
        twT[c * cs + b] = a.tw[e];
    }
    for (int e = threadIdx.x; e < p * p; e += blockDim.x) tilt[e] = a.tilt[e];
    for (int e = threadIdx.x; e < cs * cs; e += blockDim.x) mask[e] = a.mask[e];
    for (int e = threadIdx.x; e < npx * cs; e += blockDim.x) R[e] = a.rebin[e];
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.y;                       // lenslet row
    const int j = blockIdx.x * a.spc + warp;        // lenslet column
    unsigned char *wbase = smem + L.tables + warp * L.per_warp;
    float2 *E = reinterpret_cast<float2 *>(wbase + L.per_warp_E);   // [p][p+1]
    float2 *G = reinterpret_cast<float2 *>(wbase + L.per_warp_G);   // [p][cs]
    float *I = reinterpret_cast<float *>(wbase + L.per_warp_I);     // [cs][cs]
    float *H = reinterpret_cast<float *>(wbase + L.per_warp_H);     // [cs][npx]
    const int pe = p + 1;

    float local = 0.f;
    if (j < a.n) {
        // field build (electric_field.py:60-75 and sh.py:376)
        const size_t row0 = (size_t)i * p;
        const size_t col0 = (size_t)j * p;
        for (int e = lane; e < p * p; e += 32) {
            const int r = e / p, c = e - r * p;
            const size_t g = (row0 + r) * (size_t)a.ld + col0 + c;
            float amp, phn;
            field_at(a, g, amp, phn);
            const float phi = phn * a.k;
            float sn, co;
            sincosf(phi, &sn, &co);
            const float re = co * amp, im = sn * amp;
            const float2 t = tilt[e];
            E[r * pe + c] = make_float2(re * t.x - im * t.y, re * t.y + im * t.x);
        }
        __syncwarp();
        // DFT along columns on the kept frequencies: G[r][b] = sum_c E[r][c] W[b][c]
        for (int e0 = lane; e0 < p * cs; e0 += 32 * kU) {
            int rr[kU], bb[kU];
            float xr[kU], xi[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int e = min(e0 + 32 * u, p * cs - 1);
                rr[u] = e / cs;
                bb[u] = e - rr[u] * cs;
                xr[u] = 0.f;
                xi[u] = 0.f;
            }
            for (int c = 0; c < p; ++c) {
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const float2 x = E[rr[u] * pe + c], w = twT[c * cs + bb[u]];
                    xr[u] = fmaf(x.x, w.x, fmaf(-x.y, w.y, xr[u]));
                    xi[u] = fmaf(x.x, w.y, fmaf(x.y, w.x, xi[u]));
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (e0 + 32 * u < p * cs) G[rr[u] * cs + bb[u]] = make_float2(xr[u], xi[u]);
        }
        __syncwarp();
        // DFT along rows, |F|^2 and field stop (sh.py:378-399)
        for (int e0 = lane; e0 < cs * cs; e0 += 32 * kU) {
            int aa[kU], bb[kU];
            float xr[kU], xi[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int e = min(e0 + 32 * u, cs * cs - 1);
                aa[u] = e / cs;
                bb[u] = e - aa[u] * cs;
                xr[u] = 0.f;
                xi[u] = 0.f;
            }
            for (int r = 0; r < p; ++r) {
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    const float2 x = G[r * cs + bb[u]], w = twT[r * cs + aa[u]];
                    xr[u] = fmaf(x.x, w.x, fmaf(-x.y, w.y, xr[u]));
                    xi[u] = fmaf(x.x, w.y, fmaf(x.y, w.x, xi[u]));
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u)
                if (e0 + 32 * u < cs * cs) {
                    const int e = aa[u] * cs + bb[u];
                    I[e] = (xr[u] * xr[u] + xi[u] * xi[u]) * mask[e];
                }
        }
        __syncwarp();
        // LCM area rebin, separable (toccd.py:55-61): H = I R^T, D = R H
        for (int e = lane; e < cs * npx; e += 32) {
            const int aa = e / npx, q = e - aa * npx;
            float acc = 0.f;
            const float *ia = I + aa * cs;
            const float *rq = R + q * cs;
            for (int b = 0; b < cs; ++b) acc = fmaf(ia[b], rq[b], acc);
            H[e] = acc;
        }
        __syncwarp();
        const int out_ld = a.n * npx;
        for (int e = lane; e < npx * npx; e += 32) {
            const int pp = e / npx, q = e - pp * npx;
            float acc = 0.f;
            const float *rp = R + pp * cs;
            for (int aa = 0; aa < cs; ++aa) acc = fmaf(rp[aa], H[aa * npx + q], acc);
            a.out[((size_t)i * npx + pp) * out_ld + (size_t)j * npx + q] = acc;
            local += acc;
        }
    }
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    const float tot = sb::block_sum(local, red);
    // partial sum of the normalising amplitude: disjoint contiguous chunks
    const int nblk = gridDim.x * gridDim.y;
    const int chunk = (a.n_norm + nblk - 1) / nblk;
    const int lo = bid * chunk;
    const int hi = min(a.n_norm, lo + chunk);
    float sa = 0.f;
    for (int e = lo + threadIdx.x; e < hi; e += blockDim.x) sa += norm_amp(a, e);
    const float tota = sb::block_sum(sa, red);
    if (threadIdx.x == 0) {
        a.part_I[bid] = tot;
        a.part_A[bid] = tota;
    }
}

// ---------------------------------------------------------------------------
// Compile-time-sized variant for the common geometries.  Same math as
// sh_forward_kernel; every DFT product is a small complex matrix product
// computed by the warp with a register block of RB x CB outputs per lane
// (operands loaded once per k and reused RB*CB times), loops unrolled.
// ---------------------------------------------------------------------------

// this CTA's place in the grid of one realisation (a launch over several
// groups maps its flat index to it)
struct ShBlk {
    int x, y, gx, gy;
};

__device__ __forceinline__ ShBlk grid_blk(const ShArgs &a) {
    return {(int)blockIdx.x, (int)blockIdx.y + a.row0, (int)gridDim.x, a.grid_rows ? a.grid_rows : (int)gridDim.y};
}

// the compile-time kernel's shared memory (per-warp buffers for 8 warps)
// nonzero: a bounded wait of an SH kernel timed out (tensor-core stages, or 9: a field tile)
__device__ int g_sh_tc_status = 0;

template <int P, int CS, int NPX>
struct FixedSmem {
    float2 twT[P * CS];          // twT[c][b] = W[b][c]
    float2 tilt[P * P];
    float mask[CS * CS];
    float R[NPX * CS];
    float2 Es[8][P * (P + 1)];
    float2 Gs[8][P * CS > (CS * NPX + 1) / 2 ? P * CS : (CS * NPX + 1) / 2];
    float Is[8][CS * CS];
    float red[33];
};

template <int P, int CS, int NPX>
__device__ __forceinline__ void sh_fixed_body(const ShArgs &a, const ShBlk &blk, FixedSmem<P, CS, NPX> &S,
                                              const float *tileA = nullptr, const float *tileP = nullptr,
                                              uint64_t *tile_bar = nullptr) {
    constexpr int PE = P + 1;
    float2 *twT = S.twT, *tilt = S.tilt;
    float *mask = S.mask, *R = S.R, *red = S.red;
    for (int e = threadIdx.x; e < CS * P; e += blockDim.x) {
        const int b = e / P, c = e - b * P;
        twT[c * CS + b] = a.tw[e];
    }
    for (int e = threadIdx.x; e < P * P; e += blockDim.x) tilt[e] = a.tilt[e];
    for (int e = threadIdx.x; e < CS * CS; e += blockDim.x) mask[e] = a.mask[e];
    for (int e = threadIdx.x; e < NPX * CS; e += blockDim.x) R[e] = a.rebin[e];
    __syncthreads();
    if (tile_bar && !sb::mbar_wait(tile_bar, 0)) {
        // the field tile did not land in time: record it (stage 9 of the SH
        // status), give the copies one more bounded wait and read the field
        // from global memory
        atomicExch(&g_sh_tc_status, 9);
        sb::mbar_wait(tile_bar, 0);
        tileA = nullptr;
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blk.y;
    const int j = blk.x * a.spc + warp;
    float2 *E = S.Es[warp];
    float2 *G = S.Gs[warp];
    float *I = S.Is[warp];
    float local = 0.f;
    if (j < a.n) {
        const size_t row0 = (size_t)i * P, col0 = (size_t)j * P;
#pragma unroll
        for (int e = lane; e < P * P; e += 32) {
            const int r = e / P, c = e % P;
            float amp, phn;
            if (tileA) {
                // the CTA's field tile: P rows x spc * P columns, this warp's P columns
                const int o = r * (a.spc * P) + warp * P + c;
                amp = tileA[o];
                phn = tileP[o];
            } else {
                const size_t g = (row0 + r) * (size_t)a.ld + col0 + c;
                field_at(a, g, amp, phn);
            }
            const float phi = phn * a.k;
            float sn, co;
            sincosf(phi, &sn, &co);
            const float re = co * amp, im = sn * amp;
            const float2 t = tilt[e];
            E[r * PE + c] = make_float2(re * t.x - im * t.y, re * t.y + im * t.x);
        }
        __syncwarp();
        // G = E W^T  (P x CS)
        sb::warp_cgemm<P, CS, P, PE, 1, CS>(E, twT, lane, [&](int r, int b, float xr, float xi) {
            G[r * CS + b] = make_float2(xr, xi);
        });
        __syncwarp();
        // F = W G  (CS x CS); I = |F|^2 * field stop  (sh.py:378-399)
        sb::warp_cgemm<CS, CS, P, 1, CS, CS>(twT, G, lane, [&](int aa, int b, float xr, float xi) {
            I[aa * CS + b] = (xr * xr + xi * xi) * mask[aa * CS + b];
        });
        __syncwarp();
        const int out_ld = a.n * NPX;
        if constexpr (CS % NPX == 0) {
            // integer rebin factor: each detector pixel is a BF x BF box of
            // the cut window, weighted 1/BF^2 (R holds 1/BF on its band)
            constexpr int BF = CS / NPX;
            const float wgt = R[0] * R[0];
#pragma unroll
            for (int e = lane; e < NPX * NPX; e += 32) {
                const int pp = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int u = 0; u < BF; ++u)
#pragma unroll
                    for (int v = 0; v < BF; ++v) acc += I[(pp * BF + u) * CS + q * BF + v];
                acc *= wgt;
                a.out[((size_t)i * NPX + pp) * out_ld + (size_t)j * NPX + q] = acc;
                local += acc;
            }
        } else {
            // general LCM rebin (toccd.py:55-61): H = I R^T, D = R H
            float *H = reinterpret_cast<float *>(G);   // G is consumed
#pragma unroll
            for (int e = lane; e < CS * NPX; e += 32) {
                const int aa = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int b = 0; b < CS; ++b) acc = fmaf(I[aa * CS + b], R[q * CS + b], acc);
                H[e] = acc;
            }
            __syncwarp();
#pragma unroll
            for (int e = lane; e < NPX * NPX; e += 32) {
                const int pp = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int aa = 0; aa < CS; ++aa) acc = fmaf(R[pp * CS + aa], H[aa * NPX + q], acc);
                a.out[((size_t)i * NPX + pp) * out_ld + (size_t)j * NPX + q] = acc;
                local += acc;
            }
        }
    }
    const int bid = blk.y * blk.gx + blk.x;
    const float tot = sb::block_sum(local, red);
    const int nblk = blk.gx * blk.gy;
    const int chunk = (a.n_norm + nblk - 1) / nblk;
    const int lo = bid * chunk;
    const int hi = min(a.n_norm, lo + chunk);
    float sa = 0.f;
    for (int e = lo + threadIdx.x; e < hi; e += blockDim.x) sa += norm_amp(a, e);
    const float tota = sb::block_sum(sa, red);
    if (threadIdx.x == 0) {
        a.part_I[bid] = tot;
        a.part_A[bid] = tota;
    }
}

template <int P, int CS, int NPX>
__global__ void __launch_bounds__(256, 4) sh_forward_fixed_kernel(ShArgs a) {
    batch_slice(a);
    __shared__ FixedSmem<P, CS, NPX> S;
    sh_fixed_body<P, CS, NPX>(a, grid_blk(a), S);
}

// The same kernel with the CTA's field tile (its lenslet row's P field rows
// under its spc sub-apertures, amplitude and phase) staged in shared memory
// by two 2-D TMA loads issued at entry, so the tile is in flight while the
// CTA loads its DFT tables.  Single field without the mirror term; the same
// arithmetic on the same values as the plain kernel (bit-identical frames).
// Columns past the field read as zero and feed no sub-aperture.
template <int P, int CS, int NPX>
__global__ void __launch_bounds__(256, 4) sh_forward_fixed_tma_kernel(ShArgs a, const __grid_constant__ CUtensorMap mapA,
                                                                      const __grid_constant__ CUtensorMap mapP) {
    __shared__ FixedSmem<P, CS, NPX> S;
    __shared__ __align__(128) float tileA[8 * P * P];
    __shared__ __align__(128) float tileP[8 * P * P];
    __shared__ __align__(8) uint64_t bar;
    const ShBlk blk = grid_blk(a);
    if (threadIdx.x == 0) {
        sb::mbar_init(&bar, 1);
        sb::mbar_init_fence();
        sb::mbar_arrive_expect_tx(&bar, (uint32_t)(2 * a.spc * P * P * sizeof(float)));
        const uint64_t pol = sb::l2_evict_first_policy();
        sb::tma_load_2d(tileA, &mapA, blk.x * a.spc * P, blk.y * P, &bar, pol);
        sb::tma_load_2d(tileP, &mapP, blk.x * a.spc * P, blk.y * P, &bar, pol);
    }
    sh_fixed_body<P, CS, NPX>(a, blk, S, tileA, tileP, &bar);
}

// ---------------------------------------------------------------------------
// Split-BF16 tensor-core form (tcgen05).  One CTA of 128 threads takes 16
// consecutive sub-apertures of a lenslet row and runs both DFT products as
// real GEMMs on the tensor cores, every operand split as x = hi + lo (bf16)
// and each product as hi*hi + lo*hi + hi*lo: three K=16 MMAs, FP32
// accumulation in tensor memory.
//   stage 1  rows (sub-aperture s, field row r): 16 x 8 = 128
//            K    [Re E[r][c], Im E[r][c]]  (c < 8)
//            N    [Re G[r][b], Im G[r][b]]  (b < cutsize, padded to 16/32)
//   stage 2  rows (s, kept column b): two tiles of 8 sub-apertures x 16
//            K    [Re G[r][b], Im G[r][b]]  (r < 8)
//            N    [Re F[a][b], Im F[a][b]]  (a < cutsize)
// Both stages multiply by the same B, the real form of the pruned DFT rows
// W[b][c].  Between the stages G goes from tensor memory to shared memory
// in FP32 (transposed to column-major per sub-aperture) and is split again.
// The field build, |F|^2, the field stop, the rebin and the photon
// partials run on the CUDA cores as in the FP32 form.
// ---------------------------------------------------------------------------

constexpr int kTcSub = 16;              // sub-apertures per CTA
constexpr int kTcThreads = 128;         // one thread per MMA row
constexpr uint32_t kTcTmemCols = 64;    // stage 1 in columns 0-31, then stage 2 tiles in 0-31 and 32-63
constexpr int kTcOperandBytes = 128 * 32;   // one 128-row x 16 bf16 operand


template <int CS>
struct TcShape {
    static constexpr int NB = 2 * CS <= 16 ? 16 : 32;   // MMA N
};

// Dynamic shared memory per CTA: the operands (whose space holds |F|^2 once
// both products are done) and the tables, 26-29 KB: at most 8 CTAs, 512
// tensor-memory columns, share an SM, so the allocation never waits.
template <int P, int CS, int NPX>
__host__ __device__ constexpr size_t tc_smem_bytes() {
    return 6 * (size_t)kTcOperandBytes + 2 * (size_t)TcShape<CS>::NB * 32 + (size_t)P * P * 8 +
           (size_t)CS * CS * 4 + (size_t)NPX * CS * 4 + 8 + 16;
}
static_assert(tc_smem_bytes<8, 8, 8>() * 9 > 228 * 1024, "more than 8 CTAs per SM would exceed tensor memory");

template <int P, int CS, int NPX>
__device__ __forceinline__ void sh_tc_body(const ShArgs &a, const ShBlk &blk) {
    static_assert(P == 8, "one 16-byte K segment per field row");
    static_assert(CS <= 16, "one 16-row stage-2 block per sub-aperture");
    static_assert(kTcSub * CS * CS * 4 <= 6 * kTcOperandBytes, "the intensity buffer reuses the operand space");
    constexpr int NB = TcShape<CS>::NB;
    constexpr uint32_t IDESC = sb::umma_idesc_bf16_f32(128, NB);
    constexpr uint32_t LBO_A = 128 * 16, LBO_B = NB * 16;
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char *A1h = tc_smem, *A1l = tc_smem + kTcOperandBytes;
    unsigned char *A2h = tc_smem + 2 * kTcOperandBytes;   // two tiles
    unsigned char *A2l = tc_smem + 4 * kTcOperandBytes;   // two tiles
    unsigned char *Bh = tc_smem + 6 * kTcOperandBytes, *Bl = Bh + NB * 32;
    float *Ib = reinterpret_cast<float *>(tc_smem);   // |F|^2, once both products are done
    float2 *tilt = reinterpret_cast<float2 *>(Bl + NB * 32);
    float *mask = reinterpret_cast<float *>(tilt + P * P);
    float *R = mask + CS * CS;
    uint64_t *bar = reinterpret_cast<uint64_t *>((reinterpret_cast<uintptr_t>(R + NPX * CS) + 7) & ~(uintptr_t)7);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);
    __shared__ float red[33];

    const int t = threadIdx.x, warp = t >> 5;
    // issue the global loads first: this thread's field row and its share of
    // the normalising amplitude; the table set-up below overlaps them
    const int i = blk.y;
    const int s = t >> 3, r = t & 7;
    const int j = blk.x * kTcSub + s;
    float amp[8], phv[8];
    if (j < a.n) {
        const size_t g = (size_t)(i * P + r) * a.ld + (size_t)j * P;
        if (a.vec) {
            const float4 a0 = *reinterpret_cast<const float4 *>(a.A + g);
            const float4 a1 = *reinterpret_cast<const float4 *>(a.A + g + 4);
            const float4 p0 = *reinterpret_cast<const float4 *>(a.ph + g);
            const float4 p1 = *reinterpret_cast<const float4 *>(a.ph + g + 4);
            amp[0] = a0.x; amp[1] = a0.y; amp[2] = a0.z; amp[3] = a0.w;
            amp[4] = a1.x; amp[5] = a1.y; amp[6] = a1.z; amp[7] = a1.w;
            phv[0] = p0.x; phv[1] = p0.y; phv[2] = p0.z; phv[3] = p0.w;
            phv[4] = p1.x; phv[5] = p1.y; phv[6] = p1.z; phv[7] = p1.w;
        } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                amp[c] = a.A[g + c];
                phv[c] = a.ph[g + c];
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) amp[c] = phv[c] = 0.f;
    }
    const int bid = blk.y * blk.gx + blk.x;
    float sa = 0.f;
    {
        const int nblk = blk.gx * blk.gy;
        const int chunk = (a.n_norm + nblk - 1) / nblk;
        const int lo = bid * chunk;
        const int hi = min(a.n_norm, lo + chunk);
        for (int e = lo + t; e < hi; e += kTcThreads) sa += a.A_norm[e];
    }
    if (warp == 0) {
        sb::tmem_alloc(tmem_slot, kTcTmemCols);
        sb::tmem_relinquish();
    }
    if (t == 0) {
        sb::mbar_init(bar, 1);
        sb::mbar_init_fence();
    }
    for (int e = t; e < P * P; e += kTcThreads) tilt[e] = a.tilt[e];
    for (int e = t; e < CS * CS; e += kTcThreads) mask[e] = a.mask[e];
    for (int e = t; e < NPX * CS; e += kTcThreads) R[e] = a.rebin[e];
    // B: real form of W.  Row n < CS gives Re of output b = n, row CS + b its
    // Im; K segment 0 multiplies the real parts, segment 1 the imaginary ones.
    for (int e = t; e < NB * 2; e += kTcThreads) {
        const int n = e >> 1, seg = e & 1;
        float x[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float v = 0.f;
            if (n < 2 * CS) {
                const float2 w = a.tw[(n < CS ? n : n - CS) * P + c];
                v = n < CS ? (seg == 0 ? w.x : -w.y) : (seg == 0 ? w.y : w.x);
            }
            x[c] = v;
        }
        uint4 h, l;
        sb::split_bf16x8(x, h, l);
        *reinterpret_cast<uint4 *>(Bh + seg * LBO_B + n * 16) = h;
        *reinterpret_cast<uint4 *>(Bl + seg * LBO_B + n * 16) = l;
    }
    if constexpr (CS < 16) {
        // stage-2 rows b >= cutsize of every sub-aperture block stay zero
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (int e = t; e < kTcSub * (16 - CS); e += kTcThreads) {
            const int s2 = e / (16 - CS), b = CS + e % (16 - CS);
            const int off = (s2 >> 3) * kTcOperandBytes + ((s2 & 7) * 16 + b) * 16;
            *reinterpret_cast<uint4 *>(A2h + off) = z;
            *reinterpret_cast<uint4 *>(A2h + off + LBO_A) = z;
            *reinterpret_cast<uint4 *>(A2l + off) = z;
            *reinterpret_cast<uint4 *>(A2l + off + LBO_A) = z;
        }
    }
    __syncthreads();

    // field build (electric_field.py:60-75 and sh.py:376): thread t holds row r of sub-aperture s
    {
        float er[8], ei[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float phi = phv[c] * a.k;
            float sn, co;
            sincosf(phi, &sn, &co);
            const float re = co * amp[c], im = sn * amp[c];
            const float2 tl = tilt[r * P + c];
            er[c] = re * tl.x - im * tl.y;
            ei[c] = re * tl.y + im * tl.x;
        }
        uint4 h, l;
        sb::split_bf16x8(er, h, l);
        *reinterpret_cast<uint4 *>(A1h + t * 16) = h;
        *reinterpret_cast<uint4 *>(A1l + t * 16) = l;
        sb::split_bf16x8(ei, h, l);
        *reinterpret_cast<uint4 *>(A1h + LBO_A + t * 16) = h;
        *reinterpret_cast<uint4 *>(A1l + LBO_A + t * 16) = l;
    }
    sb::fence_proxy_async_smem();
    sb::tc_fence_before_sync();
    __syncthreads();
    sb::tc_fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const uint64_t bh = sb::umma_desc_kmajor(Bh, LBO_B), bl = sb::umma_desc_kmajor(Bl, LBO_B);

    // stage 1: G = E W^T
    if (t == 0) {
        const uint64_t ah = sb::umma_desc_kmajor(A1h, LBO_A), al = sb::umma_desc_kmajor(A1l, LBO_A);
        sb::umma_bf16(tmem, ah, bh, IDESC, 0u);
        sb::umma_bf16(tmem, al, bh, IDESC, 1u);
        sb::umma_bf16(tmem, ah, bl, IDESC, 1u);
        sb::umma_commit(bar);
    }
    int pending = 0;                    // parity of the commit still to be waited for after a timeout
    int failed = __syncthreads_or(!sb::mbar_wait(bar, 0));
    float local = 0.f;
    if (!failed) {
        sb::tc_fence_after_sync();
        uint32_t v[2][16];
        sb::tmem_ld16(tmem + lane_base, v[0]);
        if constexpr (NB == 32) sb::tmem_ld16(tmem + lane_base + 16, v[1]);
        sb::tmem_wait_ld(v[0]);
        if constexpr (NB == 32) sb::tmem_wait_ld(v[1]);
        // stage-2 operand rows (s, b) hold column b of G_s: K element r is
        // this thread's G[r][b], split straight from tensor memory (the
        // split of each value as split_bf16x8 forms it); the lanes of rows
        // r and r + 1 pair their 16-bit halves so the even lane stores a word
#pragma unroll
        for (int b = 0; b < CS; ++b) {
            const int nr = b, ni = CS + b;
            const float gre = __uint_as_float(v[nr >> 4][nr & 15]);
            const float gim = __uint_as_float(v[ni >> 4][ni & 15]);
            const __nv_bfloat16 hr = __float2bfloat16_rn(gre), hi = __float2bfloat16_rn(gim);
            const __nv_bfloat16 lr = __float2bfloat16_rn(gre - __bfloat162float(hr));
            const __nv_bfloat16 li = __float2bfloat16_rn(gim - __bfloat162float(hi));
            const uint32_t own_r = (uint32_t)__bfloat16_as_ushort(hr) | ((uint32_t)__bfloat16_as_ushort(lr) << 16);
            const uint32_t own_i = (uint32_t)__bfloat16_as_ushort(hi) | ((uint32_t)__bfloat16_as_ushort(li) << 16);
            const uint32_t nb_r = __shfl_xor_sync(0xffffffffu, own_r, 1);
            const uint32_t nb_i = __shfl_xor_sync(0xffffffffu, own_i, 1);
            if ((r & 1) == 0) {
                const int off = (s >> 3) * kTcOperandBytes + ((s & 7) * 16 + b) * 16 + r * 2;
                *reinterpret_cast<uint32_t *>(A2h + off) = (own_r & 0xffffu) | (nb_r << 16);
                *reinterpret_cast<uint32_t *>(A2l + off) = (own_r >> 16) | (nb_r & 0xffff0000u);
                *reinterpret_cast<uint32_t *>(A2h + off + LBO_A) = (own_i & 0xffffu) | (nb_i << 16);
                *reinterpret_cast<uint32_t *>(A2l + off + LBO_A) = (own_i >> 16) | (nb_i & 0xffff0000u);
            }
        }
        sb::fence_proxy_async_smem();
        sb::tc_fence_before_sync();
        __syncthreads();
        sb::tc_fence_after_sync();
        // stage 2: F^T = G^T W^T per sub-aperture, tile k into columns 32k..32k+31
        if (t == 0) {
#pragma unroll
            for (int tile = 0; tile < 2; ++tile) {
                const uint64_t ah = sb::umma_desc_kmajor(A2h + tile * kTcOperandBytes, LBO_A);
                const uint64_t al = sb::umma_desc_kmajor(A2l + tile * kTcOperandBytes, LBO_A);
                const uint32_t d = tmem + 32u * tile;
                sb::umma_bf16(d, ah, bh, IDESC, 0u);
                sb::umma_bf16(d, al, bh, IDESC, 1u);
                sb::umma_bf16(d, ah, bl, IDESC, 1u);
            }
            sb::umma_commit(bar);
        }
        failed = __syncthreads_or(!sb::mbar_wait(bar, 1));
        pending = 1;
        if (!failed) {
            sb::tc_fence_after_sync();
            // |F|^2 and the field stop (sh.py:378-399): thread t holds column b of sub-aperture s2
#pragma unroll
            for (int tile = 0; tile < 2; ++tile) {
                uint32_t w[2][16];
                sb::tmem_ld16(tmem + lane_base + 32u * tile, w[0]);
                if constexpr (NB == 32) sb::tmem_ld16(tmem + lane_base + 32u * tile + 16, w[1]);
                sb::tmem_wait_ld(w[0]);
                if constexpr (NB == 32) sb::tmem_wait_ld(w[1]);
                const int s2 = tile * 8 + (t >> 4), b = t & 15;
                if (b < CS) {
#pragma unroll
                    for (int aa = 0; aa < CS; ++aa) {
                        const int nr = aa, ni = CS + aa;
                        const float fr = __uint_as_float(w[nr >> 4][nr & 15]);
                        const float fi = __uint_as_float(w[ni >> 4][ni & 15]);
                        Ib[s2 * CS * CS + aa * CS + b] = (fr * fr + fi * fi) * mask[aa * CS + b];
                    }
                }
            }
            __syncthreads();
            // rebin (toccd.py:55-61) and output; consecutive threads write consecutive pixels of a detector row
            const int out_ld = a.n * NPX;
            for (int e = t; e < NPX * kTcSub * NPX; e += kTcThreads) {
                const int pp = e / (kTcSub * NPX), rem = e - pp * (kTcSub * NPX);
                const int s2 = rem / NPX, q = rem - s2 * NPX;
                const int j2 = blk.x * kTcSub + s2;
                if (j2 >= a.n) continue;
                const float *I = Ib + s2 * CS * CS;
                float acc = 0.f;
                if constexpr (CS % NPX == 0) {
                    constexpr int BF = CS / NPX;
#pragma unroll
                    for (int u = 0; u < BF; ++u)
#pragma unroll
                        for (int vv = 0; vv < BF; ++vv) acc += I[(pp * BF + u) * CS + q * BF + vv];
                    acc *= R[0] * R[0];
                } else {
#pragma unroll
                    for (int aa = 0; aa < CS; ++aa) {
                        float h = 0.f;
#pragma unroll
                        for (int b = 0; b < CS; ++b) h = fmaf(I[aa * CS + b], R[q * CS + b], h);
                        acc = fmaf(R[pp * CS + aa], h, acc);
                    }
                }
                a.out[((size_t)i * NPX + pp) * out_ld + (size_t)j2 * NPX + q] = acc;
                local += acc;
            }
        }
    }
    if (failed) {
        // record, then give the MMAs in flight one more bounded wait before the
        // tensor memory is released; the frame of this launch is not valid
        if (t == 0) atomicExch(&g_sh_tc_status, 1 + pending);
        sb::mbar_wait(bar, pending);
    }
    const float tot = sb::block_sum(local, red);
    const float tota = sb::block_sum(sa, red);
    if (t == 0) {
        a.part_I[bid] = tot;
        a.part_A[bid] = tota;
    }
    sb::tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        sb::tc_fence_after_sync();
        sb::tmem_dealloc(tmem, kTcTmemCols);
    }
}

template <int P, int CS, int NPX>
__global__ void __launch_bounds__(kTcThreads) sh_forward_tc_kernel(ShArgs a) {
    batch_slice(a);
    sh_tc_body<P, CS, NPX>(a, grid_blk(a));
}

// ---------------------------------------------------------------------------
// Laser-guide-star form (sh.py:382-394): the sub-aperture's unshifted
// |FFT|^2 on the full N x N grid is correlated with its sodium-spot kernel
// through FFTs, psf = Re(IFFT_unnormalised(FFT(|F|^2) * K)), then field stop,
// cut and rebin as usual (the kernel is centred, so no fftshift).  One warp
// per sub-aperture, every transform a small complex matrix product:
//   G  = E Wf^T                       (P x N)      Wf[k][c] = e^{-2 pi i k c / N}
//   I  = |Wf G|^2                     (N x N)
//   H  = I W                          (N x N)      W[u][x]  = e^{-2 pi i u x / N}
//   S  = (W H) .* K_s                 (N x N)      K_s: the kernel spectrum
//   T  = S V^T                        (N x CS)     V[a][u]  = e^{+2 pi i (a + c0) u / N}
//   Ic = Re(V T) .* field stop        (CS x CS)    c0 = cutpixels / 2
// ---------------------------------------------------------------------------

struct LgsArgs {
    const float2 *wf_t;     // [P][N]: Wf transposed
    const float2 *w;        // [N][N]
    const float2 *v_t;      // [N][CS]: V transposed
    const float2 *kspec;    // [n*n][N][N]
};

template <int N>
__host__ __device__ constexpr int lgs_warps() { return N >= 32 ? 4 : 8; }

template <int P, int N, int CS, int NPX>
constexpr size_t lgs_smem_bytes() {
    return ((size_t)P * N + (size_t)N * N + (size_t)N * CS + (size_t)P * P) * 8 + (size_t)CS * CS * 4 +
           (size_t)NPX * CS * 4 + (size_t)lgs_warps<N>() * ((size_t)P * (P + 1) + 2 * (size_t)N * N) * 8;
}

template <int P, int N, int CS, int NPX>
__global__ void __launch_bounds__(32 * lgs_warps<N>()) sh_forward_lgs_kernel(ShArgs a, LgsArgs g) {
    static_assert(CS <= N && P <= N, "cut window and field inside the FFT grid");
    constexpr int PE = P + 1;
    constexpr int WPC = lgs_warps<N>();
    extern __shared__ __align__(16) unsigned char lgs_smem[];
    float2 *wf_t = reinterpret_cast<float2 *>(lgs_smem);   // [P][N]
    float2 *w = wf_t + P * N;                               // [N][N]
    float2 *v_t = w + N * N;                                // [N][CS]
    float2 *tilt = v_t + N * CS;                            // [P][P]
    float *mask = reinterpret_cast<float *>(tilt + P * P);  // [CS][CS]
    float *R = mask + CS * CS;                              // [NPX][CS]
    float2 *per_warp = reinterpret_cast<float2 *>(R + NPX * CS);
    __shared__ float red[33];
    for (int e = threadIdx.x; e < P * N; e += blockDim.x) wf_t[e] = g.wf_t[e];
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) w[e] = g.w[e];
    for (int e = threadIdx.x; e < N * CS; e += blockDim.x) v_t[e] = g.v_t[e];
    for (int e = threadIdx.x; e < P * P; e += blockDim.x) tilt[e] = a.tilt[e];
    for (int e = threadIdx.x; e < CS * CS; e += blockDim.x) mask[e] = a.mask[e];
    for (int e = threadIdx.x; e < NPX * CS; e += blockDim.x) R[e] = a.rebin[e];
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.y;
    const int j = blockIdx.x * WPC + warp;
    float2 *E = per_warp + (size_t)warp * (P * PE + 2 * N * N);
    float2 *bufA = E + P * PE;
    float2 *bufB = bufA + N * N;
    float local = 0.f;
    if (j < a.n) {
        const size_t row0 = (size_t)i * P, col0 = (size_t)j * P;
#pragma unroll
        for (int e = lane; e < P * P; e += 32) {
            const int r = e / P, c = e % P;
            const size_t gi = (row0 + r) * (size_t)a.ld + col0 + c;
            const float amp = a.A[gi];
            const float phi = a.ph[gi] * a.k;
            float sn, co;
            sincosf(phi, &sn, &co);
            const float re = co * amp, im = sn * amp;
            const float2 t = tilt[e];
            E[r * PE + c] = make_float2(re * t.x - im * t.y, re * t.y + im * t.x);
        }
        __syncwarp();
        sb::warp_cgemm<P, N, P, PE, 1, N>(E, wf_t, lane, [&](int r, int k, float xr, float xi) {
            bufA[r * N + k] = make_float2(xr, xi);
        });
        __syncwarp();
        sb::warp_cgemm<N, N, P, 1, N, N>(wf_t, bufA, lane, [&](int u, int v, float xr, float xi) {
            bufB[u * N + v] = make_float2(xr * xr + xi * xi, 0.f);
        });
        __syncwarp();
        sb::warp_cgemm<N, N, N, N, 1, N>(bufB, w, lane, [&](int x, int v, float xr, float xi) {
            bufA[x * N + v] = make_float2(xr, xi);
        });
        __syncwarp();
        const float2 *ks = g.kspec + ((size_t)i * a.n + j) * (N * N);
        sb::warp_cgemm<N, N, N, N, 1, N>(w, bufA, lane, [&](int u, int v, float xr, float xi) {
            const float2 kk = __ldg(ks + u * N + v);
            bufB[u * N + v] = make_float2(xr * kk.x - xi * kk.y, xr * kk.y + xi * kk.x);
        });
        __syncwarp();
        sb::warp_cgemm<N, CS, N, N, 1, CS>(bufB, v_t, lane, [&](int u, int b, float xr, float xi) {
            bufA[u * CS + b] = make_float2(xr, xi);
        });
        __syncwarp();
        float *Ic = reinterpret_cast<float *>(bufB);
        sb::warp_cgemm<CS, CS, N, 1, CS, CS>(v_t, bufA, lane, [&](int aa, int b, float xr, float xi) {
            Ic[aa * CS + b] = xr * mask[aa * CS + b];
        });
        __syncwarp();
        const int out_ld = a.n * NPX;
        if constexpr (CS % NPX == 0) {
            constexpr int BF = CS / NPX;
            const float wgt = R[0] * R[0];
#pragma unroll
            for (int e = lane; e < NPX * NPX; e += 32) {
                const int pp = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int u = 0; u < BF; ++u)
#pragma unroll
                    for (int v = 0; v < BF; ++v) acc += Ic[(pp * BF + u) * CS + q * BF + v];
                acc *= wgt;
                a.out[((size_t)i * NPX + pp) * out_ld + (size_t)j * NPX + q] = acc;
                local += acc;
            }
        } else {
            float *H = reinterpret_cast<float *>(bufA);
#pragma unroll
            for (int e = lane; e < CS * NPX; e += 32) {
                const int aa = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int b = 0; b < CS; ++b) acc = fmaf(Ic[aa * CS + b], R[q * CS + b], acc);
                H[e] = acc;
            }
            __syncwarp();
#pragma unroll
            for (int e = lane; e < NPX * NPX; e += 32) {
                const int pp = e / NPX, q = e % NPX;
                float acc = 0.f;
#pragma unroll
                for (int aa = 0; aa < CS; ++aa) acc = fmaf(R[pp * CS + aa], H[aa * NPX + q], acc);
                a.out[((size_t)i * NPX + pp) * out_ld + (size_t)j * NPX + q] = acc;
                local += acc;
            }
        }
    }
    const int bid = blockIdx.y * gridDim.x + blockIdx.x;
    const float tot = sb::block_sum(local, red);
    const int nblk = gridDim.x * gridDim.y;
    const int chunk = (a.n_norm + nblk - 1) / nblk;
    const int lo = bid * chunk;
    const int hi = min(a.n_norm, lo + chunk);
    float sa = 0.f;
    for (int e = lo + threadIdx.x; e < hi; e += blockDim.x) sa += norm_amp(a, e);
    const float tota = sb::block_sum(sa, red);
    if (threadIdx.x == 0) {
        a.part_I[bid] = tot;
        a.part_A[bid] = tota;
    }
}

typedef void (*ShLgsKernel)(ShArgs, LgsArgs);

struct ShLgsEntry {
    ShLgsKernel fn;
    int warps;
    size_t smem;
};

// geometries with an LGS kernel: (np_sub, fft_size, cutsize, subap_npx)
template <int P, int N, int CS, int NPX>
ShLgsEntry lgs_entry() {
    return {sh_forward_lgs_kernel<P, N, CS, NPX>, lgs_warps<N>(), lgs_smem_bytes<P, N, CS, NPX>()};
}
ShLgsEntry lgs_kernel(int p, int n_fft, int cs, int npx) {
    if (p == 8 && n_fft == 16 && cs == 12 && npx == 6) return lgs_entry<8, 16, 12, 6>();
    if (p == 8 && n_fft == 32 && cs == 12 && npx == 6) return lgs_entry<8, 32, 12, 6>();
    if (p == 8 && n_fft == 16 && cs == 14 && npx == 8) return lgs_entry<8, 16, 14, 8>();
    if (p == 8 && n_fft == 32 && cs == 16 && npx == 8) return lgs_entry<8, 32, 16, 8>();
    return {nullptr, 0, 0};
}

typedef void (*ShKernel)(ShArgs);

struct ShTcKernel {
    ShKernel fn;
    size_t smem;
};

// geometries with a split-BF16 tensor-core kernel: (np_sub, cutsize, subap_npx)
ShTcKernel tc_kernel(int p, int cs, int npx) {
    if (p == 8 && cs == 12 && npx == 6) return {sh_forward_tc_kernel<8, 12, 6>, tc_smem_bytes<8, 12, 6>()};
    if (p == 8 && cs == 14 && npx == 8) return {sh_forward_tc_kernel<8, 14, 8>, tc_smem_bytes<8, 14, 8>()};
    if (p == 8 && cs == 16 && npx == 8) return {sh_forward_tc_kernel<8, 16, 8>, tc_smem_bytes<8, 16, 8>()};
    if (p == 8 && cs == 8 && npx == 8) return {sh_forward_tc_kernel<8, 8, 8>, tc_smem_bytes<8, 8, 8>()};
    if (p == 8 && cs == 12 && npx == 8) return {sh_forward_tc_kernel<8, 12, 8>, tc_smem_bytes<8, 12, 8>()};
    return {nullptr, 0};
}

// geometries with a compile-time kernel: (np_sub, cutsize, subap_npx)
typedef void (*ShTmaKernel)(ShArgs, const CUtensorMap, const CUtensorMap);

ShTmaKernel fixed_tma_kernel(int p, int cs, int npx) {
    if (p == 8 && cs == 12 && npx == 6) return sh_forward_fixed_tma_kernel<8, 12, 6>;
    if (p == 8 && cs == 14 && npx == 8) return sh_forward_fixed_tma_kernel<8, 14, 8>;
    if (p == 8 && cs == 16 && npx == 8) return sh_forward_fixed_tma_kernel<8, 16, 8>;
    if (p == 8 && cs == 8 && npx == 8) return sh_forward_fixed_tma_kernel<8, 8, 8>;
    return nullptr;     // np_sub 16: the two tiles would not fit the static shared memory
}

ShKernel fixed_kernel(int p, int cs, int npx) {
    if (p == 8 && cs == 12 && npx == 6) return sh_forward_fixed_kernel<8, 12, 6>;
    if (p == 8 && cs == 14 && npx == 8) return sh_forward_fixed_kernel<8, 14, 8>;
    if (p == 8 && cs == 16 && npx == 8) return sh_forward_fixed_kernel<8, 16, 8>;
    if (p == 8 && cs == 8 && npx == 8) return sh_forward_fixed_kernel<8, 8, 8>;
    if (p == 16 && cs == 16 && npx == 8) return sh_forward_fixed_kernel<16, 16, 8>;
    return nullptr;
}

__global__ void __launch_bounds__(256) sh_normalize_kernel(const float *part_I, const float *part_A, int nparts,
                                                           float photon_scale, float *out, int n_out) {
    __shared__ double red[33];
    // batched launches: blockIdx.y selects the realisation
    part_I += (size_t)blockIdx.y * nparts;
    part_A += (size_t)blockIdx.y * nparts;
    out += (size_t)blockIdx.y * n_out;
    double si = 0.0, sa = 0.0;
    for (int e = threadIdx.x; e < nparts; e += blockDim.x) {
        si += part_I[e];
        sa += part_A[e];
    }
    si = sb::block_sum_all_d(si, red);
    sa = sb::block_sum_all_d(sa, red);
    // phot = S0 * pitch^2 * sum(A); i *= phot / sum(i)  (sh.py:426-427)
    const float phot = (float)(photon_scale * sa);
    const float scale = phot / (float)si;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_out; e += gridDim.x * blockDim.x) out[e] *= scale;
}

__global__ void edge_extrapolate_kernel(const float *ph, const int32_t *s1, const int32_t *s2, int n, float *out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int a1 = s1[e];
        float v;
        if (a1 < 0) {
            v = ph[e];
        } else {
            const int a2 = s2[e];
            v = a2 < 0 ? ph[a1] : 2.0f * ph[a1] - ph[a2];
        }
        out[e] = v;
    }
}

__global__ void interp2d_field_kernel(const float *A, const float *P, int rows, int cols, const float *yy,
                                      const float *xx, int n_out, float *Ao, float *Po) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_out; e += gridDim.x * blockDim.x) {
        // bilinear on the integer grid in double precision, like SciPy's
        // RegularGridInterpolator on the reference CPU path (interp2d.py:117-122)
        const double y = yy[e], x = xx[e];
        int y0 = (int)floor(y), x0 = (int)floor(x);
        y0 = max(0, min(y0, rows - 2));
        x0 = max(0, min(x0, cols - 2));
        const double fy = y - y0, fx = x - x0;
        const size_t i00 = (size_t)y0 * cols + x0;
        const double w00 = (1 - fy) * (1 - fx), w01 = (1 - fy) * fx, w10 = fy * (1 - fx), w11 = fy * fx;
        Ao[e] = (float)(A[i00] * w00 + A[i00 + 1] * w01 + A[i00 + cols] * w10 + A[i00 + cols + 1] * w11);
        Po[e] = (float)(P[i00] * w00 + P[i00 + 1] * w01 + P[i00 + cols] * w10 + P[i00 + cols + 1] * w11);
    }
}

// smallest sub-apertures-per-CTA of the SB_TUNE_SH_FP32 variants (8, 4, 2):
// the scratch size covers its grid
constexpr int kShMinSpc = 2;

int sh_grid(const sb_sh_plan *pl, int *spc, dim3 *grid, size_t *smem, int spc_cap = 8) {
    const ShSmem L = sh_smem_layout(pl->np_sub, pl->cutsize, pl->subap_npx);
    const int budget = 200 * 1024;
    if (L.tables + L.per_warp > budget) return -1;
    int s = (budget - L.tables) / L.per_warp;
    s = s > spc_cap ? spc_cap : s;
    if (s > pl->n_lenses) s = pl->n_lenses;
    *spc = s;
    *grid = dim3((pl->n_lenses + s - 1) / s, pl->n_lenses, 1);
    *smem = (size_t)L.tables + (size_t)s * L.per_warp;
    return 0;
}

}  // namespace

extern "C" size_t sb_sh_scratch_bytes(const sb_sh_plan *pl) {
    if (!pl) return 0;
    int spc;
    dim3 grid;
    size_t smem;
    if (sh_grid(pl, &spc, &grid, &smem, kShMinSpc)) return 0;
    const size_t nb = (size_t)grid.x * grid.y;
    return ((2 * nb * sizeof(float)) + 255) & ~(size_t)255;
}

namespace {

// mode 0: FP32 CUDA-core DFTs; mode 1: split-BF16 tensor-core DFTs
int sh_forward_impl(const char *who, const sb_sh_plan *pl, const float *A, long long sA, const float *phase_nm,
                    long long sph, const float *A_norm, long long sAn, int n_norm, float photon_scale,
                    float *intensity, long long sout, int n_batch, void *scratch, size_t scratch_bytes, void *stream,
                    int mode = 0, bool normalize = true, int *n_parts = nullptr, const float *mirror_A = nullptr,
                    const float *mirror_phase = nullptr, float *field_A = nullptr, float *field_phase = nullptr,
                    int row0 = 0, int n_rows = -1) {
    if (!pl || !A || !phase_nm || !A_norm || !intensity || !pl->twiddle || !pl->tilt || !pl->fp_mask ||
        !pl->rebin)
        return sb::fail(SB_EINVAL, "%s: null pointer", who);
    if (pl->n_lenses < 1 || pl->np_sub < 1 || pl->cutsize < 1 || pl->subap_npx < 1 || n_norm < 0 ||
        pl->field_ld < pl->n_lenses * pl->np_sub || n_batch < 1 || n_batch > 65535)
        return sb::fail(SB_EINVAL, "%s: bad geometry", who);
    int spc;
    dim3 grid;
    size_t smem;
    const int variant = mode == 0 ? sb::tune_lookup(SB_TUNE_SH_FP32, sb_tune_key(pl->n_lenses, pl->cutsize, n_batch)) : 0;
    if (sh_grid(pl, &spc, &grid, &smem, 8 >> (variant % 3)))
        return sb::fail(SB_ESHAPE, "%s: sub-aperture (np=%d, cut=%d, npx=%d) does not fit in shared memory", who,
                        pl->np_sub, pl->cutsize, pl->subap_npx);
    const size_t need = sb_sh_scratch_bytes(pl) * (size_t)n_batch;
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "%s: scratch needs %zu bytes, got %zu", who, need, scratch_bytes);
    if (mirror_A || mirror_phase || field_A || field_phase) {
        if (!mirror_A || !mirror_phase || !field_A != !field_phase)
            return sb::fail(SB_EINVAL, "%s: the mirror amplitude and phase go together, as do the field outputs", who);
        if (mode != 0 || n_batch != 1)
            return sb::fail(SB_EUNSUPPORTED, "%s: the mirror term is applied by the single-field FP32 form only", who);
        if (field_A && pl->field_ld != pl->n_lenses * pl->np_sub)
            return sb::fail(SB_EINVAL, "%s: the field outputs need a field of exactly n_lenses x np_sub columns", who);
        if (A_norm != A || n_norm != pl->field_ld * pl->field_ld)
            return sb::fail(SB_EINVAL, "%s: with the mirror term the normalising amplitude is the whole field", who);
    }
    ShTcKernel tk = {nullptr, 0};
    if (mode == 1) {
        tk = tc_kernel(pl->np_sub, pl->cutsize, pl->subap_npx);
        if (!tk.fn)
            return sb::fail(SB_EUNSUPPORTED, "%s: no split-BF16 kernel for (np=%d, cut=%d, npx=%d)", who, pl->np_sub,
                            pl->cutsize, pl->subap_npx);
        // 16 sub-apertures per CTA (never more CTAs than the FP32 grid, so the scratch size holds)
        grid = dim3((pl->n_lenses + kTcSub - 1) / kTcSub, pl->n_lenses, 1);
    }
    const int nb = grid.x * grid.y;     // the whole grid's CTAs: the partial-sum layout
    if (n_rows >= 0) {
        // a band of lenslet rows: compile-time kernels, unnormalised, one field
        if (row0 < 0 || n_rows < 1 || row0 + n_rows > pl->n_lenses || normalize || n_batch != 1 || mirror_A)
            return sb::fail(SB_EINVAL, "%s: lenslet rows %d..%d of %d", who, row0, row0 + n_rows - 1, pl->n_lenses);
        if (!tk.fn && !(spc <= 8 && fixed_kernel(pl->np_sub, pl->cutsize, pl->subap_npx)))
            return sb::fail(SB_EUNSUPPORTED, "%s: no compile-time kernel for (np=%d, cut=%d, npx=%d)", who,
                            pl->np_sub, pl->cutsize, pl->subap_npx);
        grid.y = n_rows;
    }
    ShArgs a = {};
    if (n_rows >= 0) {
        a.row0 = row0;
        a.grid_rows = pl->n_lenses;
    }
    a.n = pl->n_lenses;
    a.p = pl->np_sub;
    a.cs = pl->cutsize;
    a.npx = pl->subap_npx;
    a.ld = pl->field_ld;
    a.spc = spc;
    a.k = pl->phase_to_rad;
    a.tw = reinterpret_cast<const float2 *>(pl->twiddle);
    a.tilt = reinterpret_cast<const float2 *>(pl->tilt);
    a.mask = pl->fp_mask;
    a.rebin = pl->rebin;
    a.A = A;
    a.ph = phase_nm;
    a.A_norm = A_norm;
    a.n_norm = n_norm;
    a.out = intensity;
    // partial sums: part_I for every realisation, then part_A
    a.part_I = static_cast<float *>(scratch);
    a.part_A = static_cast<float *>(scratch) + (size_t)nb * n_batch;
    a.sA = sA;
    a.sph = sph;
    a.sAn = sAn;
    a.sout = sout;
    a.nbp = nb;
    a.A2 = mirror_A;
    a.ph2 = mirror_phase;
    a.A_out = field_A;
    a.P_out = field_phase;
    a.vec = (a.ld % 4 == 0) && (sA % 4 == 0) && (sph % 4 == 0) && ((uintptr_t)A % 16 == 0) &&
            ((uintptr_t)phase_nm % 16 == 0) && (a.p % 4 == 0);
    grid.z = n_batch;
    cudaStream_t st = sb::as_stream(stream);
    // the compile-time kernel holds per-warp buffers for up to 8 warps
    ShKernel fk = spc <= 8 ? fixed_kernel(a.p, a.cs, a.npx) : nullptr;
    if (tk.fn) {
        if (tk.smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(tk.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tk.smem);
            if (e != cudaSuccess) return sb::fail(SB_ECUDA, "%s: smem attribute: %s", who, cudaGetErrorString(e));
        }
        tk.fn<<<grid, kTcThreads, tk.smem, st>>>(a);
    } else if (fk) {
        // variants 0-2: the field tile staged by TMA where the launch allows it
        // (single field, no mirror term, 16-byte aligned rows); variants 3-5
        // and every other launch read the field directly (the same frames)
        ShTmaKernel fkt = variant < 3 && n_batch == 1 && !mirror_A && a.ld % 4 == 0 && (uintptr_t)A % 16 == 0 &&
                                  (uintptr_t)phase_nm % 16 == 0
                              ? fixed_tma_kernel(a.p, a.cs, a.npx)
                              : nullptr;
        if (fkt) {
            const int field = pl->n_lenses * pl->np_sub;
            CUtensorMap mapA, mapP;
            int rc = sb::tensor_map_2d_f32(&mapA, A, field, field, a.ld, a.p, spc * a.p);
            if (!rc) rc = sb::tensor_map_2d_f32(&mapP, phase_nm, field, field, a.ld, a.p, spc * a.p);
            if (rc) return rc;
            fkt<<<grid, 32 * spc, 0, st>>>(a, mapA, mapP);
        } else {
            fk<<<grid, 32 * spc, 0, st>>>(a);
        }
    } else {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(sh_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return sb::fail(SB_ECUDA, "%s: smem attribute: %s", who, cudaGetErrorString(e));
        }
        sh_forward_kernel<<<grid, 32 * spc, smem, st>>>(a);
    }
    int rc = sb::check_launch("sh_forward_kernel");
    if (rc) return rc;
    if (n_parts) *n_parts = nb;
    if (!normalize) return SB_OK;
    const int n_out = pl->n_lenses * pl->subap_npx * pl->n_lenses * pl->subap_npx;
    int nblk = (n_out + 255) / 256;
    nblk = nblk > 592 ? 592 : nblk;
    sh_normalize_kernel<<<dim3(nblk, n_batch), 256, 0, st>>>(a.part_I, a.part_A, nb, photon_scale, intensity, n_out);
    return sb::check_launch("sh_normalize_kernel");
}

}  // namespace

extern "C" int sb_sh_rows_parts(const sb_sh_plan *pl, int dft_mode) {
    if (!pl || pl->n_lenses < 1) return 0;
    int spc;
    dim3 grid;
    size_t smem;
    if (dft_mode == 1) return ((pl->n_lenses + kTcSub - 1) / kTcSub) * pl->n_lenses;
    const int variant = sb::tune_lookup(SB_TUNE_SH_FP32, sb_tune_key(pl->n_lenses, pl->cutsize, 1));
    if (sh_grid(pl, &spc, &grid, &smem, 8 >> (variant % 3))) return 0;
    return (int)(grid.x * grid.y);
}

extern "C" int sb_sh_forward_rows(const sb_sh_plan *pl, int dft_mode, int row0, int n_rows, const float *A,
                                  const float *phase_nm, const float *A_norm, int n_norm, float *intensity,
                                  void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (dft_mode != 0 && dft_mode != 1) return sb::fail(SB_EINVAL, "sb_sh_forward_rows: dft_mode must be 0 or 1");
    return sh_forward_impl("sb_sh_forward_rows", pl, A, 0, phase_nm, 0, A_norm, 0, n_norm, 1.0f, intensity, 0, 1,
                           scratch, scratch_bytes, stream, dft_mode, false, nullptr, nullptr, nullptr, nullptr,
                           nullptr, row0, n_rows < 0 ? 0 : n_rows);
}

namespace sb {
int sh_forward_unnormalised(const char *who, const sb_sh_plan *pl, const float *A, const float *phase_nm,
                            const float *A_norm, int n_norm, float *intensity, void *scratch, size_t scratch_bytes,
                            void *stream, int mode, int *n_parts, const float *mirror_A, const float *mirror_phase,
                            float *field_A, float *field_phase) {
    return sh_forward_impl(who, pl, A, 0, phase_nm, 0, A_norm, 0, n_norm, 1.0f, intensity, 0, 1, scratch,
                           scratch_bytes, stream, mode, false, n_parts, mirror_A, mirror_phase, field_A, field_phase);
}
}  // namespace sb

extern "C" int sb_sh_forward(const sb_sh_plan *pl, const float *A, const float *phase_nm, const float *A_norm,
                             int n_norm, float photon_scale, float *intensity, void *scratch,
                             size_t scratch_bytes, void *stream) {
    sb::clear_error();
    return sh_forward_impl("sb_sh_forward", pl, A, 0, phase_nm, 0, A_norm, 0, n_norm, photon_scale, intensity, 0, 1,
                           scratch, scratch_bytes, stream);
}

extern "C" int sb_sh_forward_batched(const sb_sh_plan *pl, const float *A, long long A_stride, const float *phase_nm,
                                     long long phase_stride, const float *A_norm, long long A_norm_stride, int n_norm,
                                     float photon_scale, float *intensity, long long intensity_stride, int n_batch,
                                     void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (pl && intensity_stride < (long long)pl->n_lenses * pl->subap_npx * pl->n_lenses * pl->subap_npx)
        return sb::fail(SB_EINVAL, "sb_sh_forward_batched: intensity stride smaller than a frame");
    return sh_forward_impl("sb_sh_forward_batched", pl, A, A_stride, phase_nm, phase_stride, A_norm, A_norm_stride,
                           n_norm, photon_scale, intensity, intensity_stride, n_batch, scratch, scratch_bytes, stream);
}

extern "C" int sb_sh_lgs_supported(const sb_sh_plan *pl, int fft_size) {
    return (pl && lgs_kernel(pl->np_sub, fft_size, pl->cutsize, pl->subap_npx).fn) ? 1 : 0;
}

extern "C" int sb_sh_forward_lgs(const sb_sh_plan *pl, const sb_sh_lgs_tables *lgs, const float *A,
                                 const float *phase_nm, const float *A_norm, int n_norm, float photon_scale,
                                 float *intensity, void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!pl || !lgs || !A || !phase_nm || !A_norm || !intensity || !pl->tilt || !pl->fp_mask || !pl->rebin ||
        !lgs->w_full_t || !lgs->w_dft || !lgs->v_inv_t || !lgs->kernel_spectra)
        return sb::fail(SB_EINVAL, "sb_sh_forward_lgs: null pointer");
    if (pl->n_lenses < 1 || n_norm < 0 || pl->field_ld < pl->n_lenses * pl->np_sub)
        return sb::fail(SB_EINVAL, "sb_sh_forward_lgs: bad geometry");
    const ShLgsEntry ke = lgs_kernel(pl->np_sub, lgs->fft_size, pl->cutsize, pl->subap_npx);
    if (!ke.fn)
        return sb::fail(SB_EUNSUPPORTED, "sb_sh_forward_lgs: no kernel for (np=%d, fft=%d, cut=%d, npx=%d)",
                        pl->np_sub, lgs->fft_size, pl->cutsize, pl->subap_npx);
    const size_t need = sb_sh_scratch_bytes(pl);
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "sb_sh_forward_lgs: scratch needs %zu bytes, got %zu", need, scratch_bytes);
    const dim3 grid((pl->n_lenses + ke.warps - 1) / ke.warps, pl->n_lenses, 1);
    const int nb = grid.x * grid.y;
    ShArgs a = {};
    a.n = pl->n_lenses;
    a.p = pl->np_sub;
    a.cs = pl->cutsize;
    a.npx = pl->subap_npx;
    a.ld = pl->field_ld;
    a.spc = ke.warps;
    a.k = pl->phase_to_rad;
    a.tilt = reinterpret_cast<const float2 *>(pl->tilt);
    a.mask = pl->fp_mask;
    a.rebin = pl->rebin;
    a.A = A;
    a.ph = phase_nm;
    a.A_norm = A_norm;
    a.n_norm = n_norm;
    a.out = intensity;
    a.part_I = static_cast<float *>(scratch);
    a.part_A = static_cast<float *>(scratch) + nb;
    a.nbp = nb;
    LgsArgs g;
    g.wf_t = static_cast<const float2 *>(lgs->w_full_t);
    g.w = static_cast<const float2 *>(lgs->w_dft);
    g.v_t = static_cast<const float2 *>(lgs->v_inv_t);
    g.kspec = static_cast<const float2 *>(lgs->kernel_spectra);
    cudaStream_t st = sb::as_stream(stream);
    if (ke.smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(ke.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ke.smem);
        if (e != cudaSuccess) return sb::fail(SB_ECUDA, "sb_sh_forward_lgs: smem attribute: %s", cudaGetErrorString(e));
    }
    ke.fn<<<grid, 32 * ke.warps, ke.smem, st>>>(a, g);
    int rc = sb::check_launch("sh_forward_lgs_kernel");
    if (rc) return rc;
    const int n_out = pl->n_lenses * pl->subap_npx * pl->n_lenses * pl->subap_npx;
    int nblk = (n_out + 255) / 256;
    nblk = nblk > 592 ? 592 : nblk;
    sh_normalize_kernel<<<dim3(nblk, 1), 256, 0, st>>>(a.part_I, a.part_A, nb, photon_scale, intensity, n_out);
    return sb::check_launch("sh_normalize_kernel");
}

extern "C" int sb_sh_split_bf16_supported(const sb_sh_plan *pl) {
    return (pl && tc_kernel(pl->np_sub, pl->cutsize, pl->subap_npx).fn) ? 1 : 0;
}

extern "C" int sb_sh_forward_split_bf16(const sb_sh_plan *pl, const float *A, const float *phase_nm,
                                        const float *A_norm, int n_norm, float photon_scale, float *intensity,
                                        void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    return sh_forward_impl("sb_sh_forward_split_bf16", pl, A, 0, phase_nm, 0, A_norm, 0, n_norm, photon_scale,
                           intensity, 0, 1, scratch, scratch_bytes, stream, 1);
}

extern "C" int sb_sh_forward_split_bf16_batched(const sb_sh_plan *pl, const float *A, long long A_stride,
                                                const float *phase_nm, long long phase_stride, const float *A_norm,
                                                long long A_norm_stride, int n_norm, float photon_scale,
                                                float *intensity, long long intensity_stride, int n_batch,
                                                void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (pl && intensity_stride < (long long)pl->n_lenses * pl->subap_npx * pl->n_lenses * pl->subap_npx)
        return sb::fail(SB_EINVAL, "sb_sh_forward_split_bf16_batched: intensity stride smaller than a frame");
    return sh_forward_impl("sb_sh_forward_split_bf16_batched", pl, A, A_stride, phase_nm, phase_stride, A_norm,
                           A_norm_stride, n_norm, photon_scale, intensity, intensity_stride, n_batch, scratch,
                           scratch_bytes, stream, 1);
}

// ---------------------------------------------------------------------------
// Monte-Carlo step, stage 4: the SH forward of every realisation of every
// group in one launch, unnormalised, with the per-CTA partial sums that
// sb_sh_forward_batched leaves.  A CTA finds its group, realisation and
// lenslet block from the flat block index and runs that geometry's
// compile-time body (FP32, 8 sub-apertures per CTA) or tensor-core body
// (split-BF16); every group of a plan uses the same DFT form.
// ---------------------------------------------------------------------------
namespace {

struct McShGroup {
    ShArgs a;          // the group's arguments for realisation 0
    int kind, gx, gy;  // geometry index, CTAs per realisation along x / y
};

struct McShArgs {
    int n_groups;
    McShGroup g[sb::kMcMaxGroups];
    int blk0[sb::kMcMaxGroups + 1];
};

struct McShBlob {
    McShArgs args;
    int mode, blocks;
    size_t smem;
};

// geometries (np_sub, cutsize, subap_npx) of the launch over groups; the
// split-BF16 form has the first five
constexpr int kMcShKinds = 6, kMcTcKinds = 5;
constexpr int kMcShGeom[kMcShKinds][3] = {{8, 12, 6}, {8, 14, 8}, {8, 16, 8}, {8, 8, 8}, {8, 12, 8}, {16, 16, 8}};

int mc_sh_kind(int mode, const sb_sh_plan &pl) {
    const int nk = mode == 1 ? kMcTcKinds : kMcShKinds;
    for (int k = 0; k < nk; ++k)
        if (pl.np_sub == kMcShGeom[k][0] && pl.cutsize == kMcShGeom[k][1] && pl.subap_npx == kMcShGeom[k][2])
            return k;
    return -1;
}

size_t mc_fixed_smem(int kind) {
    switch (kind) {
        case 0: return sizeof(FixedSmem<8, 12, 6>);
        case 1: return sizeof(FixedSmem<8, 14, 8>);
        case 2: return sizeof(FixedSmem<8, 16, 8>);
        case 3: return sizeof(FixedSmem<8, 8, 8>);
        case 4: return sizeof(FixedSmem<8, 12, 8>);
        default: return sizeof(FixedSmem<16, 16, 8>);
    }
}

size_t mc_tc_smem(int kind) {
    switch (kind) {
        case 0: return tc_smem_bytes<8, 12, 6>();
        case 1: return tc_smem_bytes<8, 14, 8>();
        case 2: return tc_smem_bytes<8, 16, 8>();
        case 3: return tc_smem_bytes<8, 8, 8>();
        default: return tc_smem_bytes<8, 12, 8>();
    }
}

__device__ __forceinline__ int mc_sh_locate(const McShArgs &m, ShArgs &a, ShBlk &blk) {
    const int bi = blockIdx.x;
    int g = 0;
    while (g + 1 < m.n_groups && bi >= m.blk0[g + 1]) ++g;
    const McShGroup &G = m.g[g];
    const int per = G.gx * G.gy, local = bi - m.blk0[g];
    const int b = local / per, rem = local - b * per;
    a = G.a;
    slice_to(a, b);
    blk = {rem % G.gx, rem / G.gx, G.gx, G.gy};
    return G.kind;
}

__global__ void __launch_bounds__(256, 4) mc_sh_fixed_kernel(McShArgs m) {
    extern __shared__ __align__(16) unsigned char mc_sh_smem[];
    ShArgs a;
    ShBlk blk;
    switch (mc_sh_locate(m, a, blk)) {
        case 0: sh_fixed_body<8, 12, 6>(a, blk, *reinterpret_cast<FixedSmem<8, 12, 6> *>(mc_sh_smem)); break;
        case 1: sh_fixed_body<8, 14, 8>(a, blk, *reinterpret_cast<FixedSmem<8, 14, 8> *>(mc_sh_smem)); break;
        case 2: sh_fixed_body<8, 16, 8>(a, blk, *reinterpret_cast<FixedSmem<8, 16, 8> *>(mc_sh_smem)); break;
        case 3: sh_fixed_body<8, 8, 8>(a, blk, *reinterpret_cast<FixedSmem<8, 8, 8> *>(mc_sh_smem)); break;
        case 4: sh_fixed_body<8, 12, 8>(a, blk, *reinterpret_cast<FixedSmem<8, 12, 8> *>(mc_sh_smem)); break;
        default: sh_fixed_body<16, 16, 8>(a, blk, *reinterpret_cast<FixedSmem<16, 16, 8> *>(mc_sh_smem)); break;
    }
}

__global__ void __launch_bounds__(kTcThreads) mc_sh_tc_kernel(McShArgs m) {
    ShArgs a;
    ShBlk blk;
    switch (mc_sh_locate(m, a, blk)) {
        case 0: sh_tc_body<8, 12, 6>(a, blk); break;
        case 1: sh_tc_body<8, 14, 8>(a, blk); break;
        case 2: sh_tc_body<8, 16, 8>(a, blk); break;
        case 3: sh_tc_body<8, 8, 8>(a, blk); break;
        default: sh_tc_body<8, 12, 8>(a, blk); break;
    }
}

// CTAs per realisation of a group
void mc_sh_grid(int mode, const sb_sh_plan &pl, int *gx, int *gy) {
    const int per = mode == 1 ? kTcSub : 8;
    *gx = (pl.n_lenses + per - 1) / per;
    *gy = pl.n_lenses;
}

}  // namespace

namespace sb {

size_t mc_sh_workspace(const sb_mc_group *gs, int n) {
    size_t b = 0;
    for (int g = 0; g < n; ++g) {
        int gx, gy;
        mc_sh_grid(gs[g].dft_mode, gs[g].sh, &gx, &gy);
        b += mc_align(2 * (size_t)gx * gy * gs[g].n_batch * sizeof(float));
    }
    return b;
}

int mc_sh_prepare(const sb_mc_group *gs, int n, void *ws, McBlob &blob, McShParts &parts) {
    static_assert(sizeof(McShBlob) <= sizeof(McBlob), "SH stage arguments exceed the blob");
    static_assert(sizeof(McShArgs) <= 4096, "kernel arguments above 4 KB");
    const char *who = "sb_mc_create";
    McShBlob *B = new (blob.b) McShBlob();
    const int mode = gs[0].dft_mode;
    if (mode != 0 && mode != 1) return fail(SB_EINVAL, "%s: dft_mode must be 0 or 1", who);
    B->mode = mode;
    B->args.n_groups = n;
    unsigned char *w = static_cast<unsigned char *>(ws);
    int blocks = 0;
    size_t smem = 0;
    for (int g = 0; g < n; ++g) {
        const sb_mc_group &G = gs[g];
        const sb_sh_plan &pl = G.sh;
        if (G.dft_mode != mode) return fail(SB_EINVAL, "%s: every group must use the same dft_mode", who);
        if (!pl.twiddle || !pl.tilt || !pl.fp_mask || !pl.rebin || !G.intensity || !G.field_A || !G.field_phase)
            return fail(SB_EINVAL, "%s: group %d: null SH pointer", who, g);
        if (pl.n_lenses < 1 || pl.field_ld != G.L || pl.n_lenses * pl.np_sub > G.L)
            return fail(SB_EINVAL, "%s: group %d: SH field of %d columns on a %d pupil", who, g, pl.field_ld, G.L);
        const int kind = mc_sh_kind(mode, pl);
        if (kind < 0)
            return fail(SB_EUNSUPPORTED, "%s: group %d: no %s kernel for (np=%d, cut=%d, npx=%d)", who, g,
                        mode ? "split-BF16" : "compile-time", pl.np_sub, pl.cutsize, pl.subap_npx);
        const long long side = (long long)pl.n_lenses * pl.subap_npx;
        if (G.frame_stride < side * side) return fail(SB_EINVAL, "%s: group %d: frame stride below a frame", who, g);
        int gx, gy;
        mc_sh_grid(mode, pl, &gx, &gy);
        const int nb = gx * gy;
        McShGroup &q = B->args.g[g];
        ShArgs &a = q.a;
        a = ShArgs{};
        a.n = pl.n_lenses;
        a.p = pl.np_sub;
        a.cs = pl.cutsize;
        a.npx = pl.subap_npx;
        a.ld = pl.field_ld;
        a.spc = 8;
        a.k = pl.phase_to_rad;
        a.tw = reinterpret_cast<const float2 *>(pl.twiddle);
        a.tilt = reinterpret_cast<const float2 *>(pl.tilt);
        a.mask = pl.fp_mask;
        a.rebin = pl.rebin;
        a.A = G.field_A;
        a.ph = G.field_phase;
        a.A_norm = G.field_A;                   // the normalising amplitude is the whole field
        a.n_norm = G.L * G.L;
        a.out = G.intensity;
        float *part = reinterpret_cast<float *>(w);
        a.part_I = part;
        a.part_A = part + (size_t)nb * G.n_batch;
        a.sA = a.sph = a.sAn = G.field_stride;
        a.sout = G.frame_stride;
        a.nbp = nb;
        a.vec = (a.ld % 4 == 0) && (a.sA % 4 == 0) && ((uintptr_t)a.A % 16 == 0) && ((uintptr_t)a.ph % 16 == 0) &&
                (a.p % 4 == 0);
        q.kind = kind;
        q.gx = gx;
        q.gy = gy;
        parts.part_I[g] = a.part_I;
        parts.part_A[g] = a.part_A;
        parts.nparts[g] = nb;
        B->args.blk0[g] = blocks;
        blocks += nb * G.n_batch;
        const size_t sm = mode == 1 ? mc_tc_smem(kind) : mc_fixed_smem(kind);
        smem = sm > smem ? sm : smem;
        w += mc_align(2 * (size_t)nb * G.n_batch * sizeof(float));
    }
    B->args.blk0[n] = blocks;
    B->blocks = blocks;
    B->smem = smem;
    const cudaError_t e = cudaFuncSetAttribute(mode == 1 ? (const void *)mc_sh_tc_kernel : (const void *)mc_sh_fixed_kernel,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail(SB_ECUDA, "%s: SH shared memory: %s", who, cudaGetErrorString(e));
    return SB_OK;
}

int mc_sh_launch(const McBlob &blob, cudaStream_t st) {
    const McShBlob *B = reinterpret_cast<const McShBlob *>(blob.b);
    if (B->mode == 1) {
        mc_sh_tc_kernel<<<B->blocks, kTcThreads, B->smem, st>>>(B->args);
        return check_launch("mc_sh_tc_kernel");
    }
    mc_sh_fixed_kernel<<<B->blocks, 256, B->smem, st>>>(B->args);
    return check_launch("mc_sh_fixed_kernel");
}

}  // namespace sb

namespace sb {
// read and clear the tensor-core SH timeout flag (0: none)
int sh_tc_status_take() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_sh_tc_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_sh_tc_status, &zero, sizeof(int));
    }
    return v;
}
}  // namespace sb

extern "C" int sb_edge_extrapolate(const float *phase, const int32_t *src1, const int32_t *src2, int n_pixels,
                                   float *out, void *stream) {
    sb::clear_error();
    if (!phase || !src1 || !src2 || !out || n_pixels < 0) return sb::fail(SB_EINVAL, "sb_edge_extrapolate: bad args");
    if (n_pixels == 0) return SB_OK;
    int nblk = (n_pixels + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    edge_extrapolate_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(phase, src1, src2, n_pixels, out);
    return sb::check_launch("edge_extrapolate_kernel");
}

extern "C" int sb_interp2d_field(const float *A_in, const float *phase_in, int in_rows, int in_cols,
                                 const float *yy, const float *xx, int n_out, float *A_out, float *phase_out,
                                 void *stream) {
    sb::clear_error();
    if (!A_in || !phase_in || !yy || !xx || !A_out || !phase_out || n_out < 0)
        return sb::fail(SB_EINVAL, "sb_interp2d_field: bad args");
    if (in_rows < 2 || in_cols < 2) return sb::fail(SB_ESHAPE, "sb_interp2d_field: input must be at least 2x2");
    if (n_out == 0) return SB_OK;
    int nblk = (n_out + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    interp2d_field_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(A_in, phase_in, in_rows, in_cols, yy, xx, n_out,
                                                                    A_out, phase_out);
    return sb::check_launch("interp2d_field_kernel");
}

// ---------------------------------------------------------------------------
// No-allocation variant of sb_sh_forward: the partial sums live in a
// file-scope device array instead of caller scratch.  Host code must not
// pass the array's name to a kernel (on the host it is only a stand-in for
// the symbol); its device address is looked up once per device with
// cudaGetSymbolAddress while that device is current.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {
static __device__ __align__(256) unsigned char g_sh_static_scratch[SB_SH_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_static_mutex;
void *g_static_ptr[kMaxDevices] = {};

int static_scratch_address(void **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sb::fail(SB_ECUDA, "sb_sh_forward_static: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return sb::fail(SB_EUNSUPPORTED, "sb_sh_forward_static: device %d", dev);
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (!g_static_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sh_static_scratch);
        if (e != cudaSuccess || !p)
            return sb::fail(SB_ECUDA, "sb_sh_forward_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_static_ptr[dev] = p;
    }
    *out = g_static_ptr[dev];
    return SB_OK;
}
}  // namespace

extern "C" int sb_sh_forward_static(const sb_sh_plan *pl, const float *A, const float *phase_nm, const float *A_norm,
                                    int n_norm, float photon_scale, float *intensity, void *stream) {
    sb::clear_error();
    if (!pl) return sb::fail(SB_EINVAL, "sb_sh_forward_static: null plan");
    const size_t need = sb_sh_scratch_bytes(pl);
    if (need == 0) return sb::fail(SB_ESHAPE, "sb_sh_forward_static: geometry does not fit the kernel limits");
    if (need > (size_t)SB_SH_STATIC_SCRATCH_BYTES)
        return sb::fail(SB_ESCRATCH,
                        "sb_sh_forward_static: this geometry needs %zu bytes of scratch, the static array holds %d; "
                        "use sb_sh_forward with caller scratch",
                        need, SB_SH_STATIC_SCRATCH_BYTES);
    void *scratch = nullptr;
    const int rc = static_scratch_address(&scratch);
    if (rc) return rc;
    return sb_sh_forward(pl, A, phase_nm, A_norm, n_norm, photon_scale, intensity, scratch,
                         (size_t)SB_SH_STATIC_SCRATCH_BYTES, stream);
}
