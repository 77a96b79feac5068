// PSF image on the fifth-generation tensor cores (specula/processing_objects/
// psf.py:56-96: |fftshift(fft2(zero-padded field))|^2 normalised to unit sum).
//
// F = W u W^T, u = A e^{i phi} (M x M), W the N x M DFT matrix restricted to
// the field's M inputs with its rows in fftshift order; the padding to N x N
// never materialises.  Both products run as real GEMMs D = A_op * B_op^T on
// tcgen05 (BF16 operands, FP32 accumulation in tensor memory), each FP32
// operand split as hi + lo bf16 and each product taken as hi*hi + lo*hi +
// hi*lo (three MMAs; relative error of order 2^-16 per operand):
//
//   A_op (both stages)  rows q < N:  [Re W(q, .) | Im W(q, .)]          K = 2M
//   stage 1  B_op rows (Re x, Im x): [Re u(x,.) | -Im u(x,.)], [Im u | Re u]
//            D1(q, Re x) + i D1(q, Im x) = sum_y W(q, y) u(x, y) = G(x, q)
//   stage 2  B_op rows (Re q, Im q): [Re G(., q) | -Im G(., q)], [Im G | Re G]
//            D2(p, Re q) + i D2(p, Im q) = sum_x W(p, x) G(x, q) = F(p, q)
//
// Every operand is stored pre-tiled in the no-swizzle K-major layout the MMA
// reads (tiles of R rows x 32 K; within a tile the two K=16 steps, within a
// step the two 8-wide K segments, within a segment row r at r * 16 bytes), so
// a pipeline stage is four contiguous bulk copies.  The DFT operand is built
// once; the field kernel writes stage 1's B_op, stage 1's epilogue writes
// stage 2's B_op, stage 2's epilogue writes |F|^2 / total with total =
// N^2 sum |u|^2 (Parseval: the sum of the padded transform's power) and adds
// it to the integrated PSF.  M and N are padded to multiples of 128 with
// zeros.  One CTA of 128 threads per output tile of 128 rows x 64 complex
// columns: lane 0 of warp 0 issues the copies into a 6-stage ring, lane 0 of
// warp 1 the MMAs (tensor memory: 4 x 128 FP32 columns), all four warps the
// epilogue; the hi*hi products of each third of K and the hi*lo + lo*hi
// corrections accumulate in separate tensor-memory regions.  Every mbarrier wait is bounded; a timeout is recorded in
// g_psf_tc_status (read by sb_device_status) and leaves the outputs unwritten.
#include "sb_common.cuh"
#include "sb_umma.cuh"

namespace {

constexpr int kTM = 128;                       // A_op rows per tile
constexpr int kTN = 128;                       // B_op rows per tile: kCC complex columns as Re, Im
constexpr int kCC = kTN / 2;                   // complex columns per tile
constexpr int kBK = 32;                        // K per stage: two K=16 MMA steps
constexpr int kStages = 6;
constexpr int kATile = kTM * kBK * 2;          // bytes of one A_op tile (bf16)
constexpr int kBTile = kTN * kBK * 2;
constexpr int kStageBytes = 2 * kATile + 2 * kBTile;    // hi and lo of both operands
// four accumulators of kTN FP32 columns: the hi*hi products of the first,
// second and last third of K in regions 0-2, the hi*lo and lo*hi corrections
// in region 3.  The tensor cores add each product into the accumulator with a
// truncating rounding whose bias grows with the number of additions into one
// accumulator (measured at the 640 px / nd 8 PSF: 2.0e-5 of the peak with one
// accumulator, 9e-6 with the corrections apart); the regions are added with
// round-to-nearest in the epilogue.
constexpr int kRegions = 4;
constexpr uint32_t kTmemCols = kRegions * kTN;
constexpr int kThreads = 128;
constexpr int kFieldThreads = 256;
constexpr int kFieldMaxBlocks = 592;

__device__ int g_psf_tc_status = 0;

__host__ __device__ inline int pad128(int v) { return (v + 127) / 128 * 128; }

// byte offset of (row r, column k) in a pre-tiled K-major bf16 operand of
// R-row tiles and `kblocks` tiles along K
__device__ __forceinline__ size_t tiled_offset(int r, int k, int R, int kblocks) {
    const int tile = (r / R) * kblocks + k / kBK;
    const int kk = k % kBK;
    return (size_t)tile * R * kBK * 2 + (size_t)(kk / 16) * (2 * R * 16) + (size_t)((kk % 16) / 8) * (R * 16) +
           (size_t)(r % R) * 16;
}

// 8 consecutive K values (k0 a multiple of 8) of row r, split into hi and lo
__device__ __forceinline__ void store_split8(unsigned char *hi, unsigned char *lo, int r, int k0, int R, int kblocks,
                                             const float (&v)[8]) {
    uint4 h, l;
    sb::split_bf16x8(v, h, l);
    const size_t off = tiled_offset(r, k0, R, kblocks);
    *reinterpret_cast<uint4 *>(hi + off) = h;
    *reinterpret_cast<uint4 *>(lo + off) = l;
}

// the DFT operand: row q < n, K index k < 2 mp: Re W(q, k) for k < mp, Im W(q, k - mp) after;
// W(q, y) = exp(-2 pi i kq y / n), kq = (q - n/2) mod n, zero for y >= m or q >= n
__global__ void __launch_bounds__(256) psf_tc_dft_kernel(int m, int n, int mp, int np_, unsigned char *hi,
                                                         unsigned char *lo) {
    const int kblocks = 2 * mp / kBK;
    const long long groups = (long long)np_ * (2 * mp / 8);
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < groups;
         g += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(g / (2 * mp / 8));
        const int k0 = (int)(g % (2 * mp / 8)) * 8;
        const bool imag = k0 >= mp;
        const int y0 = imag ? k0 - mp : k0;
        const long long kq = ((long long)q - n / 2 + n) % n;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int y = y0 + j;
            float w = 0.f;
            if (q < n && y < m) {
                // phase -2 pi r / n with r = kq * y mod n: cos and -sin of 2 pi r / n
                const long long r = (kq * y) % n;
                const double t = 2.0 * (double)r / (double)n;
                w = imag ? (float)(-sinpi(t)) : (float)cospi(t);
            }
            v[j] = w;
        }
        store_split8(hi, lo, q, k0, kTM, kblocks, v);
    }
}

__device__ __forceinline__ float2 field_at(const float *A, const float *ph, int e, float k) {
    const float phi = __fmul_rn(ph[e], k);      // phaseInNm * (2 pi / lambda) in float32
    float s, c;
    sincosf(phi, &s, &c);
    const float a = A[e];
    return make_float2(__fmul_rn(a, c), __fmul_rn(a, s));
}

// stage 1's B_op from the field, and total = n^2 sum |u|^2 (float64, fixed
// order: per-block partials, the last block sums them)
__global__ void __launch_bounds__(kFieldThreads) psf_tc_field_kernel(const float *__restrict__ A,
                                                                    const float *__restrict__ ph, int m, int mp, int n,
                                                                    float k, unsigned char *hi, unsigned char *lo,
                                                                    double *part, unsigned int *counter,
                                                                    double *total) {
    __shared__ double red[33];
    __shared__ bool last;
    const int kblocks = 2 * mp / kBK;
    const int gpr = 2 * mp / 8;                       // 8-wide K groups per row
    const long long groups = (long long)(2 * mp) * gpr;
    double acc = 0.0;
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < groups;
         g += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(g / gpr);
        const int k0 = (int)(g % gpr) * 8;
        const int x = (row / kTN) * kCC + (row % kTN) % kCC;
        const bool im_row = (row % kTN) >= kCC;
        const bool second = k0 >= mp;
        const int y0 = second ? k0 - mp : k0;
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int y = y0 + j;
            float2 u = make_float2(0.f, 0.f);
            if (x < m && y < m) u = field_at(A, ph, x * m + y, k);
            v[j] = im_row ? (second ? u.x : u.y) : (second ? -u.y : u.x);
            if (!im_row && !second) acc += (double)u.x * u.x + (double)u.y * u.y;
        }
        store_split8(hi, lo, row, k0, kTN, kblocks, v);
    }
    acc = sb::block_sum_all_d(acc, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = acc;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += __ldcg(part + b);
    t = sb::block_sum_all_d(t, red);
    if (threadIdx.x == 0) {
        *total = t * (double)n * (double)n;
        *counter = 0u;
    }
}

struct GemmArgs {
    const unsigned char *a_hi, *a_lo;    // the DFT operand
    const unsigned char *b_hi, *b_lo;    // this stage's B_op
    int kblocks;                         // K tiles (2 mp / 32)
    // stage 1: stage 2's B_op
    unsigned char *g_hi, *g_lo;
    int g_kblocks, mp;
    // stage 2: the PSF
    float *psf, *int_psf;
    const double *total;
    int n;
};

template <int STAGE>
__global__ void __launch_bounds__(kThreads, 1) psf_tc_gemm_kernel(GemmArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *ring = smem_raw + ((1024 - (sb::smem_u32(smem_raw) & 1023)) & 1023);
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)kStages * kStageBytes);
    uint64_t *empty = full + kStages;
    uint64_t *done = empty + kStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    __shared__ int abort_flag, issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nb = blockIdx.x, rb = blockIdx.y;
    if (warp == 0) {
        sb::tmem_alloc(tmem_slot, kTmemCols);
        sb::tmem_relinquish();
    }
    if (tid == 32) {
        for (int s = 0; s < kStages; ++s) {
            sb::mbar_init(&full[s], 1);
            sb::mbar_init(&empty[s], 1);
        }
        sb::mbar_init(done, 1);
        sb::mbar_init_fence();
        abort_flag = 0;
        issued = 0;
    }
    sb::tc_fence_before_sync();
    __syncthreads();
    sb::tc_fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const int KB = a.kblocks;
    if (tid == 0) {
        // producer: four contiguous copies per stage; every tile is read by many
        // CTAs (the DFT operand by all of a stage, B_op by a column of them), so
        // its lines are kept in L2
        const uint64_t pol = sb::l2_evict_last_policy();
        const unsigned char *ah = a.a_hi + (size_t)rb * KB * kATile, *al = a.a_lo + (size_t)rb * KB * kATile;
        const unsigned char *bh = a.b_hi + (size_t)nb * KB * kBTile, *bl = a.b_lo + (size_t)nb * KB * kBTile;
        int kb = 0;
        for (; kb < KB; ++kb) {
            const int s = kb % kStages;
            if (kb >= kStages && !sb::mbar_wait(&empty[s], ((kb / kStages) - 1) & 1)) {
                atomicExch(&g_psf_tc_status, 1);
                abort_flag = 1;
                break;
            }
            if (*(volatile int *)&abort_flag) break;
            unsigned char *st = ring + (size_t)s * kStageBytes;
            sb::mbar_arrive_expect_tx(&full[s], kStageBytes);
            sb::bulk_load_1d(st, ah + (size_t)kb * kATile, kATile, &full[s], pol);
            sb::bulk_load_1d(st + kATile, al + (size_t)kb * kATile, kATile, &full[s], pol);
            sb::bulk_load_1d(st + 2 * kATile, bh + (size_t)kb * kBTile, kBTile, &full[s], pol);
            sb::bulk_load_1d(st + 2 * kATile + kBTile, bl + (size_t)kb * kBTile, kBTile, &full[s], pol);
        }
        issued = kb;
    } else if (tid == 32) {
        // MMA issuer: per stage two K steps of three products each
        constexpr uint32_t IDESC = sb::umma_idesc_bf16_f32(kTM, kTN);
        for (int kb = 0; kb < KB; ++kb) {
            const int s = kb % kStages;
            if (!sb::mbar_wait(&full[s], (kb / kStages) & 1)) {
                atomicExch(&g_psf_tc_status, 2);
                abort_flag = 1;
                break;
            }
            sb::tc_fence_after_sync();
            const unsigned char *st = ring + (size_t)s * kStageBytes;
            // region of this K block's hi*hi products: thirds of K
            const int reg = (kb * 3) / KB, reg_first = (reg * KB + 2) / 3;
            const uint32_t dm = tmem + (uint32_t)(reg * kTN), dc = tmem + (uint32_t)(3 * kTN);
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const uint64_t dah = sb::umma_desc_kmajor(st + ks * (2 * kTM * 16), kTM * 16);
                const uint64_t dal = sb::umma_desc_kmajor(st + kATile + ks * (2 * kTM * 16), kTM * 16);
                const uint64_t dbh = sb::umma_desc_kmajor(st + 2 * kATile + ks * (2 * kTN * 16), kTN * 16);
                const uint64_t dbl = sb::umma_desc_kmajor(st + 2 * kATile + kBTile + ks * (2 * kTN * 16), kTN * 16);
                sb::umma_bf16(dm, dah, dbh, IDESC, (kb != reg_first || ks != 0) ? 1u : 0u);
                sb::umma_bf16(dc, dal, dbh, IDESC, (kb | ks) != 0 ? 1u : 0u);
                sb::umma_bf16(dc, dah, dbl, IDESC, 1u);
            }
            sb::umma_commit(&empty[s]);
        }
        // completes once every MMA issued above has finished
        sb::umma_commit(done);
    }
    __syncwarp();
    const bool ok = sb::mbar_wait(done, 0);
    if (!ok && lane == 0) atomicExch(&g_psf_tc_status, 3);
    const bool write = __syncthreads_and(ok) && !*(volatile int *)&abort_flag;
    sb::tc_fence_after_sync();
    if (write) {
        const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
        const int row = rb * kTM + warp * 32 + lane;     // q (stage 1) or p (stage 2)
#pragma unroll 1
        for (int c = 0; c < kCC / 16; ++c) {
            // F = ((M0 + M1) + M2) + C, real parts in a region's first kCC columns, imaginary after
            uint32_t re[16], im[16];
            sb::tmem_ld16(tl + 16 * c, re);
            sb::tmem_ld16(tl + kCC + 16 * c, im);
            sb::tmem_wait_ld(re);
            sb::tmem_wait_ld(im);
#pragma unroll 1
            for (int r = 1; r < kRegions; ++r) {
                uint32_t rr[16], ri[16];
                sb::tmem_ld16(tl + r * kTN + 16 * c, rr);
                sb::tmem_ld16(tl + r * kTN + kCC + 16 * c, ri);
                sb::tmem_wait_ld(rr);
                sb::tmem_wait_ld(ri);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    re[j] = __float_as_uint(__fadd_rn(__uint_as_float(re[j]), __uint_as_float(rr[j])));
                    im[j] = __float_as_uint(__fadd_rn(__uint_as_float(im[j]), __uint_as_float(ri[j])));
                }
            }
            const int col0 = nb * kCC + 16 * c;          // x (stage 1) or q (stage 2)
            if constexpr (STAGE == 1) {
                // G(x, q) for x = col0 .. col0 + 15 of row q: stage 2's B_op rows Re q and Im q
                const int n_re = (row / kCC) * kTN + row % kCC, n_im = n_re + kCC;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    float gr[8], gi[8], ngi[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        gr[j] = __uint_as_float(re[8 * h + j]);
                        gi[j] = __uint_as_float(im[8 * h + j]);
                        ngi[j] = -gi[j];
                    }
                    const int x0 = col0 + 8 * h;
                    store_split8(a.g_hi, a.g_lo, n_re, x0, kTN, a.g_kblocks, gr);
                    store_split8(a.g_hi, a.g_lo, n_re, a.mp + x0, kTN, a.g_kblocks, ngi);
                    store_split8(a.g_hi, a.g_lo, n_im, x0, kTN, a.g_kblocks, gi);
                    store_split8(a.g_hi, a.g_lo, n_im, a.mp + x0, kTN, a.g_kblocks, gr);
                }
            } else {
                if (row < a.n) {
                    const float total = (float)*a.total;
                    float *out = a.psf + (size_t)row * a.n;
                    float *acc = a.int_psf ? a.int_psf + (size_t)row * a.n : nullptr;
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int q = col0 + j;
                        if (q < a.n) {
                            const float fr = __uint_as_float(re[j]), fi = __uint_as_float(im[j]);
                            const float v = __fdiv_rn(__fadd_rn(__fmul_rn(fr, fr), __fmul_rn(fi, fi)), total);
                            out[q] = v;
                            if (acc) acc[q] = __fadd_rn(acc[q], v);      // psf.py:126-137
                        }
                    }
                }
            }
        }
    }
    sb::tc_fence_before_sync();
    __syncthreads();
    if (*(volatile int *)&abort_flag) {
        // let the MMAs and copies still in flight finish before the memory is released
        if (tid == 0)
            for (int q = issued > kStages ? issued - kStages : 0; q < issued; ++q)
                sb::mbar_wait(&full[q % kStages], (q / kStages) & 1);
        if (tid == 32) sb::mbar_wait(done, 0);
        __syncthreads();
    }
    if (warp == 0) {
        sb::tc_fence_after_sync();
        sb::tmem_dealloc(tmem, kTmemCols);
    }
}

constexpr size_t kGemmSmem = 1024 + (size_t)kStages * kStageBytes + (2 * kStages + 1) * 8 + 16;

size_t dft_half_bytes(int m, int n) { return (size_t)pad128(n) * 2 * pad128(m) * 2; }
size_t b1_half_bytes(int m) { return (size_t)2 * pad128(m) * 2 * pad128(m) * 2; }
size_t b2_half_bytes(int m, int n) { return (size_t)2 * pad128(n) * 2 * pad128(m) * 2; }
size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

namespace sb {
// read and clear the timeout flag of the tensor-core PSF (0: none, <0: query failed)
int psf_tc_status_take() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_psf_tc_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_psf_tc_status, &zero, sizeof(int));
    }
    return v;
}
}  // namespace sb

extern "C" size_t sb_psf_tc_dft_bytes(int m, int n) {
    if (m < 1 || n < m) return 0;
    return 2 * align256(dft_half_bytes(m, n));
}

extern "C" int sb_psf_tc_prepare(int m, int n, void *dft, size_t dft_bytes, void *stream) {
    sb::clear_error();
    if (m < 1 || n < m || !dft) return sb::fail(SB_EINVAL, "sb_psf_tc_prepare: bad args");
    if (dft_bytes < sb_psf_tc_dft_bytes(m, n))
        return sb::fail(SB_ESCRATCH, "sb_psf_tc_prepare: the DFT operand needs %zu bytes", sb_psf_tc_dft_bytes(m, n));
    if ((uintptr_t)dft % 256) return sb::fail(SB_EINVAL, "sb_psf_tc_prepare: the DFT operand must be 256-byte aligned");
    unsigned char *hi = static_cast<unsigned char *>(dft);
    unsigned char *lo = hi + align256(dft_half_bytes(m, n));
    const int mp = pad128(m), np_ = pad128(n);
    const long long groups = (long long)np_ * (2 * mp / 8);
    int nb = (int)((groups + 255) / 256);
    nb = nb > 1184 ? 1184 : nb;
    psf_tc_dft_kernel<<<nb, 256, 0, sb::as_stream(stream)>>>(m, n, mp, np_, hi, lo);
    return sb::check_launch("psf_tc_dft_kernel");
}

extern "C" size_t sb_psf_tc_scratch_bytes(int m, int n) {
    if (m < 1 || n < m) return 0;
    return 2 * align256(b1_half_bytes(m)) + 2 * align256(b2_half_bytes(m, n)) +
           align256((size_t)kFieldMaxBlocks * sizeof(double) + 16 + sizeof(double));
}

extern "C" int sb_psf_tc(const float *A, const float *phase_nm, int m, int n, float phase_to_rad, const void *dft,
                         float *psf, float *int_psf, void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!A || !phase_nm || !dft || !psf || m < 1 || n < m) return sb::fail(SB_EINVAL, "sb_psf_tc: bad args");
    const size_t need = sb_psf_tc_scratch_bytes(m, n);
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "sb_psf_tc: scratch needs %zu bytes, got %zu", need, scratch_bytes);
    if ((uintptr_t)scratch % 256 || (uintptr_t)dft % 256)
        return sb::fail(SB_EINVAL, "sb_psf_tc: scratch and DFT operand must be 256-byte aligned");
    const int mp = pad128(m), np_ = pad128(n);
    unsigned char *s = static_cast<unsigned char *>(scratch);
    unsigned char *b1_hi = s, *b1_lo = b1_hi + align256(b1_half_bytes(m));
    unsigned char *b2_hi = b1_lo + align256(b1_half_bytes(m));
    unsigned char *b2_lo = b2_hi + align256(b2_half_bytes(m, n));
    double *part = reinterpret_cast<double *>(b2_lo + align256(b2_half_bytes(m, n)));
    unsigned int *counter = reinterpret_cast<unsigned int *>(part + kFieldMaxBlocks);
    double *total = reinterpret_cast<double *>(part + kFieldMaxBlocks + 2);
    const unsigned char *w_hi = static_cast<const unsigned char *>(dft);
    const unsigned char *w_lo = w_hi + align256(dft_half_bytes(m, n));
    cudaStream_t st = sb::as_stream(stream);

    const long long groups = (long long)(2 * mp) * (2 * mp / 8);
    int nbf = (int)((groups + kFieldThreads - 1) / kFieldThreads);
    nbf = nbf > kFieldMaxBlocks ? kFieldMaxBlocks : nbf;
    psf_tc_field_kernel<<<nbf, kFieldThreads, 0, st>>>(A, phase_nm, m, mp, n, phase_to_rad, b1_hi, b1_lo, part, counter,
                                                      total);
    int rc = sb::check_launch("psf_tc_field_kernel");
    if (rc) return rc;
    cudaError_t e1 = cudaFuncSetAttribute(psf_tc_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kGemmSmem);
    cudaError_t e2 = cudaFuncSetAttribute(psf_tc_gemm_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kGemmSmem);
    if (e1 != cudaSuccess || e2 != cudaSuccess)
        return sb::fail(SB_ECUDA, "sb_psf_tc: smem attribute: %s", cudaGetErrorString(e1 ? e1 : e2));
    const int kblocks = 2 * mp / kBK;
    GemmArgs g = {};
    g.a_hi = w_hi;
    g.a_lo = w_lo;
    g.kblocks = kblocks;
    g.mp = mp;
    g.n = n;
    // stage 1: G^T = W u^T as (q rows) x (x columns), written as stage 2's B_op
    g.b_hi = b1_hi;
    g.b_lo = b1_lo;
    g.g_hi = b2_hi;
    g.g_lo = b2_lo;
    g.g_kblocks = kblocks;
    psf_tc_gemm_kernel<1><<<dim3(mp / kCC, np_ / kTM), kThreads, kGemmSmem, st>>>(g);
    rc = sb::check_launch("psf_tc_gemm_kernel<1>");
    if (rc) return rc;
    // stage 2: F = W G, |F|^2 / total into the PSF (and the integrated PSF)
    g.b_hi = b2_hi;
    g.b_lo = b2_lo;
    g.g_hi = g.g_lo = nullptr;
    g.psf = psf;
    g.int_psf = int_psf;
    g.total = total;
    psf_tc_gemm_kernel<2><<<dim3(np_ / kCC, np_ / kTM), kThreads, kGemmSmem, st>>>(g);
    return sb::check_launch("psf_tc_gemm_kernel<2>");
}
