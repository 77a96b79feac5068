// PSF and Strehl ratio of an electric field on the B200
// (specula/processing_objects/psf.py:17-137).
//
// Strehl ratio.  The reference takes the centre pixel of the normalised,
// fftshift-ed PSF of the zero-padded field over that of the flat-phase
// reference PSF (psf.py:111-124).  The centre pixel is the zero-frequency
// term |sum_x u(x)|^2 and, by Parseval, both normalisations equal
// N^2 * sum A^2, so SR = |sum A e^{i phi}|^2 / (sum A)^2 exactly: one fused
// reduction over the pupil (float32 field values as the reference's
// complex64 exp produces them, float64 accumulation), no FFT.
//
// PSF image.  u = A e^{i phi} (M x M, complex64) is transformed by the
// caller as two complex GEMMs with the pruned DFT matrix whose rows are in
// fftshift order (the zero padding to N x N never materialises); this file
// supplies the field build and the epilogue |F|^2 / sum(|F|^2), optionally
// accumulated into the integrated PSF.
#include "sb_common.cuh"

namespace {

constexpr int kPsfThreads = 256;
constexpr int kPsfMaxBlocks = 592;     // 4 per SM

__device__ __forceinline__ float2 field_value(const float *A, const float *ph, int e, float k) {
    const float phi = __fmul_rn(ph[e], k);   // phaseInNm * (2 pi / lambda) in float32
    float s, c;
    sincosf(phi, &s, &c);
    const float a = A[e];
    return make_float2(__fmul_rn(a, c), __fmul_rn(a, s));
}

// partial sums of (Re u, Im u, A) per block; the last block to finish
// reduces them in a fixed order and writes SR (and the running integral)
__global__ void __launch_bounds__(kPsfThreads) strehl_kernel(const float *__restrict__ A,
                                                            const float *__restrict__ ph, int n, float k,
                                                            double *__restrict__ part, unsigned int *counter,
                                                            float *__restrict__ sr, double *int_sr, int integrate) {
    __shared__ double red[33];
    __shared__ bool last;
    double sc = 0.0, ss = 0.0, sa = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const float2 u = field_value(A, ph, e, k);
        sc += u.x;
        ss += u.y;
        sa += A[e];
    }
    sc = sb::block_sum_all_d(sc, red);
    ss = sb::block_sum_all_d(ss, red);
    sa = sb::block_sum_all_d(sa, red);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x + 0] = sc;
        part[3 * blockIdx.x + 1] = ss;
        part[3 * blockIdx.x + 2] = sa;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double c = 0.0, s = 0.0, a = 0.0;
    for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        c += part[3 * b + 0];
        s += part[3 * b + 1];
        a += part[3 * b + 2];
    }
    c = sb::block_sum_all_d(c, red);
    s = sb::block_sum_all_d(s, red);
    a = sb::block_sum_all_d(a, red);
    if (threadIdx.x == 0) {
        const double v = (a > 0.0) ? (c * c + s * s) / (a * a) : 0.0;
        *sr = (float)v;
        if (integrate && int_sr) {
            int_sr[0] += (double)(float)v;   // running sum of the float32 SR values
            int_sr[1] += 1.0;                // count
        }
        *counter = 0u;
    }
}

__global__ void __launch_bounds__(kPsfThreads) psf_field_kernel(const float *__restrict__ A,
                                                               const float *__restrict__ ph, int n, float k,
                                                               float2 *__restrict__ u) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        u[e] = field_value(A, ph, e, k);
}

// psf = |F|^2 and per-block partial sums (float64)
__global__ void __launch_bounds__(kPsfThreads) psf_abs2_kernel(const float2 *__restrict__ F, long long n,
                                                              float *__restrict__ psf, double *__restrict__ part) {
    __shared__ double red[33];
    double acc = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const float2 f = F[e];
        const float p = __fadd_rn(__fmul_rn(f.x, f.x), __fmul_rn(f.y, f.y));
        psf[e] = p;
        acc += p;
    }
    acc = sb::block_sum_all_d(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// psf /= sum(psf); optionally int_psf += psf (psf.py:79-96, 126-137)
__global__ void __launch_bounds__(kPsfThreads) psf_normalize_kernel(float *__restrict__ psf, long long n,
                                                                   const double *__restrict__ part, int nparts,
                                                                   float *__restrict__ int_psf) {
    __shared__ double red[33];
    double t = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) t += part[b];
    t = sb::block_sum_all_d(t, red);
    const float total = (float)t;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const float v = __fdiv_rn(psf[e], total);
        psf[e] = v;
        if (int_psf) int_psf[e] = __fadd_rn(int_psf[e], v);
    }
}

int grid_for(long long n) {
    long long b = (n + kPsfThreads - 1) / kPsfThreads;
    return (int)(b < kPsfMaxBlocks ? (b < 1 ? 1 : b) : kPsfMaxBlocks);
}

}  // namespace

extern "C" size_t sb_psf_scratch_bytes(void) {
    // Strehl partials (3 doubles per block) + counter, PSF partials
    return ((size_t)kPsfMaxBlocks * 3 * sizeof(double) + 256 + (size_t)kPsfMaxBlocks * sizeof(double) + 255) &
           ~(size_t)255;
}

extern "C" int sb_strehl(const float *A, const float *phase_nm, int n_pixels, float phase_to_rad, float *sr,
                         double *int_sr, int integrate, void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!A || !phase_nm || !sr || n_pixels < 1) return sb::fail(SB_EINVAL, "sb_strehl: bad args");
    if (!scratch || scratch_bytes < sb_psf_scratch_bytes())
        return sb::fail(SB_ESCRATCH, "sb_strehl: scratch needs %zu bytes", sb_psf_scratch_bytes());
    double *part = static_cast<double *>(scratch);
    unsigned int *counter = reinterpret_cast<unsigned int *>(part + 3 * kPsfMaxBlocks);
    strehl_kernel<<<grid_for(n_pixels), kPsfThreads, 0, sb::as_stream(stream)>>>(
        A, phase_nm, n_pixels, phase_to_rad, part, counter, sr, int_sr, integrate);
    return sb::check_launch("strehl_kernel");
}

extern "C" int sb_psf_field(const float *A, const float *phase_nm, int n_pixels, float phase_to_rad, void *field,
                            void *stream) {
    sb::clear_error();
    if (!A || !phase_nm || !field || n_pixels < 1) return sb::fail(SB_EINVAL, "sb_psf_field: bad args");
    psf_field_kernel<<<grid_for(n_pixels), kPsfThreads, 0, sb::as_stream(stream)>>>(
        A, phase_nm, n_pixels, phase_to_rad, static_cast<float2 *>(field));
    return sb::check_launch("psf_field_kernel");
}

extern "C" int sb_psf_finish(const void *focal_field, long long n_pixels, float *psf, float *int_psf, void *scratch,
                             size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!focal_field || !psf || n_pixels < 1) return sb::fail(SB_EINVAL, "sb_psf_finish: bad args");
    if (!scratch || scratch_bytes < sb_psf_scratch_bytes())
        return sb::fail(SB_ESCRATCH, "sb_psf_finish: scratch needs %zu bytes", sb_psf_scratch_bytes());
    double *part = reinterpret_cast<double *>(static_cast<char *>(scratch) + kPsfMaxBlocks * 3 * sizeof(double) + 256);
    const int nb = grid_for(n_pixels);
    cudaStream_t st = sb::as_stream(stream);
    psf_abs2_kernel<<<nb, kPsfThreads, 0, st>>>(static_cast<const float2 *>(focal_field), n_pixels, psf, part);
    int rc = sb::check_launch("psf_abs2_kernel");
    if (rc) return rc;
    psf_normalize_kernel<<<nb, kPsfThreads, 0, st>>>(psf, n_pixels, part, nb, int_psf);
    return sb::check_launch("psf_normalize_kernel");
}
