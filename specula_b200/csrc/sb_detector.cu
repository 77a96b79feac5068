// CCD detector and Shack-Hartmann slope computer on the B200.
//
// CCD (ccd.py:198-287): one thread per pixel integrates the intensity and,
// on read-out steps, applies QE, background/dark, Poisson photon noise,
// Gaussian read-out noise and the ADU quantisation.  Random numbers come
// from Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), a counter-based
// generator: the draw of pixel e in frame f is a pure function of
// (seed, f, e, draw), so results do not depend on the launch shape.
// Poisson sampling (float32): sequential-search inversion below mean 10,
// Hormann's PTRS transformed rejection (1993) above.
//
// ShSlopec (sh_slopec.py:308-438): one warp per valid sub-aperture gathers
// its pixels through the index table and reduces flux, denominator and the
// two weighted sums; a second kernel applies the 1e-3*mean cut-off that
// needs the mean over all sub-apertures, in a fixed order.
#include <new>

#include "sb_common.cuh"
#include "sb_mc.cuh"

namespace {

struct u4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
    const uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds; multipliers and Weyl key increments as published.
__host__ __device__ __forceinline__ u4 philox4x32_10(u4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo(M0, c.x, hi0, lo0);
        mulhilo(M1, c.z, hi1, lo1);
        u4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

// uniform in (0,1) from the top 24 bits of a word
__device__ __forceinline__ float u01f(uint32_t a) { return ((float)(a >> 8) + 0.5f) * (1.0f / 16777216.0f); }

constexpr uint32_t kPhotonTag = 0x50484f54u;   // "PHOT"
constexpr uint32_t kReadoutTag = 0x52454144u;  // "READ"
constexpr uint32_t kCicTag = 0x4349434eu;      // "CICN"
constexpr uint32_t kExcessTag = 0x45584353u;   // "EXCS"

// log(k!) for k < 32 (math.lgamma(k + 1) rounded to float)
__constant__ float c_logfact[32] = {0.0f, 0.0f, 0.693147181f, 1.79175947f, 3.17805383f, 4.78749174f, 6.57925121f, 8.52516136f, 10.6046029f, 12.8018275f, 15.1044126f, 17.5023078f, 19.9872145f, 22.5521639f, 25.1912212f, 27.8992714f, 30.6718601f, 33.5050735f, 36.3954452f, 39.3398842f, 42.3356165f, 45.3801389f, 48.4711814f, 51.6066756f, 54.7847294f, 58.0036052f, 61.2617018f, 64.5575386f, 67.8897431f, 71.257039f, 74.6582363f, 78.0922236f};

// log(k!) for integer-valued k >= 0: table below 32 (staged in shared memory
// by the caller), Stirling's series for log Gamma(k + 1) above (error < 1e-9
// relative there)
__device__ __forceinline__ float log_factorial(float k, const float *tbl) {
    if (k < 32.0f) return tbl[(int)k];
    const float z = k + 1.0f, iz = 1.0f / z, iz2 = iz * iz;
    return (z - 0.5f) * __logf(z) - z + 0.91893853f + iz * (0.083333333f - iz2 * (0.0027777778f - iz2 * 0.00079365079f));
}

// Poisson(lam) in float32 arithmetic.  lam < 10: sequential-search
// inversion of one uniform.  lam >= 10: PTRS transformed rejection
// (Hormann 1993), two uniforms per try, at most 64 tries (acceptance per try
// is above 0.9, so the bound is never reached in practice).
__device__ float poisson_sample(float lam, uint32_t e, uint64_t frame, uint64_t seed, const float *logfact) {
    if (!(lam > 0.0f)) return 0.0f;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kPhotonTag;
    if (lam < 10.0f) {
        const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 0u}, k0, k1);
        const float u = u01f(r.x);
        float pk = __expf(-lam), cdf = pk;
        int k = 0;
        while (u > cdf && k < 100) {
            ++k;
            pk *= __fdividef(lam, (float)k);
            cdf += pk;
        }
        return (float)k;
    }
    // acceptance tests use the fast log / divide intrinsics: their few-ulp
    // errors move only decisions that sit on the acceptance boundary
    const float slam = sqrtf(lam), loglam = __logf(lam);
    const float b = 0.931f + 2.53f * slam;
    const float a = -0.059f + 0.02483f * b;
    const float log_inv_alpha = __logf(1.1239f + __fdividef(1.1328f, b - 3.4f));
    const float vr = 0.9277f - __fdividef(3.6224f, b - 2.0f);
    const float two_a = 2.0f * a;
    for (uint32_t it = 0; it < 32; ++it) {
        const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 1u + it}, k0, k1);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float U = u01f(h ? r.z : r.x) - 0.5f;
            const float V = u01f(h ? r.w : r.y);
            const float us = 0.5f - fabsf(U);
            const float k = floorf((__fdividef(two_a, us) + b) * U + lam + 0.43f);
            if (us >= 0.07f && V <= vr) return k;
            if (k < 0.0f || (us < 0.013f && V > us)) continue;
            if (__logf(V) + log_inv_alpha - __logf(__fdividef(a, us * us) + b) <=
                -lam + k * loglam - log_factorial(k, logfact))
                return k;
        }
    }
    return floorf(lam + 0.5f);
}

// Gamma(shape, 1) by Marsaglia and Tsang's squeeze-and-reject method
// ("A simple method for generating gamma variables", ACM TOMS 26, 2000):
// d = shape - 1/3, c = 1/sqrt(9 d), v = (1 + c x)^3 for x ~ N(0,1), accepted
// with u ~ U(0,1) when u < 1 - 0.0331 x^4 or log u < x^2/2 + d (1 - v + log v);
// shapes below 1 as Gamma(shape + 1) u^(1/shape).  Draws from the excess
// stream of pixel e in frame f; at most 32 tries (acceptance per try > 0.95).
__device__ float gamma_sample(float shape, uint32_t e, uint64_t frame, uint64_t seed) {
    if (!(shape > 0.0f)) return 0.0f;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kExcessTag;
    const bool boost = shape < 1.0f;
    const float a = boost ? shape + 1.0f : shape;
    const float d = a - 1.0f / 3.0f, c = rsqrtf(9.0f * d);
    float g = d;
    uint32_t it = 0;
    for (; it < 32; ++it) {
        const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 16u + it}, k0, k1);
        const float x = sqrtf(-2.0f * __logf(u01f(r.x))) * cospif(2.0f * u01f(r.y));
        float v = fmaf(c, x, 1.0f);
        if (v <= 0.0f) continue;
        v = v * v * v;
        const float u = u01f(r.z);
        const float x2 = x * x;
        if (u < 1.0f - 0.0331f * x2 * x2 || __logf(u) < 0.5f * x2 + d * (1.0f - v + __logf(v))) {
            g = d * v;
            break;
        }
    }
    if (boost) {
        const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 15u}, k0, k1);
        g *= __powf(u01f(r.w), 1.0f / shape);
    }
    return g;
}

// Bernoulli(p) electron of clock-induced charge
__device__ __forceinline__ float cic_sample(float p, uint32_t e, uint64_t frame, uint64_t seed) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kCicTag;
    const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 0u}, k0, k1);
    return u01f(r.x) < p ? 1.0f : 0.0f;
}

// N(0,1) by Box-Muller from one Philox block
__device__ __forceinline__ float std_normal(uint32_t e, uint64_t frame, uint64_t seed) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kReadoutTag;
    const u4 r = philox4x32_10({e, (uint32_t)frame, (uint32_t)(frame >> 32), 0u}, k0, k1);
    return sqrtf(-2.0f * __logf(u01f(r.x))) * cospif(2.0f * u01f(r.y));
}

// Batched launches (seeds != NULL): the pixels of n_batch realisations are
// contiguous, n_per each; realisation b draws with photon_seeds[b] /
// readout_seeds[b] and its own pixel index, so its frame equals what a
// single-realisation launch with those seeds gives.
//
// With photon noise the block's 256 pixels are first ordered by sampler
// branch (mean < 10: sequential inversion, else PTRS) through shared memory,
// so that most warps run one branch with all lanes; each pixel's draw
// depends only on its mean, index, frame and seeds, so the frame is the same
// bit for bit as with pixels sampled in place.
constexpr int kCcdThreads = 256;

__device__ __forceinline__ float ccd_sample(const sb_ccd_params &p, float f, int e, uint64_t frame,
                                            const uint64_t *photon_seeds, const uint64_t *readout_seeds, int n_per,
                                            const float *logfact, double inv_gain, bool gain_pow2) {
    uint32_t eloc = (uint32_t)e;
    uint64_t pseed = p.photon_seed, rseed = p.readout_seed;
    if (photon_seeds) {
        const int b = e / n_per;
        eloc = (uint32_t)(e - b * n_per);
        pseed = photon_seeds[b];
        rseed = readout_seeds[b];
    }
    if (p.cic_noise) f = __fadd_rn(f, cic_sample(p.cic_level, eloc, frame, pseed));       // ccd.py:226-227
    const bool excess = p.excess_noise != 0;
    if (p.photon_noise) {
        double v = poisson_sample(f, eloc, frame, pseed, logfact);
        // EMCCD multiplication (ccd.py:232-233); the frame stays an integer
        // array (truncating read-out noise and ADU division) only without it
        if (excess) v = (double)gamma_sample((float)(p.excess_delta * v), eloc, frame, p.excess_seed) *
                        (double)p.emccd_gain / (double)p.excess_delta;
        if (p.readout_noise) {
            const double ron = (double)(std_normal(eloc, frame, rseed) * p.readout_level);
            v += excess ? ron : trunc(ron);
        }
        // float frames only (the host rejects gains on the integer frame)
        if (p.pixel_gains) v *= (double)p.pixel_gains[eloc];                                  // ccd.py:239-240
        if (p.qe_map && p.qe_map_normalise) v *= 1.0 / (double)p.qe_map[eloc];                 // ccd.py:242-245
        // ADU: round(x*g)+bias, clamp at 0, -bias, /g (ccd.py:247-258)
        double x = rint(v * (double)p.adu_gain) + (double)p.adu_bias;
        x = x < 0.0 ? 0.0 : x;
        x -= (double)p.adu_bias;
        // a power-of-two gain (the default 8) divides exactly by its
        // reciprocal; any other gain takes the float64 division
        x = gain_pow2 ? x * inv_gain : x / (double)p.adu_gain;
        if (excess)
            x /= (double)p.emccd_gain;
        else
            x = trunc(x);
        if (p.dark_noise) x -= (double)p.dark_level;
        return (float)x;
    }
    if (excess)
        f = (float)((double)gamma_sample(__fmul_rn(p.excess_delta, f), eloc, frame, p.excess_seed) *
                    (double)p.emccd_gain / (double)p.excess_delta);
    if (p.readout_noise) f = __fadd_rn(f, __fmul_rn(std_normal(eloc, frame, rseed), p.readout_level));
    if (p.pixel_gains) f = __fmul_rn(f, p.pixel_gains[eloc]);
    if (p.qe_map && p.qe_map_normalise) f = __fmul_rn(f, 1.0f / p.qe_map[eloc]);
    return f;
}

__global__ void __launch_bounds__(kCcdThreads, 4) ccd_kernel(sb_ccd_params p, const float *__restrict__ in,
                                                          float *__restrict__ integ, float *__restrict__ pix,
                                                          const uint64_t *__restrict__ photon_seeds,
                                                          const uint64_t *__restrict__ readout_seeds, int n_per) {
    // frame bookkeeping lives on the device; every block reads it before the
    // last block to finish advances it (see the end of the kernel)
    volatile sb_ccd_state *vs = p.state;
    __shared__ unsigned int warps_done;
    __shared__ float logfact[32];
    __shared__ int s_idx[kCcdThreads];
    __shared__ float s_mean[kCcdThreads];
    __shared__ int s_small[kCcdThreads / 32];
    if (threadIdx.x == 0) warps_done = 0u;
    if (threadIdx.x < 32) logfact[threadIdx.x] = c_logfact[threadIdx.x];
    const uint64_t frame = vs->frame_index;
    const int nint = vs->n_integrated + 1;
    const bool readout = nint >= p.frames_per_read;
    const double inv_gain = 1.0 / (double)p.adu_gain;
    const bool gain_pow2 = (__double_as_longlong((double)p.adu_gain) & 0x000FFFFFFFFFFFFFLL) == 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    // block-uniform loop: every thread takes part in the shared-memory ordering
    for (int base = blockIdx.x * kCcdThreads; base < p.n_pixels; base += gridDim.x * kCcdThreads) {
        const int e = base + threadIdx.x;
        const bool valid = e < p.n_pixels;
        float f = 0.f;
        if (valid) {
            // integrated_i += i * (loop_dt * bandw)   (ccd.py:205)
            const float acc = __fadd_rn(integ[e], __fmul_rn(in[e], p.rate));
            if (!readout) {
                integ[e] = acc;
            } else {
                f = acc;
                if (p.qe != 1.0f) f = __fmul_rn(f, p.qe);                  // ccd.py:282-287
                if (p.qe_map) f = __fmul_rn(f, p.qe_map[photon_seeds ? e % n_per : e]);
                f = __fadd_rn(f, p.bg_plus_dark);                           // ccd.py:220-221
            }
        }
        if (!readout) continue;
        if (!p.photon_noise) {
            if (valid) {
                pix[e] = ccd_sample(p, f, e, frame, photon_seeds, readout_seeds, n_per, logfact, inv_gain, gain_pow2);
                integ[e] = 0.0f;                                            // ccd.py:216
            }
            continue;
        }
        // order by sampler branch: means below 10 first, then the rest
        const bool small = valid && f < 10.0f;
        const unsigned int bal = __ballot_sync(0xffffffffu, small);
        if (lane == 0) s_small[warp] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kCcdThreads / 32; ++w) {
            const int c = s_small[w];
            before += w < warp ? c : 0;
            total += c;
        }
        const int rank = __popc(bal & ((1u << lane) - 1u));
        const int slot = small ? before + rank : total + (warp * 32 - before) + (lane - rank);
        s_idx[slot] = valid ? e : -1;
        s_mean[slot] = f;
        __syncthreads();
        const int ei = s_idx[threadIdx.x];
        const float fi = s_mean[threadIdx.x];
        __syncthreads();                        // the tables are refilled by the next pass
        if (ei >= 0) {
            pix[ei] = ccd_sample(p, fi, ei, frame, photon_seeds, readout_seeds, n_per, logfact, inv_gain, gain_pow2);
            integ[ei] = 0.0f;                                               // ccd.py:216
        }
    }
    // the last warp to finish in the last block to finish advances the frame
    // state; warps that are done do not wait for the slower ones (the noise
    // sampling loops diverge)
    __syncwarp();
    if (lane == 0) {
        const unsigned int nwarps = (blockDim.x + 31) >> 5;
        if (atomicAdd(&warps_done, 1u) == nwarps - 1) {
            __threadfence();
            if (atomicAdd(&p.state->blocks_done, 1u) == gridDim.x - 1) {
                vs->n_integrated = readout ? 0 : nint;
                if (readout) vs->frame_index = frame + 1;
                vs->blocks_done = 0u;
                __threadfence();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Binned readout (ccd.py:198-216, 262-280).  Every step the full-resolution
// frame is integrated; on a readout step the b x b block sums S are formed
// and scaled as the reference does, S * b^2 * (sum(frame) / sum(S)), and the
// QE / noise / ADU model runs on the binned pixels.  Three launches, each
// reading the device frame state; the last one resets the integration and
// advances the state.
// ---------------------------------------------------------------------------
constexpr int kBinBlocks = 592;

__device__ __forceinline__ bool ccd_readout_now(const sb_ccd_params &p) {
    volatile sb_ccd_state *vs = p.state;
    return vs->n_integrated + 1 >= p.frames_per_read;
}

__global__ void __launch_bounds__(256) ccd_integrate_kernel(sb_ccd_params p, const float *__restrict__ in,
                                                            float *__restrict__ integ, int n) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        integ[e] = __fadd_rn(integ[e], __fmul_rn(in[e], p.rate));     // ccd.py:205
}

// binned[e] = block sum; per-CTA partial sums (float64) of the full frame
// and of the block sums
__global__ void __launch_bounds__(256) ccd_bin_sums_kernel(sb_ccd_params p, const float *__restrict__ integ,
                                                           int cols, int b, int out_rows, int out_cols,
                                                           float *__restrict__ binned, double *__restrict__ part) {
    __shared__ double red[33];
    if (!ccd_readout_now(p)) return;
    const int n_out = out_rows * out_cols;
    double tot = 0.0, sb = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_out; e += gridDim.x * blockDim.x) {
        const int r = e / out_cols, c = e - r * out_cols;
        double acc = 0.0;
        for (int u = 0; u < b; ++u)
            for (int v = 0; v < b; ++v) acc += integ[(size_t)(r * b + u) * cols + c * b + v];
        const float s = (float)acc;
        binned[e] = s;
        tot += acc;
        sb += s;
    }
    tot = sb::block_sum_all_d(tot, red);
    sb = sb::block_sum_all_d(sb, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = tot;
        part[2 * blockIdx.x + 1] = sb;
    }
}

__global__ void __launch_bounds__(kCcdThreads) ccd_bin_noise_kernel(sb_ccd_params p, const float *__restrict__ binned,
                                                                   const double *__restrict__ part, int nparts,
                                                                   int b, int n_out, float *__restrict__ pix,
                                                                   float *__restrict__ integ, int n_full) {
    volatile sb_ccd_state *vs = p.state;
    __shared__ double red[33];
    __shared__ float logfact[32];
    __shared__ unsigned int warps_done;
    if (threadIdx.x == 0) warps_done = 0u;
    if (threadIdx.x < 32) logfact[threadIdx.x] = c_logfact[threadIdx.x];
    const uint64_t frame = vs->frame_index;
    const int nint = vs->n_integrated + 1;
    const bool readout = nint >= p.frames_per_read;
    const double inv_gain = 1.0 / (double)p.adu_gain;
    const bool gain_pow2 = (__double_as_longlong((double)p.adu_gain) & 0x000FFFFFFFFFFFFFLL) == 0;
    __syncthreads();
    if (readout) {
        double tot = 0.0, sb = 0.0;
        for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
            tot += part[2 * k];
            sb += part[2 * k + 1];
        }
        tot = sb::block_sum_all_d(tot, red);
        sb = sb::block_sum_all_d(sb, red);
        const float ratio = (float)sb != 0.f ? __fdiv_rn((float)tot, (float)sb) : 0.f;
        const float b2 = (float)(b * b);
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_out; e += gridDim.x * blockDim.x) {
            float f = __fmul_rn(__fmul_rn(binned[e], b2), ratio);
            if (p.qe != 1.0f) f = __fmul_rn(f, p.qe);                        // ccd.py:282-287
            if (p.qe_map) f = __fmul_rn(f, p.qe_map[e]);
            f = __fadd_rn(f, p.bg_plus_dark);                                 // ccd.py:220-221
            pix[e] = ccd_sample(p, f, e, frame, nullptr, nullptr, n_out, logfact, inv_gain, gain_pow2);
        }
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_full; e += gridDim.x * blockDim.x)
            integ[e] = 0.0f;                                                  // ccd.py:216
    }
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        const unsigned int nwarps = (blockDim.x + 31) >> 5;
        if (atomicAdd(&warps_done, 1u) == nwarps - 1) {
            __threadfence();
            if (atomicAdd(&p.state->blocks_done, 1u) == gridDim.x - 1) {
                vs->n_integrated = readout ? 0 : nint;
                if (readout) vs->frame_index = frame + 1;
                vs->blocks_done = 0u;
                __threadfence();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Charge-transfer inefficiency (ccd.py:223-224): on a read-out step the frame
// after QE and background goes through M0 * frame * M1 before the noise.
// Four launches, each gated on the device frame state: the pre-noise frame,
// the two products (16 x 16 shared-memory tiles, FP32), the noise.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) ccd_cte_frame_kernel(sb_ccd_params p, const float *__restrict__ in,
                                                            float *__restrict__ integ, float *__restrict__ frame) {
    volatile sb_ccd_state *vs = p.state;
    const bool readout = vs->n_integrated + 1 >= p.frames_per_read;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < p.n_pixels; e += gridDim.x * blockDim.x) {
        const float acc = __fadd_rn(integ[e], __fmul_rn(in[e], p.rate));        // ccd.py:205
        if (!readout) {
            integ[e] = acc;
            continue;
        }
        float f = acc;
        if (p.qe != 1.0f) f = __fmul_rn(f, p.qe);                              // ccd.py:282-287
        if (p.qe_map) f = __fmul_rn(f, p.qe_map[e]);
        frame[e] = __fadd_rn(f, p.bg_plus_dark);                                // ccd.py:220-221
        integ[e] = 0.0f;                                                        // ccd.py:216
    }
}

// C (m x n) = A (m x k) * B (k x n), row-major, on read-out steps only
__global__ void __launch_bounds__(256) ccd_cte_matmul_kernel(sb_ccd_params p, const float *__restrict__ A,
                                                             const float *__restrict__ B, float *__restrict__ Cm,
                                                             int m, int n, int k) {
    __shared__ float As[16][17], Bs[16][17];
    volatile sb_ccd_state *vs = p.state;
    if (vs->n_integrated + 1 < p.frames_per_read) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
    float acc = 0.f;
    for (int k0 = 0; k0 < k; k0 += 16) {
        As[ty][tx] = (row < m && k0 + tx < k) ? A[(size_t)row * k + k0 + tx] : 0.f;
        Bs[ty][tx] = (k0 + ty < k && col < n) ? B[(size_t)(k0 + ty) * n + col] : 0.f;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 16; ++j) acc = fmaf(As[ty][j], Bs[j][tx], acc);
        __syncthreads();
    }
    if (row < m && col < n) Cm[(size_t)row * n + col] = acc;
}

__global__ void __launch_bounds__(kCcdThreads) ccd_cte_noise_kernel(sb_ccd_params p, const float *__restrict__ frame,
                                                                    float *__restrict__ pix) {
    volatile sb_ccd_state *vs = p.state;
    __shared__ float logfact[32];
    __shared__ unsigned int warps_done;
    if (threadIdx.x == 0) warps_done = 0u;
    if (threadIdx.x < 32) logfact[threadIdx.x] = c_logfact[threadIdx.x];
    const uint64_t frame_idx = vs->frame_index;
    const int nint = vs->n_integrated + 1;
    const bool readout = nint >= p.frames_per_read;
    const double inv_gain = 1.0 / (double)p.adu_gain;
    const bool gain_pow2 = (__double_as_longlong((double)p.adu_gain) & 0x000FFFFFFFFFFFFFLL) == 0;
    __syncthreads();
    if (readout)
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < p.n_pixels; e += gridDim.x * blockDim.x)
            pix[e] = ccd_sample(p, frame[e], e, frame_idx, nullptr, nullptr, p.n_pixels, logfact, inv_gain, gain_pow2);
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        const unsigned int nwarps = (blockDim.x + 31) >> 5;
        if (atomicAdd(&warps_done, 1u) == nwarps - 1) {
            __threadfence();
            if (atomicAdd(&p.state->blocks_done, 1u) == gridDim.x - 1) {
                vs->n_integrated = readout ? 0 : nint;
                if (readout) vs->frame_index = frame_idx + 1;
                vs->blocks_done = 0u;
                __threadfence();
            }
        }
    }
}

__global__ void philox_raw_kernel(uint32_t k0, uint32_t k1, uint32_t c1, uint32_t c2, uint32_t c3, int n,
                                  uint32_t *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u4 r = philox4x32_10({(uint32_t)i, c1, c2, c3}, k0, k1);
        out[4 * i + 0] = r.x;
        out[4 * i + 1] = r.y;
        out[4 * i + 2] = r.z;
        out[4 * i + 3] = r.w;
    }
}

__global__ void __launch_bounds__(256) slopec_sums_kernel(sb_slopec_plan pl, const float *__restrict__ pix,
                                                          float *__restrict__ flux, float *__restrict__ tot,
                                                          float *__restrict__ sxn, float *__restrict__ syn,
                                                          float *__restrict__ part_tot, long long frame_stride,
                                                          int flux_stride, int work_stride) {
    __shared__ float wsum[8];
    // batched launches: blockIdx.y selects the realisation
    pix += blockIdx.y * frame_stride;
    flux += (size_t)blockIdx.y * flux_stride;
    tot += (size_t)blockIdx.y * work_stride;
    sxn += (size_t)blockIdx.y * work_stride;
    syn += (size_t)blockIdx.y * work_stride;
    part_tot += (size_t)blockIdx.y * gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const bool valid = s < pl.n_subaps;
    const int32_t *ix = pl.idxs + (size_t)(valid ? s : 0) * pl.npx2;
    float thr = pl.thr;
    if (pl.thr_ratio > 0.f) {
        // thr = thr_ratio * the sub-aperture's largest (windowed) pixel
        // (sh_slopec.py:215-232); the first pass only reads the pixels
        float m = -INFINITY;
        for (int e = lane; valid && e < pl.npx2; e += 32) {
            float v = pix[ix[e]];
            if (pl.window) v = __fmul_rn(v, pl.window[(size_t)e * pl.n_subaps + s]);
            m = fmaxf(m, v);
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        thr = pl.thr_ratio * m;
    }
    float f = 0.f, t = 0.f, x = 0.f, y = 0.f;
    for (int e = lane; valid && e < pl.npx2; e += 32) {
        float v = pix[ix[e]];
        f += v;
        if (pl.window) v = __fmul_rn(v, pl.window[(size_t)e * pl.n_subaps + s]);    // sh_slopec.py:368-371
        float w;
        if (pl.thr_pedestal) {
            w = v < thr ? 0.f : v;            // pixels below thr -> 0 (sh_slopec.py:381-382)
        } else {
            w = v - thr;                      // pixels -= thr; clamp < 0 -> 0
            w = w < 0.f ? 0.f : w;
        }
        t = fmaf(w, pl.mw[e], t);
        x = fmaf(w, pl.xw[e], x);
        y = fmaf(w, pl.yw[e], y);
    }
    f = sb::warp_sum(f);
    t = sb::warp_sum(t);
    x = sb::warp_sum(x);
    y = sb::warp_sum(y);
    if (lane == 0) {
        if (valid) {
            flux[s] = f;
            tot[s] = t;
            sxn[s] = x;
            syn[s] = y;
        }
        wsum[warp] = valid ? t : 0.f;
    }
    __syncthreads();
    // per-block partial of the denominators, summed in warp order
    if (threadIdx.x == 0) {
        float b = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += wsum[w];
        part_tot[blockIdx.x] = b;
    }
}

__global__ void __launch_bounds__(256) slopec_finish_kernel(int n, const float *__restrict__ tot,
                                                            const float *__restrict__ sxn,
                                                            const float *__restrict__ syn,
                                                            const float *__restrict__ part_tot, int nparts,
                                                            float *__restrict__ slopes, int slopes_stride,
                                                            int work_stride, float mult) {
    __shared__ double red[33];
    tot += (size_t)blockIdx.y * work_stride;
    sxn += (size_t)blockIdx.y * work_stride;
    syn += (size_t)blockIdx.y * work_stride;
    part_tot += (size_t)blockIdx.y * nparts;
    slopes += (size_t)blockIdx.y * slopes_stride;
    double acc = 0.0;
    for (int e = threadIdx.x; e < nparts; e += blockDim.x) acc += part_tot[e];
    acc = sb::block_sum_all_d(acc, red);
    const float mean = (float)(acc / n);
    const float cut = 1.0f / (mean * 1e-3f);   // sh_slopec.py:393-400
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float fac = 1.0f / tot[s];
        fac = fac > cut ? 0.0f : fac;
        float sx = sxn[s] * fac, sy = syn[s] * fac;
        if (mult != 0.0f) {                   // sh_slopec.py:416-418
            sx *= mult;
            sy *= mult;
        }
        slopes[s] = sx;
        slopes[n + s] = sy;
    }
}

// ---------------------------------------------------------------------------
// The per-sub-aperture chain of one loop step in one launch, after the SH
// forward has left its unnormalised frame and per-CTA partial sums:
//   photon normalisation (sh.py:425-427), CCD integrate / QE / noise / ADU
//   (ccd.py:198-287, detector dt = loop dt, no binning), CoG sums of every
//   valid sub-aperture (sh_slopec.py:368-404) and, in the last CTA, the
//   1e-3 * mean flux cut-off and the detector frame state.
// A CTA owns up to 8 lenslets of one lenslet row: their npx x 8 npx pixel
// tile is sampled into shared memory and each warp reduces one lenslet's box.
// Every sum is taken in the order of the separate kernels
// (sh_normalize_kernel, ccd_kernel, slopec_sums_kernel, slopec_finish_kernel),
// so the results are the same bits; the sub-aperture table must list each
// valid box's pixels row-major (the caller checks it and passes the lenslet
// -> sub-aperture map).
// ---------------------------------------------------------------------------
constexpr int kChainSumThreads = 256;    // thread count whose summation orders the sums reproduce
constexpr int kChainMaxThreads = 512;    // a CTA samples up to this many pixels per pass
constexpr int kChainLenses = 8;          // lenslets per CTA: one CoG warp each
constexpr int kChainMaxNpx = 16;
constexpr int kChainTile = 4096;         // pixels of a CTA's lenslets (npx x width*npx)

// threads of a CTA: the lenslet tile (npx x 8 npx pixels) in one pass when it
// fits in 512, never fewer than the 256 whose sums are reproduced
__host__ __device__ inline int chain_threads(int npx) {
    const int tile = (npx * kChainLenses * npx + 31) / 32 * 32;
    return tile < kChainSumThreads ? kChainSumThreads : (tile > kChainMaxThreads ? kChainMaxThreads : tile);
}

struct ChainArgs {
    sb_ccd_params p;
    const float *part_I;          // SH partial sums of the frame
    const float *part_A;          // SH partial sums of the normalising amplitude
    int nparts;
    float photon_scale;
    float *I;                     // frame: unnormalised in, normalised out
    float *integ;
    float *pix;
    int n, npx, side;
    const int32_t *lenslet_subap; // [n*n] valid sub-aperture index or -1
    int n_valid;
    float thr;
    const float *xw, *yw, *mw;
    float *slopes, *flux, *tot, *sxn, *syn;
};

// element offsets of a CTA's realisation in the buffers of ChainArgs
struct ChainOff {
    long long frame;
    size_t part, slopes, flux, work;
};

// where a CTA's realisation keeps its seeds and completion counters
struct ChainSlot {
    const uint64_t *photon_seed, *readout_seed;  // NULL: the parameters' seeds
    unsigned int *real_done;    // NULL: the frame state's counter serves the whole launch
    unsigned int real_ctas;     // CTAs of the realisation
    unsigned int group_ctas;    // CTAs sharing the frame state
    int cutoff;                 // 0: leave the flux cut-off to sb_slopec_cutoff (a band of rows)
};

// the 1e-3 * mean flux cut-off of sh_slopec.py:393-404 over every valid
// sub-aperture, by one CTA of at least kChainSumThreads threads: the mean of
// the denominators as slopec_finish_kernel forms it (partials of 8
// consecutive sub-apertures summed in float in warp order, then in float64
// over 256 threads), then the slopes of the sub-apertures below it zeroed
__device__ __forceinline__ void chain_cutoff(const float *tot, const float *sxn, const float *syn, float *slopes,
                                             int nv, double *dred) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int ngroups = (nv + 7) / 8;
    double acc = 0.0;
    for (int g = tid; tid < kChainSumThreads && g < ngroups; g += kChainSumThreads) {
        float b = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int s = 8 * g + k;
            b += s < nv ? __ldcg(tot + s) : 0.f;
        }
        acc += b;
    }
    acc = sb::block_sum_all_d(acc, dred);
    const float mean = (float)(acc / nv);
    const float cut = 1.0f / (mean * 1e-3f);
    for (int s = tid; s < nv; s += nthr) {
        const float fac = 1.0f / __ldcg(tot + s);
        if (fac > cut) {
            slopes[s] = __ldcg(sxn + s) * 0.0f;
            slopes[nv + s] = __ldcg(syn + s) * 0.0f;
        }
    }
}

// the chain for lenslet block (bx, by) of one realisation; any CTA size from
// 256 to 512 threads gives the same bits
// the chain for lenslets j0 .. j0 + width - 1 of lenslet row by (their
// npx x width*npx pixels staged in shared memory, at most kChainTile)
template <int IPT>
__device__ __forceinline__ void chain_body(const ChainArgs &a, const ChainOff &o, int j0, int width, int by,
                                           const ChainSlot &slot) {
    static_assert(IPT >= 1 && IPT * kChainSumThreads <= kChainMaxThreads * 2, "pixels per pass");
    __shared__ double dred[33];
    __shared__ float logfact[32];
    __shared__ int s_idx[IPT * kChainMaxThreads];
    __shared__ float s_mean[IPT * kChainMaxThreads];
    __shared__ int s_small[IPT * kChainMaxThreads / 32];
    __shared__ float tile[kChainTile];
    __shared__ int s_last, s_group_last;
    const sb_ccd_params &p = a.p;
    const float *part_I = a.part_I + o.part, *part_A = a.part_A + o.part;
    float *I = a.I + o.frame, *integ = a.integ + o.frame, *pix = a.pix + o.frame;
    float *slopes = a.slopes + o.slopes, *flux = a.flux + o.flux;
    float *tot = a.tot + o.work, *sxn = a.sxn + o.work, *syn = a.syn + o.work;
    volatile sb_ccd_state *vs = p.state;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 32) logfact[tid] = c_logfact[tid];
    const uint64_t frame = vs->frame_index;
    const double inv_gain = 1.0 / (double)p.adu_gain;
    const bool gain_pow2 = (__double_as_longlong((double)p.adu_gain) & 0x000FFFFFFFFFFFFFLL) == 0;

    const int nthr = blockDim.x, nwarps = nthr >> 5;
    // photon normalisation: the sums of sh_normalize_kernel (256 threads), in
    // its order; warps past the eighth add exact zeros
    double si = 0.0, sa = 0.0;
    if (tid < kChainSumThreads)
        for (int e = tid; e < a.nparts; e += kChainSumThreads) {
            si += part_I[e];
            sa += part_A[e];
        }
    si = sb::block_sum_all_d(si, dred);
    sa = sb::block_sum_all_d(sa, dred);
    const float phot = (float)(a.photon_scale * sa);
    const float scale = phot / (float)si;

    const int i = by;
    const int w = min(width, a.n - j0);
    const int npx = a.npx, wc = w * npx, P = npx * wc, tld = wc;
    // detector: every pass samples up to IPT * blockDim pixels of the tile
    // (IPT per thread), ordered by Poisson sampler branch as in ccd_kernel
    // (the draws do not depend on the order); item j of thread t is pass
    // entry j * blockDim + t, in virtual warp j * nwarps + warp
    for (int base = 0; base < P; base += IPT * nthr) {
        int qi[IPT];
        float fi[IPT];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const int q = base + j * nthr + tid;
            const bool valid = q < P;
            float f = 0.f;
            if (valid) {
                const int r = q / wc, c = q - r * wc;
                const int e = (i * npx + r) * a.side + j0 * npx + c;
                const float v = I[e] * scale;
                I[e] = v;
                f = __fadd_rn(integ[e], __fmul_rn(v, p.rate));           // ccd.py:205
                if (p.qe != 1.0f) f = __fmul_rn(f, p.qe);                  // ccd.py:282-287
                if (p.qe_map) f = __fmul_rn(f, p.qe_map[e]);
                f = __fadd_rn(f, p.bg_plus_dark);                           // ccd.py:220-221
            }
            qi[j] = valid ? q : -1;
            fi[j] = f;
        }
        if (p.photon_noise) {
            unsigned int bal[IPT];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                bal[j] = __ballot_sync(0xffffffffu, qi[j] >= 0 && fi[j] < 10.0f);
                if (lane == 0) s_small[j * nwarps + warp] = __popc(bal[j]);
            }
            __syncthreads();
            int total = 0;
            for (int k = 0; k < IPT * nwarps; ++k) total += s_small[k];
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const int vw = j * nwarps + warp;
                int before = 0;
                for (int k = 0; k < vw; ++k) before += s_small[k];
                const bool small = (bal[j] >> lane) & 1u;
                const int rank = __popc(bal[j] & ((1u << lane) - 1u));
                const int pos = small ? before + rank : total + (vw * 32 - before) + (lane - rank);
                s_idx[pos] = qi[j];
                s_mean[pos] = fi[j];
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                qi[j] = s_idx[j * nthr + tid];
                fi[j] = s_mean[j * nthr + tid];
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            if (qi[j] < 0) continue;
            const int r = qi[j] / wc, c = qi[j] - r * wc;
            const int e = (i * npx + r) * a.side + j0 * npx + c;
            const float v = ccd_sample(p, fi[j], e, frame, slot.photon_seed, slot.readout_seed, p.n_pixels, logfact,
                                       inv_gain, gain_pow2);
            pix[e] = v;
            integ[e] = 0.0f;                                          // ccd.py:216
            tile[r * tld + c] = v;
        }
    }
    __syncthreads();

    // CoG sums, one warp per lenslet, in slopec_sums_kernel's lane order
    for (int k = warp; k < w; k += nwarps) {
        const int s = a.lenslet_subap[i * a.n + j0 + k];
        if (s >= 0) {
            float fl = 0.f, t = 0.f, x = 0.f, y = 0.f;
            for (int e = lane; e < npx * npx; e += 32) {
                const int r = e / npx, c = e - r * npx;
                const float v = tile[r * tld + k * npx + c];
                fl += v;
                float wv = v - a.thr;                 // pixels -= thr; clamp < 0 -> 0
                wv = wv < 0.f ? 0.f : wv;
                t = fmaf(wv, a.mw[e], t);
                x = fmaf(wv, a.xw[e], x);
                y = fmaf(wv, a.yw[e], y);
            }
            fl = sb::warp_sum(fl);
            t = sb::warp_sum(t);
            x = sb::warp_sum(x);
            y = sb::warp_sum(y);
            if (lane == 0) {
                flux[s] = fl;
                tot[s] = t;
                sxn[s] = x;
                syn[s] = y;
                const float fac = 1.0f / t;
                slopes[s] = x * fac;
                slopes[a.n_valid + s] = y * fac;
            }
        }
    }

    // the last CTA sharing the frame state advances it; the last CTA of the
    // realisation applies the flux cut-off
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        if (!slot.real_done) {
            s_last = s_group_last = atomicAdd(&p.state->blocks_done, 1u) == slot.group_ctas - 1u;
        } else {
            s_last = atomicAdd(slot.real_done, 1u) == slot.real_ctas - 1u;
            s_group_last = atomicAdd(&p.state->blocks_done, 1u) == slot.group_ctas - 1u;
        }
    }
    __syncthreads();
    if (s_group_last) {
        __threadfence();
        if (tid == 0) {
            vs->n_integrated = 0;
            vs->frame_index = frame + 1;
            vs->blocks_done = 0u;
        }
    }
    if (!s_last || !slot.cutoff) return;
    __threadfence();
    if (slot.real_done && tid == 0) *slot.real_done = 0u;
    chain_cutoff(tot, sxn, syn, slopes, a.n_valid, dred);
}

// lenslet rows row0 .. row0 + gridDim.y - 1 of a system split by rows; the
// cut-off waits for every band (sb_slopec_cutoff)
__global__ void __launch_bounds__(kChainMaxThreads) ccd_slopec_rows_kernel(ChainArgs a, int row0) {
    const unsigned int ctas = gridDim.x * gridDim.y;
    chain_body<1>(a, ChainOff{0, 0, 0, 0, 0}, blockIdx.x * kChainLenses, kChainLenses, blockIdx.y + row0,
               ChainSlot{nullptr, nullptr, nullptr, ctas, ctas, 0});
}

__global__ void __launch_bounds__(kChainSumThreads) slopec_cutoff_kernel(const float *tot, const float *sxn,
                                                                        const float *syn, float *slopes, int nv) {
    __shared__ double dred[33];
    chain_cutoff(tot, sxn, syn, slopes, nv, dred);
}

__global__ void __launch_bounds__(kChainMaxThreads) sh_ccd_slopec_kernel(ChainArgs a) {
    const unsigned int ctas = gridDim.x * gridDim.y;
    chain_body<1>(a, ChainOff{0, 0, 0, 0, 0}, blockIdx.x * kChainLenses, kChainLenses, blockIdx.y,
               ChainSlot{nullptr, nullptr, nullptr, ctas, ctas, 1});
}

}  // namespace

extern "C" size_t sb_ccd_binned_scratch_bytes(int rows, int cols, int binning) {
    if (rows < 1 || cols < 1 || binning < 1 || rows % binning || cols % binning) return 0;
    const size_t n_out = (size_t)(rows / binning) * (cols / binning);
    return ((n_out * sizeof(float) + 255) & ~(size_t)255) + 2 * kBinBlocks * sizeof(double);
}

extern "C" int sb_ccd_step_binned(const sb_ccd_params *p, int rows, int cols, int binning, const float *intensity,
                                  float *integrated, float *pixels, void *scratch, size_t scratch_bytes,
                                  void *stream) {
    sb::clear_error();
    if (!p || !intensity || !integrated || !pixels || !p->state)
        return sb::fail(SB_EINVAL, "sb_ccd_step_binned: null pointer");
    if (p->frames_per_read < 1 || rows < 1 || cols < 1 || binning < 1 || p->n_pixels != rows * cols)
        return sb::fail(SB_EINVAL, "sb_ccd_step_binned: bad sizes");
    if (rows % binning || cols % binning)
        return sb::fail(SB_ESHAPE, "sb_ccd_step_binned: %d x %d frame not divisible by binning %d", rows, cols, binning);
    if (p->photon_noise && !(p->adu_gain > 0.f))
        return sb::fail(SB_EINVAL, "sb_ccd_step_binned: ADU gain must be > 0");
    const size_t need = sb_ccd_binned_scratch_bytes(rows, cols, binning);
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "sb_ccd_step_binned: scratch needs %zu bytes", need);
    const int orow = rows / binning, ocol = cols / binning, n_out = orow * ocol, n_full = rows * cols;
    float *binned = static_cast<float *>(scratch);
    double *part = reinterpret_cast<double *>(static_cast<char *>(scratch) +
                                              (((size_t)n_out * sizeof(float) + 255) & ~(size_t)255));
    cudaStream_t st = sb::as_stream(stream);
    int nb = (n_full + 255) / 256;
    nb = nb < 1 ? 1 : (nb > 1184 ? 1184 : nb);
    ccd_integrate_kernel<<<nb, 256, 0, st>>>(*p, intensity, integrated, n_full);
    int rc = sb::check_launch("ccd_integrate_kernel");
    if (rc) return rc;
    int ns = (n_out + 255) / 256;
    ns = ns < 1 ? 1 : (ns > kBinBlocks ? kBinBlocks : ns);
    ccd_bin_sums_kernel<<<ns, 256, 0, st>>>(*p, integrated, cols, binning, orow, ocol, binned, part);
    rc = sb::check_launch("ccd_bin_sums_kernel");
    if (rc) return rc;
    int nn = (n_full + kCcdThreads - 1) / kCcdThreads;
    nn = nn < 1 ? 1 : (nn > 1184 ? 1184 : nn);
    ccd_bin_noise_kernel<<<nn, kCcdThreads, 0, st>>>(*p, binned, part, ns, binning, n_out, pixels, integrated,
                                                     n_full);
    return sb::check_launch("ccd_bin_noise_kernel");
}

extern "C" int sb_ccd_step(const sb_ccd_params *p, const float *intensity, float *integrated, float *pixels,
                           void *stream) {
    sb::clear_error();
    if (!p || !intensity || !integrated || !pixels || !p->state)
        return sb::fail(SB_EINVAL, "sb_ccd_step: null pointer");
    if (p->n_pixels < 0 || p->frames_per_read < 1) return sb::fail(SB_EINVAL, "sb_ccd_step: bad sizes");
    if (p->photon_noise && !(p->adu_gain > 0.f)) return sb::fail(SB_EINVAL, "sb_ccd_step: ADU gain must be > 0");
    int nblk = (p->n_pixels + 255) / 256;
    nblk = nblk < 1 ? 1 : (nblk > 1184 ? 1184 : nblk);
    ccd_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(*p, intensity, integrated, pixels, nullptr, nullptr,
                                                        p->n_pixels);
    return sb::check_launch("ccd_kernel");
}

extern "C" int sb_ccd_step_batched(const sb_ccd_params *p, const uint64_t *photon_seeds,
                                   const uint64_t *readout_seeds, int n_batch, const float *intensity,
                                   float *integrated, float *pixels, void *stream) {
    sb::clear_error();
    if (!p || !photon_seeds || !readout_seeds || !intensity || !integrated || !pixels || !p->state || n_batch < 1)
        return sb::fail(SB_EINVAL, "sb_ccd_step_batched: null pointer");
    if (p->n_pixels < 1 || p->frames_per_read < 1 || (long long)p->n_pixels * n_batch > 0x7fffffffLL)
        return sb::fail(SB_EINVAL, "sb_ccd_step_batched: bad sizes");
    if (p->photon_noise && !(p->adu_gain > 0.f))
        return sb::fail(SB_EINVAL, "sb_ccd_step_batched: ADU gain must be > 0");
    sb_ccd_params q = *p;
    q.n_pixels = p->n_pixels * n_batch;
    int nblk = (q.n_pixels + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    ccd_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(q, intensity, integrated, pixels, photon_seeds, readout_seeds,
                                                        p->n_pixels);
    return sb::check_launch("ccd_kernel");
}

extern "C" int sb_philox_raw(uint32_t key0, uint32_t key1, uint32_t c1, uint32_t c2, uint32_t c3, int n_blocks,
                             uint32_t *out, void *stream) {
    sb::clear_error();
    if (!out || n_blocks < 0) return sb::fail(SB_EINVAL, "sb_philox_raw: bad args");
    if (n_blocks == 0) return SB_OK;
    int nblk = (n_blocks + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    philox_raw_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(key0, key1, c1, c2, c3, n_blocks, out);
    return sb::check_launch("philox_raw_kernel");
}

extern "C" size_t sb_slopec_scratch_bytes(const sb_slopec_plan *pl) {
    if (!pl || pl->n_subaps < 0) return 0;
    const size_t nparts = ((size_t)pl->n_subaps + 7) / 8;
    return ((size_t)(3 * pl->n_subaps + nparts) * sizeof(float) + 255) & ~(size_t)255;
}

namespace {

int slopec_impl(const char *who, const sb_slopec_plan *pl, const float *pixels, long long frame_stride, float *slopes,
                int slopes_stride, float *flux, int flux_stride, int n_batch, void *scratch, size_t scratch_bytes,
                void *stream) {
    if (!pl || !pixels || !slopes || !flux || !pl->idxs || !pl->xw || !pl->yw || !pl->mw)
        return sb::fail(SB_EINVAL, "%s: null pointer", who);
    if (pl->n_subaps < 1 || pl->npx2 < 1 || n_batch < 1 || n_batch > 65535)
        return sb::fail(SB_EINVAL, "%s: empty sub-aperture set", who);
    const size_t one = sb_slopec_scratch_bytes(pl);
    const size_t need = one * (size_t)n_batch;
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "%s: scratch needs %zu bytes, got %zu", who, need, scratch_bytes);
    // per realisation: tot, sxn, syn (n_subaps each) in one region, then the block partials
    const int n = pl->n_subaps;
    const int work_stride = 3 * n;
    float *tot = static_cast<float *>(scratch);
    float *sxn = tot + n;
    float *syn = sxn + n;
    cudaStream_t st = sb::as_stream(stream);
    const int warps_per_block = 8;
    const int nblk = (n + warps_per_block - 1) / warps_per_block;
    float *part = tot + (size_t)work_stride * n_batch;
    slopec_sums_kernel<<<dim3(nblk, n_batch), 32 * warps_per_block, 0, st>>>(*pl, pixels, flux, tot, sxn, syn, part,
                                                                            frame_stride, flux_stride, work_stride);
    int rc = sb::check_launch("slopec_sums_kernel");
    if (rc) return rc;
    int nb2 = (n + 255) / 256;
    nb2 = nb2 > 148 ? 148 : nb2;
    slopec_finish_kernel<<<dim3(nb2, n_batch), 256, 0, st>>>(n, tot, sxn, syn, part, nblk, slopes, slopes_stride,
                                                             work_stride, pl->mult);
    return sb::check_launch("slopec_finish_kernel");
}

}  // namespace

extern "C" int sb_slopec(const sb_slopec_plan *pl, const float *pixels, float *slopes, float *flux, void *scratch,
                         size_t scratch_bytes, void *stream) {
    sb::clear_error();
    return slopec_impl("sb_slopec", pl, pixels, 0, slopes, 0, flux, 0, 1, scratch, scratch_bytes, stream);
}

extern "C" int sb_slopec_batched(const sb_slopec_plan *pl, const float *pixels, long long frame_stride, float *slopes,
                                 int slopes_stride, float *flux, int flux_stride, int n_batch, void *scratch,
                                 size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (pl && (slopes_stride < 2 * pl->n_subaps || flux_stride < pl->n_subaps || frame_stride < 1))
        return sb::fail(SB_EINVAL, "sb_slopec_batched: strides smaller than one realisation");
    return slopec_impl("sb_slopec_batched", pl, pixels, frame_stride, slopes, slopes_stride, flux, flux_stride,
                       n_batch, scratch, scratch_bytes, stream);
}

extern "C" size_t sb_sh_ccd_slopec_scratch_bytes(const sb_sh_plan *sh, int n_valid) {
    const size_t a = sb_sh_scratch_bytes(sh);
    if (!a || n_valid < 1) return 0;
    return a + ((3 * (size_t)n_valid * sizeof(float) + 255) & ~(size_t)255);
}

extern "C" int sb_sh_ccd_slopec(const sb_sh_plan *sh, int dft_mode, const float *A, const float *phase_nm,
                                const float *A_norm, int n_norm, const float *mirror_A, const float *mirror_phase,
                                float *field_A, float *field_phase, float photon_scale, float *intensity,
                                const sb_ccd_params *ccd, float *integrated, float *pixels,
                                const sb_slopec_plan *slopec, const int32_t *lenslet_subap, float *slopes,
                                float *flux, void *scratch, size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!sh || !A || !phase_nm || !A_norm || !intensity || !ccd || !ccd->state || !integrated || !pixels ||
        !slopec || !slopec->xw || !slopec->yw || !slopec->mw || !lenslet_subap || !slopes || !flux)
        return sb::fail(SB_EINVAL, "sb_sh_ccd_slopec: null pointer");
    if (dft_mode != 0 && dft_mode != 1) return sb::fail(SB_EINVAL, "sb_sh_ccd_slopec: dft_mode must be 0 or 1");
    const int n = sh->n_lenses, npx = sh->subap_npx, side = n * npx;
    if (n < 1 || npx < 1 || npx > kChainMaxNpx)
        return sb::fail(SB_ESHAPE, "sb_sh_ccd_slopec: %d detector pixels per sub-aperture (1..%d supported)", npx,
                        kChainMaxNpx);
    if (ccd->frames_per_read != 1)
        return sb::fail(SB_EUNSUPPORTED, "sb_sh_ccd_slopec: the detector must read out every loop step");
    if (ccd->n_pixels != side * side)
        return sb::fail(SB_EINVAL, "sb_sh_ccd_slopec: detector of %d pixels for a %d x %d frame", ccd->n_pixels, side,
                        side);
    if (ccd->photon_noise && !(ccd->adu_gain > 0.f))
        return sb::fail(SB_EINVAL, "sb_sh_ccd_slopec: ADU gain must be > 0");
    if (slopec->npx2 != npx * npx || slopec->n_subaps < 1 || slopec->n_subaps > n * n)
        return sb::fail(SB_EINVAL, "sb_sh_ccd_slopec: slope plan of %d sub-apertures x %d pixels", slopec->n_subaps,
                        slopec->npx2);
    if (slopec->thr_pedestal || slopec->thr_ratio > 0.f || slopec->window || slopec->mult != 0.f)
        return sb::fail(SB_EUNSUPPORTED, "sb_sh_ccd_slopec: the slope options beyond thr go through sb_slopec");
    const size_t need = sb_sh_ccd_slopec_scratch_bytes(sh, slopec->n_subaps);
    if (!scratch || need == 0 || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "sb_sh_ccd_slopec: scratch needs %zu bytes, got %zu", need, scratch_bytes);
    int nparts = 0;
    const size_t sh_bytes = sb_sh_scratch_bytes(sh);
    int rc = sb::sh_forward_unnormalised("sb_sh_ccd_slopec", sh, A, phase_nm, A_norm, n_norm, intensity, scratch,
                                         sh_bytes, stream, dft_mode, &nparts, mirror_A, mirror_phase, field_A,
                                         field_phase);
    if (rc) return rc;
    ChainArgs a;
    a.p = *ccd;
    a.part_I = static_cast<const float *>(scratch);
    a.part_A = static_cast<const float *>(scratch) + nparts;
    a.nparts = nparts;
    a.photon_scale = photon_scale;
    a.I = intensity;
    a.integ = integrated;
    a.pix = pixels;
    a.n = n;
    a.npx = npx;
    a.side = side;
    a.lenslet_subap = lenslet_subap;
    a.n_valid = slopec->n_subaps;
    a.thr = slopec->thr;
    a.xw = slopec->xw;
    a.yw = slopec->yw;
    a.mw = slopec->mw;
    a.slopes = slopes;
    a.flux = flux;
    a.tot = reinterpret_cast<float *>(static_cast<char *>(scratch) + sh_bytes);
    a.sxn = a.tot + a.n_valid;
    a.syn = a.sxn + a.n_valid;
    const dim3 grid((n + kChainLenses - 1) / kChainLenses, n);
    sh_ccd_slopec_kernel<<<grid, chain_threads(npx), 0, sb::as_stream(stream)>>>(a);
    return sb::check_launch("sh_ccd_slopec_kernel");
}

// ---------------------------------------------------------------------------
// Monte-Carlo step, stage 5: the chain of every realisation of every group in
// one launch.  A CTA finds its group, realisation and lenslet block from the
// flat block index; realisation b draws with its own seeds, keeps its own
// completion counter (the flux cut-off), and the group's CTAs share the
// group's frame state, as sb_ccd_step_batched does.
// ---------------------------------------------------------------------------
namespace {

constexpr int kMcChainIpt = 1;          // pixels per thread and pass in the Monte-Carlo detector stage (2 measured slower)

struct McChainGroup {
    ChainArgs a;                     // realisation 0
    long long frame_stride;
    const uint64_t *photon_seeds, *readout_seeds;
    unsigned int *done;              // [n_batch] realisation counters
    int gx, gy, slopes_stride, flux_stride;
    int lpc;                         // lenslets per CTA (a lenslet row, or as much of it as the tile holds)
};

struct McChainArgs {
    int n_groups;
    McChainGroup g[sb::kMcMaxGroups];
    int blk0[sb::kMcMaxGroups + 1];
};

struct McChainBlob {
    McChainArgs args;
    int blocks, threads;
};

__global__ void __launch_bounds__(kChainSumThreads, 6) mc_chain_kernel(McChainArgs m) {
    // the group's arguments staged in shared memory: read there on use, not
    // held in registers
    __shared__ __align__(16) McChainGroup G;
    static_assert(sizeof(McChainGroup) % 4 == 0, "staged as words");
    const int bi = blockIdx.x;
    int g = 0;
    while (g + 1 < m.n_groups && bi >= m.blk0[g + 1]) ++g;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&m.g[g]);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&G);
        for (int k = threadIdx.x; k < (int)(sizeof(McChainGroup) / 4); k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int per = G.gx * G.gy, local = bi - m.blk0[g];
    const int b = local / per, rem = local - b * per;
    const ChainOff off{(long long)b * G.frame_stride, (size_t)b * G.a.nparts, (size_t)b * G.slopes_stride,
                       (size_t)b * G.flux_stride, (size_t)b * 3 * G.a.n_valid};
    const ChainSlot slot{G.photon_seeds + b, G.readout_seeds + b, G.done + b, (unsigned int)per,
                         (unsigned int)(m.blk0[g + 1] - m.blk0[g]), 1};
    chain_body<kMcChainIpt>(G.a, off, (rem % G.gx) * G.lpc, G.lpc, rem / G.gx, slot);
}

}  // namespace

namespace sb {

size_t mc_chain_workspace(const sb_mc_group *gs, int n) {
    size_t b = 0;
    for (int g = 0; g < n; ++g)
        b += mc_align((size_t)gs[g].n_batch * 3 * gs[g].slopec.n_subaps * sizeof(float)) +
             mc_align((size_t)gs[g].n_batch * sizeof(unsigned int));
    return b;
}

int mc_chain_prepare(const sb_mc_group *gs, int n, const McShParts &parts, void *ws, McBlob &blob) {
    static_assert(sizeof(McChainBlob) <= sizeof(McBlob), "detector stage arguments exceed the blob");
    static_assert(sizeof(McChainArgs) <= 4096, "kernel arguments above 4 KB");
    const char *who = "sb_mc_create";
    McChainBlob *B = new (blob.b) McChainBlob();
    B->args.n_groups = n;
    unsigned char *w = static_cast<unsigned char *>(ws);
    // 256 threads: several passes over a block's pixels when npx > 8 (the
    // sums do not depend on the CTA size)
    int blocks = 0, threads = kChainSumThreads;
    for (int g = 0; g < n; ++g) {
        const sb_mc_group &G = gs[g];
        const sb_ccd_params &c = G.ccd;
        const sb_slopec_plan &sl = G.slopec;
        const int nl = G.sh.n_lenses, npx = G.sh.subap_npx, side = nl * npx;
        if (!c.state || !G.integrated || !G.pixels || !G.photon_seeds || !G.readout_seeds || !sl.xw || !sl.yw ||
            !sl.mw || !G.lenslet_subap || !G.slopes || !G.flux)
            return fail(SB_EINVAL, "%s: group %d: null detector / slope pointer", who, g);
        if (npx < 1 || npx > kChainMaxNpx)
            return fail(SB_ESHAPE, "%s: group %d: %d pixels per sub-aperture (1..%d)", who, g, npx, kChainMaxNpx);
        if (c.frames_per_read != 1 || c.n_pixels != side * side)
            return fail(SB_EUNSUPPORTED, "%s: group %d: the detector must read a %d x %d frame every step", who, g,
                        side, side);
        if (c.photon_noise && !(c.adu_gain > 0.f)) return fail(SB_EINVAL, "%s: group %d: ADU gain <= 0", who, g);
        // the group's CTAs count down on its own frame state
        for (int h = 0; h < g; ++h)
            if (gs[h].ccd.state == c.state)
                return fail(SB_EINVAL, "%s: groups %d and %d share a detector frame state", who, h, g);
        if (sl.npx2 != npx * npx || sl.n_subaps < 1 || sl.n_subaps > nl * nl)
            return fail(SB_EINVAL, "%s: group %d: slope plan of %d sub-apertures x %d pixels", who, g, sl.n_subaps,
                        sl.npx2);
        if (sl.thr_pedestal || sl.thr_ratio > 0.f || sl.window || sl.mult != 0.f)
            return fail(SB_EUNSUPPORTED, "%s: group %d: slope options beyond thr are not in the step", who, g);
        if (G.slopes_stride < 2 * sl.n_subaps || G.flux_stride < sl.n_subaps)
            return fail(SB_EINVAL, "%s: group %d: slope / flux strides below one realisation", who, g);
        McChainGroup &q = B->args.g[g];
        ChainArgs &a = q.a;
        a.p = c;
        a.part_I = parts.part_I[g];
        a.part_A = parts.part_A[g];
        a.nparts = parts.nparts[g];
        a.photon_scale = G.photon_scale;
        a.I = G.intensity;
        a.integ = G.integrated;
        a.pix = G.pixels;
        a.n = nl;
        a.npx = npx;
        a.side = side;
        a.lenslet_subap = G.lenslet_subap;
        a.n_valid = sl.n_subaps;
        a.thr = sl.thr;
        a.xw = sl.xw;
        a.yw = sl.yw;
        a.mw = sl.mw;
        a.slopes = G.slopes;
        a.flux = G.flux;
        a.tot = reinterpret_cast<float *>(w);
        a.sxn = a.tot + a.n_valid;
        a.syn = a.sxn + a.n_valid;
        w += mc_align((size_t)G.n_batch * 3 * sl.n_subaps * sizeof(float));
        q.done = reinterpret_cast<unsigned int *>(w);
        w += mc_align((size_t)G.n_batch * sizeof(unsigned int));
        q.frame_stride = G.frame_stride;
        q.photon_seeds = G.photon_seeds;
        q.readout_seeds = G.readout_seeds;
        // whole lenslet rows per CTA where the tile holds them: the per-CTA
        // work (normalisation sums, completion counters) is paid once per
        // row and the pixel passes run over the row
        q.lpc = kChainTile / (npx * npx) < nl ? kChainTile / (npx * npx) : nl;
        q.gx = (nl + q.lpc - 1) / q.lpc;
        q.gy = nl;
        q.slopes_stride = G.slopes_stride;
        q.flux_stride = G.flux_stride;
        B->args.blk0[g] = blocks;
        blocks += q.gx * q.gy * G.n_batch;
    }
    B->args.blk0[n] = blocks;
    B->blocks = blocks;
    B->threads = threads;
    return SB_OK;
}

int mc_chain_launch(const McBlob &blob, cudaStream_t st) {
    const McChainBlob *B = reinterpret_cast<const McChainBlob *>(blob.b);
    mc_chain_kernel<<<B->blocks, B->threads, 0, st>>>(B->args);
    return check_launch("mc_chain_kernel");
}

}  // namespace sb

extern "C" int sb_ccd_slopec_rows(const sb_sh_plan *sh, const float *parts, int nparts, float photon_scale, int row0,
                                  int n_rows, float *intensity, const sb_ccd_params *ccd, float *integrated,
                                  float *pixels, const sb_slopec_plan *slopec, const int32_t *lenslet_subap,
                                  float *slopes, float *flux, float *work, void *stream) {
    sb::clear_error();
    const char *who = "sb_ccd_slopec_rows";
    if (!sh || !parts || !intensity || !ccd || !ccd->state || !integrated || !pixels || !slopec || !slopec->xw ||
        !slopec->yw || !slopec->mw || !lenslet_subap || !slopes || !flux || !work)
        return sb::fail(SB_EINVAL, "%s: null pointer", who);
    const int n = sh->n_lenses, npx = sh->subap_npx, side = n * npx;
    if (n < 1 || npx < 1 || npx > kChainMaxNpx || nparts < 1)
        return sb::fail(SB_ESHAPE, "%s: %d detector pixels per sub-aperture (1..%d supported)", who, npx, kChainMaxNpx);
    if (row0 < 0 || n_rows < 1 || row0 + n_rows > n)
        return sb::fail(SB_EINVAL, "%s: lenslet rows %d..%d of %d", who, row0, row0 + n_rows - 1, n);
    if (ccd->frames_per_read != 1 || ccd->n_pixels != side * side)
        return sb::fail(SB_EUNSUPPORTED, "%s: the detector must read a %d x %d frame every step", who, side, side);
    if (ccd->photon_noise && !(ccd->adu_gain > 0.f)) return sb::fail(SB_EINVAL, "%s: ADU gain must be > 0", who);
    if (slopec->npx2 != npx * npx || slopec->n_subaps < 1 || slopec->n_subaps > n * n)
        return sb::fail(SB_EINVAL, "%s: slope plan of %d sub-apertures x %d pixels", who, slopec->n_subaps,
                        slopec->npx2);
    if (slopec->thr_pedestal || slopec->thr_ratio > 0.f || slopec->window || slopec->mult != 0.f)
        return sb::fail(SB_EUNSUPPORTED, "%s: the slope options beyond thr go through sb_slopec", who);
    ChainArgs a;
    a.p = *ccd;
    a.part_I = parts;
    a.part_A = parts + nparts;
    a.nparts = nparts;
    a.photon_scale = photon_scale;
    a.I = intensity;
    a.integ = integrated;
    a.pix = pixels;
    a.n = n;
    a.npx = npx;
    a.side = side;
    a.lenslet_subap = lenslet_subap;
    a.n_valid = slopec->n_subaps;
    a.thr = slopec->thr;
    a.xw = slopec->xw;
    a.yw = slopec->yw;
    a.mw = slopec->mw;
    a.slopes = slopes;
    a.flux = flux;
    a.tot = work;
    a.sxn = work + a.n_valid;
    a.syn = a.sxn + a.n_valid;
    const dim3 grid((n + kChainLenses - 1) / kChainLenses, n_rows);
    ccd_slopec_rows_kernel<<<grid, chain_threads(npx), 0, sb::as_stream(stream)>>>(a, row0);
    return sb::check_launch("ccd_slopec_rows_kernel");
}

extern "C" int sb_slopec_cutoff(const float *tot, const float *sxn, const float *syn, int n_valid, float *slopes,
                                void *stream) {
    sb::clear_error();
    if (!tot || !sxn || !syn || !slopes || n_valid < 1) return sb::fail(SB_EINVAL, "sb_slopec_cutoff: bad args");
    slopec_cutoff_kernel<<<1, kChainSumThreads, 0, sb::as_stream(stream)>>>(tot, sxn, syn, slopes, n_valid);
    return sb::check_launch("slopec_cutoff_kernel");
}

extern "C" size_t sb_ccd_cte_scratch_bytes(int side) {
    if (side < 1) return 0;
    return 2 * (((size_t)side * side * sizeof(float) + 255) & ~(size_t)255);
}

extern "C" int sb_ccd_step_cte(const sb_ccd_params *p, int side, const float *cte0, const float *cte1,
                               const float *intensity, float *integrated, float *pixels, void *scratch,
                               size_t scratch_bytes, void *stream) {
    sb::clear_error();
    if (!p || !p->state || !cte0 || !cte1 || !intensity || !integrated || !pixels)
        return sb::fail(SB_EINVAL, "sb_ccd_step_cte: null pointer");
    if (side < 1 || p->n_pixels != side * side || p->frames_per_read < 1)
        return sb::fail(SB_EINVAL, "sb_ccd_step_cte: a square frame of side x side pixels is needed");
    if (p->photon_noise && !(p->adu_gain > 0.f)) return sb::fail(SB_EINVAL, "sb_ccd_step_cte: ADU gain must be > 0");
    const size_t need = sb_ccd_cte_scratch_bytes(side);
    if (!scratch || scratch_bytes < need)
        return sb::fail(SB_ESCRATCH, "sb_ccd_step_cte: scratch needs %zu bytes", need);
    float *f0 = static_cast<float *>(scratch);
    float *f1 = reinterpret_cast<float *>(static_cast<char *>(scratch) + need / 2);
    cudaStream_t st = sb::as_stream(stream);
    int nb = (p->n_pixels + 255) / 256;
    nb = nb > 1184 ? 1184 : nb;
    ccd_cte_frame_kernel<<<nb, 256, 0, st>>>(*p, intensity, integrated, f0);
    int rc = sb::check_launch("ccd_cte_frame_kernel");
    if (rc) return rc;
    const dim3 g((side + 15) / 16, (side + 15) / 16);
    ccd_cte_matmul_kernel<<<g, 256, 0, st>>>(*p, cte0, f0, f1, side, side, side);     // M0 * frame
    rc = sb::check_launch("ccd_cte_matmul_kernel");
    if (rc) return rc;
    ccd_cte_matmul_kernel<<<g, 256, 0, st>>>(*p, f1, cte1, f0, side, side, side);     // ... * M1
    rc = sb::check_launch("ccd_cte_matmul_kernel");
    if (rc) return rc;
    ccd_cte_noise_kernel<<<nb, kCcdThreads, 0, st>>>(*p, f0, pixels);
    return sb::check_launch("ccd_cte_noise_kernel");
}
