// Shared helpers of the specula_b200 CUDA library: status reporting, launch
// checks and small device reductions.  Compiled for sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdint.h>

#include "specula_b200.h"

namespace sb {

// Record a failure message for sb_last_error() and return the status.
int fail(int status, const char *fmt, ...);
void clear_error();
// read and clear the timeout flag of the tensor-core SH kernels (0: none, <0: query failed)
int sh_tc_status_take();
// read and clear the timeout flag of the TMA interaction-matrix contraction
int contract_status_take();
// read and clear the timeout flag of the tensor-core PSF
int psf_tc_status_take();
// tile-shape variant registered for (family, key); 0 when none
int tune_lookup(int family, unsigned long long key);
// SH forward without its photon-normalisation launch: the unnormalised frame
// in `intensity`, the per-CTA partial sums at the start of `scratch` (n_parts
// sums of the frame, then n_parts sums of A_norm); *n_parts receives the
// number of CTAs.  mode 0: FP32 DFTs, 1: split-BF16 tensor-core DFTs.
// mirror_A / mirror_phase (FP32 form): the field is A * mirror_A, phase_nm +
// mirror_phase, written to field_A / field_phase when those are given.
int sh_forward_unnormalised(const char *who, const sb_sh_plan *pl, const float *A, const float *phase_nm,
                            const float *A_norm, int n_norm, float *intensity, void *scratch, size_t scratch_bytes,
                            void *stream, int mode, int *n_parts, const float *mirror_A = nullptr,
                            const float *mirror_phase = nullptr, float *field_A = nullptr,
                            float *field_phase = nullptr);

// Check the launch that just happened on this thread.
inline int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    return SB_OK;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kWarp = 32;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum in a fixed order (deterministic); `red` holds >= 32 floats.
// Every thread of the block must call it; the result is valid in thread 0.
__device__ __forceinline__ float block_sum(float v, float *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    float r = 0.f;
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        r = lane < nw ? red[lane] : 0.f;
        r = warp_sum(r);
    }
    return r;
}

// Same in double precision; `red` holds >= 32 doubles.  Result valid in
// every thread (broadcast through shared memory).
__device__ __forceinline__ double block_sum_all_d(double v, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum_d(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double r = lane < nw ? red[lane] : 0.0;
        r = warp_sum_d(r);
        if (lane == 0) red[32] = r;
    }
    __syncthreads();
    double out = red[32];
    __syncthreads();
    return out;
}

}  // namespace sb
