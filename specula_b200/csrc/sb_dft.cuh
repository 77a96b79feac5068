// Warp-level small complex matrix products used by the SH forward model and
// its adjoint: one warp computes C = A * B for compile-time sizes, each lane
// holding an RB x CB register block of C (operands loaded once per k and
// reused RB*CB times).
#pragma once

namespace sb {

// cost of an RB x CB block for an M x N output (infeasible: huge)
__host__ __device__ constexpr int blk_cost(int M, int N, int rb, int cb) {
    return (M % rb || N % cb || (M / rb) * (N / cb) > 32) ? 1 << 20 : rb * cb * 64 + rb + cb;
}
__host__ __device__ constexpr int best_rb(int M, int N) {
    int best = 1, bestc = 1 << 30;
    for (int rb = 1; rb <= M; ++rb)
        for (int cb = 1; cb <= N; ++cb)
            if (blk_cost(M, N, rb, cb) < bestc) { bestc = blk_cost(M, N, rb, cb); best = rb; }
    return best;
}
__host__ __device__ constexpr int best_cb(int M, int N) {
    int best = 1, bestc = 1 << 30;
    for (int rb = 1; rb <= M; ++rb)
        for (int cb = 1; cb <= N; ++cb)
            if (blk_cost(M, N, rb, cb) < bestc) { bestc = blk_cost(M, N, rb, cb); best = cb; }
    return best;
}

// C(M x N) = A(M x K) * B(K x N), complex, A(i,k) = A[i*SAI + k*SAK],
// B(k,j) = B[k*SBK + j]; each result goes to store(i, j, re, im).
template <int M, int N, int K, int SAI, int SAK, int SBK, typename Store>
__device__ __forceinline__ void warp_cgemm(const float2 *A, const float2 *B, int lane, Store store) {
    constexpr int RB = best_rb(M, N), CB = best_cb(M, N);
    constexpr int NBC = N / CB;
    if (lane < (M / RB) * NBC) {
        const int i0 = (lane / NBC) * RB, j0 = (lane % NBC) * CB;
        float xr[RB][CB], xi[RB][CB];
#pragma unroll
        for (int i = 0; i < RB; ++i)
#pragma unroll
            for (int j = 0; j < CB; ++j) xr[i][j] = xi[i][j] = 0.f;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            float2 av[RB], bv[CB];
#pragma unroll
            for (int i = 0; i < RB; ++i) av[i] = A[(i0 + i) * SAI + k * SAK];
#pragma unroll
            for (int j = 0; j < CB; ++j) bv[j] = B[k * SBK + j0 + j];
#pragma unroll
            for (int i = 0; i < RB; ++i)
#pragma unroll
                for (int j = 0; j < CB; ++j) {
                    xr[i][j] = fmaf(av[i].x, bv[j].x, fmaf(-av[i].y, bv[j].y, xr[i][j]));
                    xi[i][j] = fmaf(av[i].x, bv[j].y, fmaf(av[i].y, bv[j].x, xi[i][j]));
                }
        }
#pragma unroll
        for (int i = 0; i < RB; ++i)
#pragma unroll
            for (int j = 0; j < CB; ++j) store(i0 + i, j0 + j, xr[i][j], xi[i][j]);
    }
}

}  // namespace sb
