// Adjoint of the noise-free Shack-Hartmann chain and the interaction matrix.
//
// With a linear (noise-free) detector the slopes of a sub-aperture depend
// only on that sub-aperture's phase samples, and the global photon
// normalisation cancels in the centre of gravity (sh.py:426-427 against
// sh_slopec.py:392-404).  So d(slopes)/d(phase) is block-diagonal: per valid
// sub-aperture a 2 x np^2 block.  One warp per sub-aperture recomputes the
// forward model and back-propagates both slope axes:
//   s      = sum_px D w / sum_px D mw           (CoG, thr = 0)
//   dL/dD  = (w - s mw) / tot                   (active sub-apertures only)
//   dL/dI  = R^T (dL/dD) R                      (LCM rebin)
//   dL/dF  = 2 (dL/dI) M F                      (|F|^2 times field stop)
//   dL/dE  = W^H (dL/dF) conj(W)                (pruned DFT, F = W E W^T)
//   dL/dphi = -k Im(conj(dL/dE) E)              (E = A exp(i k phi) T)
// The interaction matrix is then IM[m][j] = scale * sum_px J[j][px] IF[m][px]
// over the pixels of slope j's sub-aperture (sb_intmat_contract): every
// influence-function element is read once.
#include "sb_common.cuh"
#include "sb_dft.cuh"
#include "sb_tma.cuh"

namespace {

struct AdjArgs {
    int n, p, cs, npx, ld;
    float k;
    const float2 *tw;
    const float2 *tilt;
    const float *mask;
    const float *rebin;
    const float *A;
    const float *ph;
    int n_valid;
    const int32_t *lenslet;
    const float *xw, *yw, *mw;
    const float *active;   // NULL: every sub-aperture with flux
    float *tot_out;        // optional [n_valid]: the sub-aperture flux (CoG denominator)
    const float *seed;   // VJP seed [2][n_valid], or NULL for the Jacobian
    float *jac;          // [2][n_valid][P*P] (Jacobian)
    float *grad;         // field-shaped, row stride ld (VJP)
};

// Warps per block so that the static shared memory stays within 48 KB.
__host__ __device__ constexpr int adj_warps(int P, int CS, int NPX) {
    const int shared = 8 * (2 * P * CS + P * P) + 4 * (CS * CS + NPX * CS + 3 * NPX * NPX);
    const int per_warp = 8 * (P * (P + 1) + 2 * CS * CS + CS * P) + 4 * NPX * NPX;
    const int w = (48 * 1024 - shared) / per_warp;
    return w > 8 ? 8 : w;
}

template <int P, int CS, int NPX>
__global__ void __launch_bounds__(256) sh_slopes_adjoint_kernel(AdjArgs a) {
    constexpr int PE = P + 1;
    constexpr int NPX2 = NPX * NPX;
    constexpr int WPB = adj_warps(P, CS, NPX);
    static_assert(WPB >= 1, "sub-aperture too large for the adjoint kernel");
    __shared__ float2 twT[P * CS];   // twT[c][b] = W[b][c]
    __shared__ float2 Wc[CS * P];    // Wc[b][c] = conj(W[b][c])
    __shared__ float2 tilt[P * P];
    __shared__ float mask[CS * CS];
    __shared__ float R[NPX * CS];
    __shared__ float wts[3][NPX2];
    __shared__ float2 Es[WPB][P * PE];
    __shared__ float2 Fs[WPB][CS * CS];
    __shared__ float2 Gs[WPB][CS * CS];
    __shared__ float2 Ys[WPB][CS * P];
    __shared__ float Ds[WPB][NPX2];
    for (int e = threadIdx.x; e < CS * P; e += blockDim.x) {
        const int b = e / P, c = e - b * P;
        const float2 w = a.tw[e];
        twT[c * CS + b] = w;
        Wc[e] = make_float2(w.x, -w.y);
    }
    for (int e = threadIdx.x; e < P * P; e += blockDim.x) tilt[e] = a.tilt[e];
    for (int e = threadIdx.x; e < CS * CS; e += blockDim.x) mask[e] = a.mask[e];
    for (int e = threadIdx.x; e < NPX * CS; e += blockDim.x) R[e] = a.rebin[e];
    for (int e = threadIdx.x; e < NPX2; e += blockDim.x) {
        wts[0][e] = a.xw[e];
        wts[1][e] = a.yw[e];
        wts[2][e] = a.mw[e];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Jacobian: one warp per (sub-aperture, slope axis); VJP: one warp per
    // sub-aperture (a single seeded backward pass)
    const int item = blockIdx.x * WPB + warp;
    const int s = a.seed ? item : item >> 1;
    const int axis = a.seed ? 0 : item & 1;
    if (s >= a.n_valid) return;
    float2 *E = Es[warp], *F = Fs[warp], *Gf = Gs[warp], *Y = Ys[warp];
    float *D = Ds[warp];
    const int L = a.lenslet[s];
    const int li = L / a.n, lj = L - li * a.n;
    const size_t row0 = (size_t)li * P, col0 = (size_t)lj * P;
    // ---- forward (same arithmetic as sh_forward_fixed_kernel) ----
    for (int e = lane; e < P * P; e += 32) {
        const int r = e / P, c = e % P;
        const size_t g = (row0 + r) * (size_t)a.ld + col0 + c;
        const float amp = a.A[g];
        float sn, co;
        sincosf(a.ph[g] * a.k, &sn, &co);
        const float re = co * amp, im = sn * amp;
        const float2 t = tilt[e];
        E[r * PE + c] = make_float2(re * t.x - im * t.y, re * t.y + im * t.x);
    }
    __syncwarp();
    float2 *G = Y;   // P x CS forward intermediate, reused as Y later
    sb::warp_cgemm<P, CS, P, PE, 1, CS>(E, twT, lane, [&](int r, int b, float xr, float xi) {
        G[r * CS + b] = make_float2(xr, xi);
    });
    __syncwarp();
    sb::warp_cgemm<CS, CS, P, 1, CS, CS>(twT, G, lane, [&](int aa, int b, float xr, float xi) {
        F[aa * CS + b] = make_float2(xr, xi);
    });
    __syncwarp();
    // detector pixels of the sub-aperture: D = R (|F|^2 M) R^T
    if constexpr (CS % NPX == 0) {
        // integer rebin factor: BF x BF boxes weighted 1/BF^2 (R holds 1/BF
        // on its band), as in the forward kernel
        constexpr int BF = CS / NPX;
        const float wgt = R[0] * R[0];
        for (int e = lane; e < NPX2; e += 32) {
            const int pp = e / NPX, q = e % NPX;
            float acc = 0.f;
#pragma unroll
            for (int u = 0; u < BF; ++u)
#pragma unroll
                for (int v = 0; v < BF; ++v) {
                    const int i = (pp * BF + u) * CS + q * BF + v;
                    const float2 f = F[i];
                    acc += (f.x * f.x + f.y * f.y) * mask[i];
                }
            D[e] = acc * wgt;
        }
    } else {
        // separable: H = I R^T (CS x NPX, in Gf's storage), D = R H
        float *H = reinterpret_cast<float *>(Gf);
        for (int e = lane; e < CS * NPX; e += 32) {
            const int aa = e / NPX, q = e % NPX;
            float h = 0.f;
#pragma unroll
            for (int b = 0; b < CS; ++b) {
                const float2 f = F[aa * CS + b];
                h = fmaf((f.x * f.x + f.y * f.y) * mask[aa * CS + b], R[q * CS + b], h);
            }
            H[e] = h;
        }
        __syncwarp();
        for (int e = lane; e < NPX2; e += 32) {
            const int pp = e / NPX, q = e % NPX;
            float acc = 0.f;
#pragma unroll
            for (int aa = 0; aa < CS; ++aa) acc = fmaf(R[pp * CS + aa], H[aa * NPX + q], acc);
            D[e] = acc;
        }
    }
    __syncwarp();
    float tot = 0.f, nx = 0.f, ny = 0.f;
    for (int e = lane; e < NPX2; e += 32) {
        tot = fmaf(D[e], wts[2][e], tot);
        nx = fmaf(D[e], wts[0][e], nx);
        ny = fmaf(D[e], wts[1][e], ny);
    }
    tot = sb::warp_sum(tot);
    nx = sb::warp_sum(nx);
    ny = sb::warp_sum(ny);
    if (a.tot_out && axis == 0 && lane == 0) a.tot_out[s] = tot;
    const bool act = (a.active ? a.active[s] != 0.f : true) && tot > 0.f;
    const float inv = act ? 1.0f / tot : 0.f;
    const float sx = nx * inv, sy = ny * inv;
    float vx = 0.f, vy = 0.f;
    if (a.seed) {
        vx = a.seed[s];
        vy = a.seed[a.n_valid + s];
    }
    __syncwarp();
    // ---- backward: one slope axis (Jacobian) or the seeded sum (VJP) ----
    {
        // g = d(seed . slopes)/dD = (w - s mw) / tot, into D (consumed)
        for (int e = lane; e < NPX2; e += 32) {
            const float gx = wts[0][e] - sx * wts[2][e];
            const float gy = wts[1][e] - sy * wts[2][e];
            D[e] = (a.seed ? vx * gx + vy * gy : (axis == 0 ? gx : gy)) * inv;
        }
        __syncwarp();
        if constexpr (CS % NPX == 0) {
            // R^T g R = g[a / BF][b / BF] / BF^2
            constexpr int BF = CS / NPX;
            const float wgt2 = 2.0f * R[0] * R[0];
            for (int e = lane; e < CS * CS; e += 32) {
                const int aa = e / CS, b = e % CS;
                const float2 f = F[e];
                const float gm = wgt2 * D[(aa / BF) * NPX + b / BF] * mask[e];
                Gf[e] = make_float2(gm * f.x, gm * f.y);
            }
        } else {
            // T = g R   (NPX x CS), in Y's storage (free until the first GEMM)
            float *T = reinterpret_cast<float *>(Y);
            for (int e = lane; e < NPX * CS; e += 32) {
                const int pp = e / CS, b = e % CS;
                float t = 0.f;
#pragma unroll
                for (int q = 0; q < NPX; ++q) t = fmaf(D[pp * NPX + q], R[q * CS + b], t);
                T[e] = t;
            }
            __syncwarp();
            // dL/dF = 2 (R^T g R) M F
            for (int e = lane; e < CS * CS; e += 32) {
                const int aa = e / CS, b = e % CS;
                float h = 0.f;
#pragma unroll
                for (int pp = 0; pp < NPX; ++pp) h = fmaf(R[pp * CS + aa], T[pp * CS + b], h);
                const float2 f = F[e];
                const float gm = 2.0f * h * mask[e];
                Gf[e] = make_float2(gm * f.x, gm * f.y);
            }
        }
        __syncwarp();
        // Y = Gf conj(W)   (CS x P)
        sb::warp_cgemm<CS, P, CS, CS, 1, P>(Gf, Wc, lane, [&](int aa, int c, float xr, float xi) {
            Y[aa * P + c] = make_float2(xr, xi);
        });
        __syncwarp();
        // dL/dE = W^H Y   (P x P); A(r, a) = conj(W[a][r]) = Wc[a*P + r];
        // dL/dphi = -k Im(conj(dL/dE) E) = -k (g.x e.y - g.y e.x)
        if (a.seed) {
            sb::warp_cgemm<P, P, CS, 1, P, P>(Wc, Y, lane, [&](int r, int c, float xr, float xi) {
                const float2 e = E[r * PE + c];
                a.grad[(row0 + r) * (size_t)a.ld + col0 + c] = -a.k * (xr * e.y - xi * e.x);
            });
        } else {
            float *out = a.jac + ((size_t)axis * a.n_valid + s) * (P * P);
            sb::warp_cgemm<P, P, CS, 1, P, P>(Wc, Y, lane, [&](int r, int c, float xr, float xi) {
                const float2 e = E[r * PE + c];
                out[r * P + c] = -a.k * (xr * e.y - xi * e.x);
            });
        }
        __syncwarp();
    }
}

struct AdjKernel {
    void (*fn)(AdjArgs);
    int warps;
};

template <int P, int CS, int NPX>
AdjKernel adj_entry() {
    return {sh_slopes_adjoint_kernel<P, CS, NPX>, adj_warps(P, CS, NPX)};
}

AdjKernel adjoint_kernel(int p, int cs, int npx) {
    if (p == 8 && cs == 12 && npx == 6) return adj_entry<8, 12, 6>();
    if (p == 8 && cs == 14 && npx == 8) return adj_entry<8, 14, 8>();
    if (p == 8 && cs == 16 && npx == 8) return adj_entry<8, 16, 8>();
    if (p == 8 && cs == 8 && npx == 8) return adj_entry<8, 8, 8>();
    if (p == 16 && cs == 16 && npx == 8) return adj_entry<16, 16, 8>();   // 2x-resampled 8-px lenslets
    return {nullptr, 0};
}

// IM[m][s] and IM[m][n_valid + s].  CTA = one row of lenslets x a chunk of
// modes; thread x = field column x.  For each mode the CTA reads the np_sub
// field rows of that lenslet row from the influence function (consecutive x
// -> consecutive mirror columns inside a pupil row: coalesced), multiplies
// by the Jacobian (held in registers for the whole chunk), sums the np_sub
// rows in registers and the np_sub columns of each lenslet with shuffles
// inside groups of np_sub lanes.  Every influence-function sample under a
// valid sub-aperture is read exactly once.
constexpr int kContractModes = 16;  // modes per CTA (even)

template <int P>
constexpr int contract_max_threads() { return P >= 16 ? 512 : 1024; }

template <int P>
__global__ void __launch_bounds__(contract_max_threads<P>()) intmat_contract_kernel(
    const float *__restrict__ jac, const float *__restrict__ tot, int n_valid, int n, int field_ld,
    const int32_t *__restrict__ slot, const int32_t *__restrict__ pix2col, const float *__restrict__ IF, int n_modes,
    int ld_if, float scale, float *__restrict__ im) {
    __shared__ double red[33];
    const int x = threadIdx.x;
    const int li = blockIdx.y;
    const int lj = x / P, c = x - lj * P;
    const int s = (lj < n) ? slot[li * n + lj] : -1;
    bool act = s >= 0;
    if (tot) {
        // the CoG cut-off of sh_slopec.py:400: factor = 1/tot, zeroed where
        // factor > 1/(1e-3 * mean(tot)); tot <= 0 is inactive as well
        double part = 0.0;
        for (int e = threadIdx.x; e < n_valid; e += blockDim.x) part += (double)tot[e];
        const double mean = sb::block_sum_all_d(part, red) / n_valid;
        if (act) {
            const float t = tot[s];
            act = t > 0.f && (double)(1.0f / t) <= 1.0 / (mean * 1e-3);
        }
    }
    float jx[P], jy[P];
    int col[P];
#pragma unroll
    for (int rr = 0; rr < P; ++rr) {
        col[rr] = -1;
        jx[rr] = jy[rr] = 0.f;
        if (act) {
            col[rr] = pix2col[(size_t)(li * P + rr) * field_ld + x];
            jx[rr] = jac[(size_t)s * (P * P) + rr * P + c];
            jy[rr] = jac[((size_t)n_valid + s) * (P * P) + rr * P + c];
        }
    }
    const int m0 = blockIdx.x * kContractModes;
    const int m1 = min(n_modes, m0 + kContractModes);
    const size_t ld_im = 2 * (size_t)n_valid;
    for (int m = m0; m < m1; m += 2) {
        // two modes per iteration: 2 P independent loads in flight
        const bool two = m + 1 < m1;
        const float *row0 = IF + (size_t)m * ld_if;
        const float *row1 = IF + (size_t)(two ? m + 1 : m) * ld_if;
        float vx0 = 0.f, vy0 = 0.f, vx1 = 0.f, vy1 = 0.f;
#pragma unroll
        for (int rr = 0; rr < P; ++rr) {
            const bool in = col[rr] >= 0;
            const float f0 = in ? __ldg(row0 + col[rr]) : 0.f;
            const float f1 = in ? __ldg(row1 + col[rr]) : 0.f;
            vx0 = fmaf(jx[rr], f0, vx0);
            vy0 = fmaf(jy[rr], f0, vy0);
            vx1 = fmaf(jx[rr], f1, vx1);
            vy1 = fmaf(jy[rr], f1, vy1);
        }
#pragma unroll
        for (int o = P / 2; o > 0; o >>= 1) {
            vx0 += __shfl_down_sync(0xffffffffu, vx0, o, P);
            vy0 += __shfl_down_sync(0xffffffffu, vy0, o, P);
            vx1 += __shfl_down_sync(0xffffffffu, vx1, o, P);
            vy1 += __shfl_down_sync(0xffffffffu, vy1, o, P);
        }
        if (c == 0 && s >= 0) {
            im[(size_t)m * ld_im + s] = scale * vx0;
            im[(size_t)m * ld_im + n_valid + s] = scale * vy0;
            if (two) {
                im[(size_t)(m + 1) * ld_im + s] = scale * vx1;
                im[(size_t)(m + 1) * ld_im + n_valid + s] = scale * vy1;
            }
        }
    }
}

}  // namespace

namespace {

int launch_adjoint(const char *who, const sb_sh_plan *pl, const float *A, const float *phase_nm, int n_valid,
                   const int32_t *lenslet, const float *xw, const float *yw, const float *mw, const float *active,
                   const float *seed, float *jac, float *tot_out, float *grad, void *stream) {
    if (!pl || !A || !phase_nm || !lenslet || !xw || !yw || !mw || !(jac || grad) || !pl->twiddle ||
        !pl->tilt || !pl->fp_mask || !pl->rebin)
        return sb::fail(SB_EINVAL, "%s: null pointer", who);
    if (n_valid < 1 || pl->n_lenses < 1 || pl->field_ld < pl->n_lenses * pl->np_sub)
        return sb::fail(SB_EINVAL, "%s: bad sizes", who);
    const AdjKernel k = adjoint_kernel(pl->np_sub, pl->cutsize, pl->subap_npx);
    if (!k.fn)
        return sb::fail(SB_EUNSUPPORTED, "%s: no adjoint kernel for np_sub=%d cutsize=%d subap_npx=%d", who,
                        pl->np_sub, pl->cutsize, pl->subap_npx);
    AdjArgs a;
    a.n = pl->n_lenses;
    a.p = pl->np_sub;
    a.cs = pl->cutsize;
    a.npx = pl->subap_npx;
    a.ld = pl->field_ld;
    a.k = pl->phase_to_rad;
    a.tw = reinterpret_cast<const float2 *>(pl->twiddle);
    a.tilt = reinterpret_cast<const float2 *>(pl->tilt);
    a.mask = pl->fp_mask;
    a.rebin = pl->rebin;
    a.A = A;
    a.ph = phase_nm;
    a.n_valid = n_valid;
    a.lenslet = lenslet;
    a.xw = xw;
    a.yw = yw;
    a.mw = mw;
    a.active = active;
    a.tot_out = tot_out;
    a.seed = seed;
    a.jac = jac;
    a.grad = grad;
    const int items = seed ? n_valid : 2 * n_valid;
    k.fn<<<(items + k.warps - 1) / k.warps, 32 * k.warps, 0, sb::as_stream(stream)>>>(a);
    return sb::check_launch(who);
}

}  // namespace

extern "C" int sb_sh_slopes_jacobian(const sb_sh_plan *pl, const float *A, const float *phase_nm, int n_valid,
                                     const int32_t *lenslet, const float *xw, const float *yw, const float *mw,
                                     const float *active, float *jac, float *tot_out, void *stream) {
    sb::clear_error();
    if (!jac) return sb::fail(SB_EINVAL, "sb_sh_slopes_jacobian: null output");
    return launch_adjoint("sb_sh_slopes_jacobian", pl, A, phase_nm, n_valid, lenslet, xw, yw, mw, active, nullptr,
                          jac, tot_out, nullptr, stream);
}

extern "C" int sb_sh_slopes_vjp(const sb_sh_plan *pl, const float *A, const float *phase_nm, int n_valid,
                                const int32_t *lenslet, const float *xw, const float *yw, const float *mw,
                                const float *active, const float *seed, float *grad_phase, void *stream) {
    sb::clear_error();
    if (!seed || !grad_phase) return sb::fail(SB_EINVAL, "sb_sh_slopes_vjp: null seed or output");
    return launch_adjoint("sb_sh_slopes_vjp", pl, A, phase_nm, n_valid, lenslet, xw, yw, mw, active, seed, nullptr,
                          nullptr, grad_phase, stream);
}

// ---------------------------------------------------------------------------
// The same contraction with the influence functions streamed by TMA.  The
// mirror's influence-function columns enumerate its pixels row-major, so
// the np_sub field rows of lenslet row li fall inside one contiguous column
// range of every mode's row: row_seg[li] = {start, count} (floats, both
// multiples of 32).  A work unit is (lenslet row, kCbUnitModes consecutive
// modes): one ring stage, filled by ceil(count / 256) 2-D TMA boxes of 256
// columns x kCbUnitModes modes, so a thread's sample of mode k sits k * 1 KB
// past its sample of mode 0.  A persistent CTA walks a contiguous range of units in
// row-major order; one producer lane loads each unit's box into the ring (L2
// evict-first) and the consumer warps, one thread per field column as in
// intmat_contract_kernel, read their np_sub samples per mode from shared
// memory.  Each column's products are summed over its np_sub rows in the
// order of intmat_contract_kernel; the np_sub columns of a lenslet are then
// summed by a transposed butterfly (group_sum_transposed) that adds the same
// pairs as that kernel's shuffle tree, so the matrices are the same bits.
// Every wait is bounded: on timeout the kernel records it in
// g_contract_status, stops issuing, lets the copies in flight land
// (bounded) and returns.
// ---------------------------------------------------------------------------
constexpr int kCbMaxStages = 8;
constexpr int kCbUnitModes = 4;        // modes per TMA box and work unit
constexpr int kCbMaxConsumers = 992;   // field columns (+ one producer warp <= 1024 threads)
constexpr int kCbRingBytes = 100 * 1024;
constexpr int kCbBoxCols = 256;        // columns per TMA box (the largest box extent)
constexpr int kCbMaxSegment = 7168;    // two stages of kCbUnitModes modes: 224 KB

__device__ int g_contract_status = 0;

struct ContractTmaArgs {
    const float *jac;
    const float *tot;
    int n_valid, n, field_ld;
    const int32_t *slot;
    const int32_t *pix2col;
    const int32_t *row_seg;
    const float *IF;
    int n_modes, ld_if;
    float scale;
    float *im;
    int stages, stage_floats;          // ring stages; floats per mode in a stage (multiple of kCbBoxCols)
};

// Columns streamed for lenslet row li: 0 when the row has none, or when its
// segment is not on 32-float boundaries or does not fit the row or a ring stage
// (recorded in g_contract_status; nothing is copied for it).
__device__ __forceinline__ int seg_count(const ContractTmaArgs &a, int li) {
    const int start = a.row_seg[2 * li], cnt = a.row_seg[2 * li + 1];
    if (cnt <= 0) return 0;
    if (start < 0 || (start & 31) || (cnt & 31) || cnt > a.stage_floats || (long long)start + cnt > a.ld_if) {
        atomicExch(&g_contract_status, 3);
        return 0;
    }
    return cnt;
}

// Sums v[0..NV) of the P lanes of each aligned lane group (P a power of two
// dividing 32) with NV / 2 + NV / 4 + ... shuffles instead of NV * log2(P):
// at the level of lane distance o every lane keeps half of its values (the
// upper half when lane bit o is set), adds its partner's copy of that half
// and passes the other half on.  On return lane c of a group holds, in
// v[0..NV / P), the sums of values c * NV / P .. c * NV / P + NV / P - 1.
// Each sum adds the same pairs as v += shfl_down(v, o, P) for o = P/2 .. 1
// (addition commutes exactly), so it has the same bits as that tree's lane 0.
template <int P, int NV>
__device__ __forceinline__ void group_sum_transposed(float (&v)[NV], int c) {
    static_assert(NV % P == 0, "whole values per lane");
#pragma unroll
    for (int o = P / 2, h = NV / 2; o >= 1; o >>= 1, h >>= 1) {
        const bool upper = (c & o) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = upper ? v[i] : v[i + h];
            const float keep = upper ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
}

// Weight of each unit of a lenslet row with cnt columns: its TMA boxes + 1
// (a unit's fixed cost).
__device__ __forceinline__ int cb_unit_weight(const ContractTmaArgs &a, int cnt) {
    cnt = cnt < 0 ? 0 : cnt > a.stage_floats ? a.stage_floats : cnt;
    return (cnt + kCbBoxCols - 1) / kCbBoxCols + 1;
}

constexpr int kCbMaxRows = (kCbMaxConsumers + 3) / 4;      // lenslet rows (np_sub >= 4)
constexpr int kCbRowBlocks = (kCbMaxRows + 31) / 32;

// The range [r[0], r[1]) of units of work part `part` of `parts`, in
// row-major order.  Unit (li, j) starts at weight W(li) + j * w(li), W(li) the
// weight of the rows before li; part b takes the units starting in
// [T * b / parts, T * (b + 1) / parts), T the total, so the ranges tile the
// units and carry about equal numbers of boxes.  Run by the 32 lanes of one
// warp (every row's count loaded in one round); lane 0 writes r.
__device__ void cb_unit_range(const ContractTmaArgs &a, int per_row, int part, int parts, int lane, int *r) {
    int w[kCbRowBlocks];
#pragma unroll
    for (int k = 0; k < kCbRowBlocks; ++k) {
        const int li = 32 * k + lane;
        w[k] = li < a.n ? cb_unit_weight(a, a.row_seg[2 * li + 1]) : 0;
    }
    long long T = 0;
#pragma unroll
    for (int k = 0; k < kCbRowBlocks; ++k) {
        long long t = (long long)per_row * w[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        T += t;
    }
    const long long lo = T * part / parts, hi = T * (part + 1) / parts;
    const int n_units = per_row * a.n;
    int u0 = n_units, u1 = n_units;
    bool f0 = false, f1 = false;
    long long W = 0;
#pragma unroll
    for (int k = 0; k < kCbRowBlocks; ++k) {
        const int li = 32 * k + lane;
        const bool row = li < a.n;
        const long long rw = (long long)per_row * w[k];
        long long incl = rw;     // inclusive scan of the row weights over the lanes
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const long long wr = W + incl - rw;
        // the row's first unit starting at or after weight t (per_row: none)
        const auto first = [&](long long t) -> int {
            if (!row) return per_row;
            if (t <= wr) return 0;
            const long long j = (t - wr + w[k] - 1) / w[k];
            return j < per_row ? (int)j : per_row;
        };
        const int j0 = first(lo), j1 = first(hi);
        const unsigned m0 = __ballot_sync(0xffffffffu, j0 < per_row);
        const unsigned m1 = __ballot_sync(0xffffffffu, j1 < per_row);
        if (!f0 && m0) {
            const int L = __ffs(m0) - 1;
            u0 = (32 * k + L) * per_row + __shfl_sync(0xffffffffu, j0, L);
            f0 = true;
        }
        if (!f1 && m1) {
            const int L = __ffs(m1) - 1;
            u1 = (32 * k + L) * per_row + __shfl_sync(0xffffffffu, j1, L);
            f1 = true;
        }
        W += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
        r[0] = u0;
        r[1] = u1;
    }
}

template <int P>
__global__ void __launch_bounds__(1024, 1) intmat_contract_tma_kernel(const __grid_constant__ CUtensorMap map,
                                                                      ContractTmaArgs a) {
    constexpr int MU = kCbUnitModes;
    constexpr int NV = 2 * MU;                  // (mode, axis) sums per unit
    constexpr int R = NV / P > 0 ? NV / P : 1;  // of them left on each lane
    static_assert(NV % P == 0, "a lenslet's lanes share the unit's sums");
    extern __shared__ __align__(128) unsigned char cb_smem[];
    // TMA destinations on 128-byte boundaries (segments are multiples of 128 bytes)
    unsigned char *base = cb_smem + ((128 - (sb::smem_u32(cb_smem) & 127)) & 127);
    float *ring = reinterpret_cast<float *>(base);
    const int stage = MU * a.stage_floats;      // floats per ring stage
    uint64_t *full = reinterpret_cast<uint64_t *>(base + (size_t)a.stages * stage * 4);
    uint64_t *empty = full + a.stages;
    __shared__ double red[33];
    __shared__ int abort_flag, issued, unit_range[2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncons = blockDim.x - 32;           // consumer threads (a multiple of 32)
    const int nwc = ncons >> 5;
    const int S = a.stages;
    if (tid == 0) {
        for (int k = 0; k < S; ++k) {
            sb::mbar_init(&full[k], 1);
            sb::mbar_init(&empty[k], nwc);
        }
        sb::mbar_init_fence();
        abort_flag = 0;
        issued = 0;
    }
    __syncthreads();
    const int per_row = (a.n_modes + MU - 1) / MU;
    const size_t ld_im = 2 * (size_t)a.n_valid;
    if (warp == nwc) {
        // the CTA's contiguous range of units (lenslet row, MU modes) in row-major
        // order, balanced by the boxes they load; published to the consumers
        // through named barrier 1 (arrive here, sync there)
        cb_unit_range(a, per_row, blockIdx.x, gridDim.x, lane, unit_range);
        asm volatile("bar.arrive 1, %0;" ::"r"(blockDim.x) : "memory");
        if (lane == 0) {
            const int u_begin = unit_range[0], u_end = unit_range[1];
            const uint64_t pol = sb::l2_evict_first_policy();
            int q = 0, st = 0, cur = -1, cnt = 0, start = 0;
            uint32_t ph = 0;
            for (int u = u_begin; u < u_end; ++u) {
                const int li = u / per_row, m0 = (u - li * per_row) * MU;
                if (li != cur) {
                    cur = li;
                    cnt = seg_count(a, li);
                    start = a.row_seg[2 * li];
                }
                if (cnt <= 0) continue;
                // reuse a slot once every consumer warp released its previous use
                if (q >= S && !sb::mbar_wait(&empty[st], ph ^ 1u)) {
                    atomicExch(&g_contract_status, 1);
                    abort_flag = 1;
                    break;
                }
                // whole boxes: columns and modes past the matrix read as zeros
                const int nb = (cnt + kCbBoxCols - 1) / kCbBoxCols;
                sb::mbar_arrive_expect_tx(&full[st], (uint32_t)(nb * kCbBoxCols * MU * 4));
                for (int b = 0; b < nb; ++b)
                    sb::tma_load_2d(ring + (size_t)st * stage + b * (kCbBoxCols * MU), &map, start + b * kCbBoxCols,
                                    m0, &full[st], pol);
                ++q;
                if (++st == S) {
                    st = 0;
                    ph ^= 1u;
                }
            }
            issued = q;
        }
    } else {
        // the CoG cut-off's mean over the consumer threads (named barrier 2),
        // while the producer already streams
        double mean = 0.0;
        if (a.tot) {
            double part = 0.0;
            for (int e = tid; e < a.n_valid; e += ncons) part += (double)a.tot[e];
            part = sb::warp_sum_d(part);
            if (lane == 0) red[warp] = part;
            asm volatile("bar.sync 2, %0;" ::"r"(ncons) : "memory");
            if (warp == 0) {
                double r = lane < nwc ? red[lane] : 0.0;
                r = sb::warp_sum_d(r);
                if (lane == 0) red[32] = r;
            }
            asm volatile("bar.sync 2, %0;" ::"r"(ncons) : "memory");
            mean = red[32] / a.n_valid;
        }
        asm volatile("bar.sync 1, %0;" ::"r"(blockDim.x) : "memory");
        const int u_begin = unit_range[0], u_end = unit_range[1];
        const int x = tid;
        const int lj = x / P, c = x - lj * P;
        int st = 0;
        uint32_t ph = 0;
        int cur = -1, cnt = 0, s = -1;
        // a masked pixel reads offset 0 with zero weights: fmaf(0, f, v) == v for the finite
        // influence functions, as fmaf(j, 0, v) in intmat_contract_kernel
        float jx[P], jy[P];
        int off[P];      // offset of the sample of mode 0 in a stage
        for (int u = u_begin; u < u_end; ++u) {
            const int li = u / per_row, m0 = (u - li * per_row) * MU;
            if (li != cur) {
                // a new lenslet row: slot and column map, then flux and Jacobian
                // (two dependent rounds of loads)
                cur = li;
                cnt = seg_count(a, li);
                const int start = a.row_seg[2 * li];
                s = (lj < a.n) ? a.slot[li * a.n + lj] : -1;
                int col[P];
#pragma unroll
                for (int rr = 0; rr < P; ++rr)
                    col[rr] = (lj < a.n) ? a.pix2col[(size_t)(li * P + rr) * a.field_ld + x] : -1;
                float t = 1.f;
#pragma unroll
                for (int rr = 0; rr < P; ++rr) jx[rr] = jy[rr] = 0.f;
                if (s >= 0) {
                    if (a.tot) t = a.tot[s];
#pragma unroll
                    for (int rr = 0; rr < P; ++rr) {
                        jx[rr] = a.jac[(size_t)s * (P * P) + rr * P + c];
                        jy[rr] = a.jac[((size_t)a.n_valid + s) * (P * P) + rr * P + c];
                    }
                }
                const bool act = s >= 0 && (!a.tot || (t > 0.f && (double)(1.0f / t) <= 1.0 / (mean * 1e-3)));
#pragma unroll
                for (int rr = 0; rr < P; ++rr) {
                    off[rr] = 0;
                    const int cl = act ? col[rr] : -1;
                    if (cl >= 0 && (cl < start || cl - start >= cnt))
                        atomicExch(&g_contract_status, 3);      // a column outside its row's segment
                    if (cl >= 0 && cl >= start && cl - start < cnt) {
                        const int o = cl - start;
                        off[rr] = (o / kCbBoxCols) * (kCbBoxCols * MU) + o % kCbBoxCols;
                    } else {
                        jx[rr] = jy[rr] = 0.f;
                    }
                }
            }
            float v[NV];
#pragma unroll
            for (int i = 0; i < NV; ++i) v[i] = 0.f;
            if (cnt > 0) {
                const bool ok = sb::mbar_wait_sleep(&full[st], ph);
                if (__any_sync(0xffffffffu, !ok)) {
                    if (lane == 0) atomicExch(&g_contract_status, 2);
                    abort_flag = 1;
                    break;
                }
                const float *seg = ring + (size_t)st * stage;
#pragma unroll
                for (int rr = 0; rr < P; ++rr) {
                    const float *p = seg + off[rr];
#pragma unroll
                    for (int k = 0; k < MU; ++k) {
                        const float f = p[kCbBoxCols * k];
                        v[2 * k] = fmaf(jx[rr], f, v[2 * k]);
                        v[2 * k + 1] = fmaf(jy[rr], f, v[2 * k + 1]);
                    }
                }
                __syncwarp();
                if (lane == 0) sb::mbar_arrive(&empty[st]);
                if (++st == S) {
                    st = 0;
                    ph ^= 1u;
                }
            }
            group_sum_transposed<P, NV>(v, c);
            if (s >= 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int i = c * R + r;          // (mode, axis) of this sum
                    const int m = m0 + (i >> 1);
                    if (m < a.n_modes) a.im[(size_t)m * ld_im + (i & 1) * a.n_valid + s] = a.scale * v[r];
                }
            }
        }
    }
    __syncthreads();
    if (abort_flag && tid == ncons) {
        // let the copies still in flight (at most the last S issued) land
        // before the shared memory is released
        for (int q = issued > S ? issued - S : 0; q < issued; ++q) sb::mbar_wait(&full[q % S], (q / S) & 1);
    }
}

extern "C" int sb_intmat_contract(const float *jac, const float *tot, int n_valid, int np_sub, int n_lenses,
                                  int field_ld, const int32_t *slot, const int32_t *pix2col, const float *ifunc,
                                  int n_modes, int ld_if, float scale, float *intmat, void *stream) {
    sb::clear_error();
    if (!jac || !slot || !pix2col || !ifunc || !intmat || n_valid < 1 || n_modes < 0 || n_lenses < 1 ||
        ld_if < 1)
        return sb::fail(SB_EINVAL, "sb_intmat_contract: bad args");
    if (field_ld < n_lenses * np_sub) return sb::fail(SB_EINVAL, "sb_intmat_contract: bad field stride");
    const int threads = (n_lenses * np_sub + 31) / 32 * 32;
    const int max_threads = np_sub >= 16 ? contract_max_threads<16>() : contract_max_threads<8>();
    if (threads > max_threads)
        return sb::fail(SB_ESHAPE, "sb_intmat_contract: field of %d columns (at most %d for np_sub=%d)",
                        n_lenses * np_sub, max_threads, np_sub);
    if (n_modes == 0) return SB_OK;
    const dim3 grid((n_modes + kContractModes - 1) / kContractModes, n_lenses);
    cudaStream_t st = sb::as_stream(stream);
    switch (np_sub) {
    case 4:
        intmat_contract_kernel<4><<<grid, threads, 0, st>>>(jac, tot, n_valid, n_lenses, field_ld, slot, pix2col,
                                                            ifunc, n_modes, ld_if, scale, intmat);
        break;
    case 8:
        intmat_contract_kernel<8><<<grid, threads, 0, st>>>(jac, tot, n_valid, n_lenses, field_ld, slot, pix2col,
                                                            ifunc, n_modes, ld_if, scale, intmat);
        break;
    case 16:
        intmat_contract_kernel<16><<<grid, threads, 0, st>>>(jac, tot, n_valid, n_lenses, field_ld, slot, pix2col,
                                                             ifunc, n_modes, ld_if, scale, intmat);
        break;
    default:
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_contract: np_sub=%d (4, 8 or 16)", np_sub);
    }
    return sb::check_launch("intmat_contract_kernel");
}

namespace sb {
// read and clear the timeout flag of the TMA contraction (0: none, <0: query failed)
int contract_status_take() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_contract_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_contract_status, &zero, sizeof(int));
    }
    return v;
}
}  // namespace sb

extern "C" int sb_intmat_contract_rows(const float *jac, const float *tot, int n_valid, int np_sub, int n_lenses,
                                       int field_ld, const int32_t *slot, const int32_t *pix2col,
                                       const int32_t *row_seg, int seg_max, const float *ifunc, int n_modes,
                                       int ld_if, float scale, float *intmat, void *stream) {
    sb::clear_error();
    if (!jac || !slot || !pix2col || !row_seg || !ifunc || !intmat || n_valid < 1 || n_modes < 0 ||
        n_lenses < 1 || ld_if < 1 || seg_max < 0)
        return sb::fail(SB_EINVAL, "sb_intmat_contract_rows: bad args");
    if (field_ld < n_lenses * np_sub) return sb::fail(SB_EINVAL, "sb_intmat_contract_rows: bad field stride");
    if (ld_if % 32 || (uintptr_t)ifunc % 16 || seg_max % 32 || seg_max > kCbMaxSegment)
        return sb::fail(SB_EINVAL, "sb_intmat_contract_rows: ld_if and seg_max must be multiples of 32 floats "
                                   "(seg_max <= %d), ifunc 16-byte aligned", kCbMaxSegment);
    const int ncons = (n_lenses * np_sub + 31) / 32 * 32;
    if (ncons > kCbMaxConsumers)
        return sb::fail(SB_ESHAPE, "sb_intmat_contract_rows: field of %d columns (at most %d)", n_lenses * np_sub,
                        kCbMaxConsumers);
    if (n_modes == 0) return SB_OK;
    const int stage_floats = seg_max > 0 ? (seg_max + kCbBoxCols - 1) / kCbBoxCols * kCbBoxCols : kCbBoxCols;
    // a ring of kCbRingBytes (two CTAs per SM), else two stages in one CTA's shared memory
    int stages = (int)(kCbRingBytes / ((size_t)stage_floats * 4 * kCbUnitModes));
    stages = stages > kCbMaxStages ? kCbMaxStages : stages < 2 ? 2 : stages;
    CUtensorMap map;
    int rc = sb::tensor_map_2d_f32(&map, ifunc, n_modes, ld_if, ld_if, kCbUnitModes, kCbBoxCols);
    if (rc) return rc;
    const size_t smem = 128 + (size_t)stages * stage_floats * 4 * kCbUnitModes + 2 * (size_t)stages * 8;
    ContractTmaArgs a;
    a.jac = jac;
    a.tot = tot;
    a.n_valid = n_valid;
    a.n = n_lenses;
    a.field_ld = field_ld;
    a.slot = slot;
    a.pix2col = pix2col;
    a.row_seg = row_seg;
    a.IF = ifunc;
    a.n_modes = n_modes;
    a.ld_if = ld_if;
    a.scale = scale;
    a.im = intmat;
    a.stages = stages;
    a.stage_floats = stage_floats;
    void (*fn)(const CUtensorMap, ContractTmaArgs) = nullptr;
    switch (np_sub) {
    case 4: fn = intmat_contract_tma_kernel<4>; break;
    case 8: fn = intmat_contract_tma_kernel<8>; break;
    default:
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_contract_rows: np_sub=%d (4 or 8)", np_sub);
    }
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return sb::fail(SB_ECUDA, "sb_intmat_contract_rows: smem attribute: %s", cudaGetErrorString(e));
    const int threads = ncons + 32;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess || per_sm < 1)
        return sb::fail(SB_ECUDA, "sb_intmat_contract_rows: occupancy query: %s",
                        e != cudaSuccess ? cudaGetErrorString(e) : "no CTA fits an SM");
    const int nsm = sb::sm_count();
    if (nsm < 1) return sb::fail(SB_ECUDA, "sb_intmat_contract_rows: SM count query failed");
    const int units = (n_modes + kCbUnitModes - 1) / kCbUnitModes * n_lenses;
    int grid = per_sm * nsm;
    grid = grid > units ? units : grid;
    fn<<<grid, threads, smem, sb::as_stream(stream)>>>(map, a);
    return sb::check_launch("intmat_contract_tma_kernel");
}

// ---------------------------------------------------------------------------
// The contraction on a lenslet-major copy of the influence functions.  At
// set-up (once per mirror and column map) sb_intmat_lenslet_ifunc gathers
// the samples under each valid sub-aperture into
//   ifl[m][s][c][r] = IF[m][pix2col[(li * P + r) * field_ld + lj * P + c]]
// (0 where pix2col < 0; (li, lj) the lenslet of valid sub-aperture s), so a
// sub-aperture's P x P samples of one mode are one contiguous run and field
// column c's P rows are P consecutive floats.  sb_intmat_contract_lenslets
// then streams that copy once: thread (s, c) reads its P rows as float4
// loads, sums jac * sample over them in row order and the P columns of the
// sub-aperture by group_sum_transposed: the pairs and order of
// intmat_contract_kernel, so the same matrix bit for bit.  No shared-memory
// ring, no producer: CTAs of 256 threads (256 / P sub-apertures) over a
// chunk of modes each, loads marked streaming (read once).
// ---------------------------------------------------------------------------
namespace {

constexpr int kClThreads = 256;
constexpr int kClModes = 4;           // modes summed per pass (2 * 4 sums per lenslet)

template <int P>
__global__ void intmat_lenslet_layout_kernel(const float *__restrict__ IF, int n_modes, int ld_if,
                                             const int32_t *__restrict__ lenslet, int n_valid, int n, int field_ld,
                                             const int32_t *__restrict__ pix2col, float *__restrict__ ifl) {
    const long long per_mode = (long long)n_valid * P * P;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= per_mode) return;
    const int s = (int)(e / (P * P)), q = (int)(e - (long long)s * P * P);
    const int c = q / P, r = q - c * P;
    const int L = lenslet[s];
    const int li = L / n, lj = L - li * n;
    const int col = pix2col[(size_t)(li * P + r) * field_ld + lj * P + c];
    for (int m = blockIdx.y; m < n_modes; m += gridDim.y)
        ifl[(size_t)m * per_mode + e] = col >= 0 ? IF[(size_t)m * ld_if + col] : 0.f;
}

template <int P>
__global__ void __launch_bounds__(kClThreads, 3) intmat_contract_lenslet_kernel(
    const float *__restrict__ jac, const float *__restrict__ tot, int n_valid, const float *__restrict__ ifl,
    int n_modes, int modes_per_cta, float scale, float *__restrict__ im) {
    constexpr int NV = 2 * kClModes;
    constexpr int R = NV / P > 0 ? NV / P : 1;
    static_assert(NV % P == 0 && P % 4 == 0, "whole sums per lane, float4 rows");
    __shared__ double red[33];
    const int t = blockIdx.x * kClThreads + threadIdx.x;
    const int s = t / P, c = t - s * P;
    const bool in = s < n_valid;
    bool act = in;
    if (tot) {
        // the CoG cut-off of sh_slopec.py:400, as intmat_contract_kernel applies it
        double part = 0.0;
        for (int e = threadIdx.x; e < n_valid; e += kClThreads) part += (double)tot[e];
        const double mean = sb::block_sum_all_d(part, red) / n_valid;
        if (act) {
            const float tt = tot[s];
            act = tt > 0.f && (double)(1.0f / tt) <= 1.0 / (mean * 1e-3);
        }
    }
    float jx[P], jy[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
        jx[r] = act ? jac[(size_t)s * (P * P) + r * P + c] : 0.f;
        jy[r] = act ? jac[((size_t)n_valid + s) * (P * P) + r * P + c] : 0.f;
    }
    const size_t per_mode = (size_t)n_valid * P * P;
    const float *mine = ifl + (in ? (size_t)s * (P * P) + c * P : 0);
    const int m0 = blockIdx.y * modes_per_cta;
    const int m1 = min(n_modes, m0 + modes_per_cta);
    const size_t ld_im = 2 * (size_t)n_valid;
    for (int m = m0; m < m1; m += kClModes) {
        float4 f[kClModes][P / 4];
#pragma unroll
        for (int k = 0; k < kClModes; ++k) {
            const bool ok = in && m + k < m1;
            const float4 *p = reinterpret_cast<const float4 *>(mine + (size_t)(ok ? m + k : 0) * per_mode);
#pragma unroll
            for (int b = 0; b < P / 4; ++b) f[k][b] = ok ? __ldcs(p + b) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float v[NV];
#pragma unroll
        for (int k = 0; k < kClModes; ++k) {
            float vx = 0.f, vy = 0.f;
#pragma unroll
            for (int b = 0; b < P / 4; ++b) {
                vx = fmaf(jx[4 * b + 0], f[k][b].x, vx);
                vy = fmaf(jy[4 * b + 0], f[k][b].x, vy);
                vx = fmaf(jx[4 * b + 1], f[k][b].y, vx);
                vy = fmaf(jy[4 * b + 1], f[k][b].y, vy);
                vx = fmaf(jx[4 * b + 2], f[k][b].z, vx);
                vy = fmaf(jy[4 * b + 2], f[k][b].z, vy);
                vx = fmaf(jx[4 * b + 3], f[k][b].w, vx);
                vy = fmaf(jy[4 * b + 3], f[k][b].w, vy);
            }
            v[2 * k] = vx;
            v[2 * k + 1] = vy;
        }
        group_sum_transposed<P, NV>(v, c);
        if (in) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = c * R + r;          // (mode, axis) of this sum
                const int mm = m + (i >> 1);
                if (mm < m1) im[(size_t)mm * ld_im + (i & 1) * n_valid + s] = scale * v[r];
            }
        }
    }
}

// modes per CTA: whole passes of kClModes, about four waves of three CTAs
// per SM (the kernel holds four at 64 registers; chunks of 4 to 64 modes
// measured the same on the 500-mode calibration system)
int lenslet_modes_per_cta(int n_valid, int np_sub, int n_modes) {
    const int bx = (int)(((long long)n_valid * np_sub + kClThreads - 1) / kClThreads);
    const int nsm = sb::sm_count();
    const long long target = 4LL * 3 * (nsm > 0 ? nsm : 148);
    long long chunks = (target + bx - 1) / bx;
    const long long passes = (n_modes + kClModes - 1) / kClModes;
    chunks = chunks < 1 ? 1 : chunks > passes ? passes : chunks;
    const long long per = (passes + chunks - 1) / chunks;
    return (int)(per * kClModes);
}

}  // namespace

extern "C" int sb_intmat_lenslet_ifunc(const float *ifunc, int n_modes, int ld_if, const int32_t *lenslet,
                                       int n_valid, int np_sub, int n_lenses, int field_ld, const int32_t *pix2col,
                                       float *ifl, void *stream) {
    sb::clear_error();
    if (!ifunc || !lenslet || !pix2col || !ifl || n_modes < 0 || n_valid < 1 || n_lenses < 1 || ld_if < 1)
        return sb::fail(SB_EINVAL, "sb_intmat_lenslet_ifunc: bad args");
    if (np_sub != 4 && np_sub != 8)
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_lenslet_ifunc: np_sub=%d (4 or 8)", np_sub);
    if (field_ld < n_lenses * np_sub) return sb::fail(SB_EINVAL, "sb_intmat_lenslet_ifunc: bad field stride");
    if ((uintptr_t)ifl % 16) return sb::fail(SB_EINVAL, "sb_intmat_lenslet_ifunc: ifl must be 16-byte aligned");
    if (n_modes == 0) return SB_OK;
    const long long per_mode = (long long)n_valid * np_sub * np_sub;
    const unsigned bx = (unsigned)((per_mode + 255) / 256);
    const dim3 grid(bx, (unsigned)(n_modes < 64 ? n_modes : 64));
    cudaStream_t st = sb::as_stream(stream);
    switch (np_sub) {
    case 4:
        intmat_lenslet_layout_kernel<4><<<grid, 256, 0, st>>>(ifunc, n_modes, ld_if, lenslet, n_valid, n_lenses,
                                                             field_ld, pix2col, ifl);
        break;
    case 8:
        intmat_lenslet_layout_kernel<8><<<grid, 256, 0, st>>>(ifunc, n_modes, ld_if, lenslet, n_valid, n_lenses,
                                                             field_ld, pix2col, ifl);
        break;
    default:
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_lenslet_ifunc: np_sub=%d (4 or 8)", np_sub);
    }
    return sb::check_launch("intmat_lenslet_layout_kernel");
}

extern "C" int sb_intmat_contract_lenslets(const float *jac, const float *tot, int n_valid, int np_sub,
                                           const float *ifl, int n_modes, float scale, float *intmat,
                                           void *stream) {
    sb::clear_error();
    if (!jac || !ifl || !intmat || n_valid < 1 || n_modes < 0)
        return sb::fail(SB_EINVAL, "sb_intmat_contract_lenslets: bad args");
    if (np_sub != 4 && np_sub != 8)
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_contract_lenslets: np_sub=%d (4 or 8)", np_sub);
    if ((uintptr_t)ifl % 16) return sb::fail(SB_EINVAL, "sb_intmat_contract_lenslets: ifl must be 16-byte aligned");
    if (n_modes == 0) return SB_OK;
    const int per = lenslet_modes_per_cta(n_valid, np_sub, n_modes);
    const dim3 grid((unsigned)(((long long)n_valid * np_sub + kClThreads - 1) / kClThreads),
                    (unsigned)((n_modes + per - 1) / per));
    cudaStream_t st = sb::as_stream(stream);
    switch (np_sub) {
    case 4:
        intmat_contract_lenslet_kernel<4><<<grid, kClThreads, 0, st>>>(jac, tot, n_valid, ifl, n_modes, per, scale,
                                                                      intmat);
        break;
    case 8:
        intmat_contract_lenslet_kernel<8><<<grid, kClThreads, 0, st>>>(jac, tot, n_valid, ifl, n_modes, per, scale,
                                                                      intmat);
        break;
    default:
        return sb::fail(SB_EUNSUPPORTED, "sb_intmat_contract_lenslets: np_sub=%d (4 or 8)", np_sub);
    }
    return sb::check_launch("intmat_contract_lenslet_kernel");
}
