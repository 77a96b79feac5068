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
