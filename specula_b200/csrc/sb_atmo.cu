// Turbulence layer update and on-axis propagation on the B200.
//
// sb_atmo_evolve: one launch updates every layer; blockIdx.z selects the
// layer.  Each output pixel is evaluated straight from the screen strip:
// the column lerp (atmo_evolution.py:290), the rot90 index map (:291), the
// order-1 fractional-degree rotation with scipy's 'constant' boundary (:293;
// a sample outside [0, L-1] on either axis gives 0, otherwise bilinear from
// the four neighbours, neighbours off the grid counting 0) and the r0 scale
// (:294).  The lerp and scale keep NumPy's float32 operation order (no FMA
// contraction); the rotation samples are evaluated as small float32 offsets
// from the output pixel, with SciPy's exact float64 expression deciding the
// edge test wherever it is within 1e-4 px.
#include "sb_common.cuh"

namespace {

struct EvolveArgs {
    sb_atmo_layer layer[SB_MAX_LAYERS];
    int n, L;
    double *pos;
};

// new = last + delta; cycle to 0 when new + L reaches the strip width;
// float64 like the reference's NumPy arithmetic (atmo_evolution.py:269-277)
__global__ void atmo_advance_kernel(EvolveArgs a) {
    const int k = threadIdx.x;
    if (k >= a.n) return;
    double np = __dadd_rn(a.pos[k], a.layer[k].delta);
    if (__dadd_rn(np, (double)a.L) >= (double)a.layer[k].screen_cols) np = 0.0;
    a.pos[k] = np;
}

// Output tiles of 32 x 32 pixels per CTA (32 x 8 threads, 4 rows each).
// The tile's footprint in the rot90'd, lerped layer is staged in shared
// memory first: that read is ordered so consecutive threads touch
// consecutive screen columns whatever the rot90 quarter, which keeps the
// strip reads coalesced (a direct gather is column-strided for odd k).
constexpr int kTile = 32;
constexpr int kBox = kTile + 8;   // footprint of a tile rotated by < 1 degree, plus the bilinear +1

__global__ void __launch_bounds__(256) atmo_evolve_kernel(EvolveArgs a) {
    __shared__ float Q[kBox][kBox + 1];
    __shared__ int fp[5];                 // footprint br0, br1, bc0, bc1 and the interior flag
    const sb_atmo_layer &ly = a.layer[blockIdx.z];
    const int L = a.L;
    const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) {
        // footprint [br0, br1] x [bc0, bc1] of the tile in the rot90'd layer
        int br0 = y0, br1 = min(y0 + kTile, L) - 1, bc0 = x0, bc1 = min(x0 + kTile, L) - 1;
        int interior = 0;
        if (ly.rotate) {
            double rmin = 1e300, rmax = -1e300, cmin = 1e300, cmax = -1e300;
            for (int cy = 0; cy < 2; ++cy)
                for (int cx = 0; cx < 2; ++cx) {
                    const double yy = cy ? br1 : br0, xx = cx ? bc1 : bc0;
                    const double ir = __dadd_rn(__dadd_rn(__dmul_rn(ly.m00, yy), __dmul_rn(ly.m01, xx)), ly.off0);
                    const double ic = __dadd_rn(__dadd_rn(__dmul_rn(ly.m10, yy), __dmul_rn(ly.m11, xx)), ly.off1);
                    rmin = fmin(rmin, ir); rmax = fmax(rmax, ir);
                    cmin = fmin(cmin, ic); cmax = fmax(cmax, ic);
                }
            // every sample of the tile at least 0.01 px inside [0, L-1) on
            // both axes: no edge test, no clamp, all four neighbours on the
            // grid (the float32 sample positions are within 1e-4 px of these)
            interior = rmin >= 0.01 && rmax <= L - 1 - 0.01 && cmin >= 0.01 && cmax <= L - 1 - 0.01;
            br0 = max(0, (int)floor(rmin) - 1);
            br1 = min(L - 1, (int)floor(rmax) + 2);
            bc0 = max(0, (int)floor(cmin) - 1);
            bc1 = min(L - 1, (int)floor(cmax) + 2);
            // a footprint wider than the staging box means |angle| >= ~6
            // degrees, which the fractional-degree rotation never produces
            br1 = min(br1, br0 + kBox - 1);
            bc1 = min(bc1, bc0 + kBox - 1);
        }
        fp[0] = br0; fp[1] = br1; fp[2] = bc0; fp[3] = bc1; fp[4] = interior;
    }
    // integer position and float32 remainder (atmo_evolution.py:278-279)
    const double np = a.pos[blockIdx.z];
    const double q = floor(np);
    const float *row0 = ly.screen + (long long)q;
    const int ld = ly.screen_ld;
    const float frac = (float)(np - q);
    const float w0 = __fsub_rn(1.0f, frac);
    const int k = ly.rot90;
    __syncthreads();
    const int br0 = fp[0], br1 = fp[1], bc0 = fp[2], bc1 = fp[3];
    const bool interior = fp[4] != 0;
    const int R = br1 - br0 + 1, Cc = bc1 - bc0 + 1;
    // rot90(lerped)[yy][xx] reads screen element base + ra*dR + cb*dC
    // (ra, cb: footprint row / column); thread (tx, ty) of the 32 x 8 block
    // walks the footprint so that tx always runs along screen columns:
    // along footprint columns for even k, along footprint rows for odd k.
    // Offsets fit in 32 bits (strip rows x row stride < 2^31, checked on the host).
    int dR, dC, b0;
    switch (k) {
        case 1: dR = -1; dC = ld; b0 = bc0 * ld + (L - 1 - br0); break;
        case 2: dR = -ld; dC = -1; b0 = (L - 1 - br0) * ld + (L - 1 - bc0); break;
        case 3: dR = 1; dC = -ld; b0 = (L - 1 - bc0) * ld + br0; break;
        default: dR = ld; dC = 1; b0 = br0 * ld + bc0;
    }
    const bool odd = k & 1;
    const int n_fast = odd ? R : Cc, n_slow = odd ? Cc : R;
    const int d_fast = odd ? dR : dC, d_slow = odd ? dC : dR;
    {
        // Q strides of the fast and slow walk: Q[sl][fa] for even k, Q[fa][sl] for odd k
        const int qs_fast = odd ? kBox + 1 : 1, qs_slow = odd ? 1 : kBox + 1;
        float *qbase = &Q[0][0];
        for (int sl = threadIdx.y; sl < n_slow; sl += blockDim.y) {
            int off = b0 + sl * d_slow + threadIdx.x * d_fast;
            int qo = sl * qs_slow + threadIdx.x * qs_fast;
            for (int fa = threadIdx.x; fa < n_fast; fa += blockDim.x) {
                const float *p = row0 + off;
                qbase[qo] = __fadd_rn(__fmul_rn(w0, p[0]), __fmul_rn(frac, p[1]));
                off += 32 * d_fast;
                qo += 32 * qs_fast;
            }
        }
    }
    __syncthreads();
    const int x = x0 + threadIdx.x;
    if (x >= L) return;
    float *out = ly.out + x;
    const float scale = ly.scale;
    if (!ly.rotate) {
        for (int yi = threadIdx.y; yi < kTile; yi += blockDim.y) {
            const int y = y0 + yi;
            if (y < L) out[(size_t)y * L] = __fmul_rn(Q[y - br0][x - bc0], scale);   // atmo_evolution.py:294
        }
        return;
    }
    // the rotation is below one degree: sample = (y + dr, x + dc) with
    // dr = (m00-1) y + m01 x + off0 and dc = m10 y + (m11-1) x + off1 small
    // (|dr|, |dc| < ~12 px), so they are evaluated in float32 to ~1e-6 px.
    const float a00 = (float)(ly.m00 - 1.0), a01 = (float)ly.m01, a10 = (float)ly.m10, a11 = (float)(ly.m11 - 1.0);
    const float b0f = (float)ly.off0, b1f = (float)ly.off1;
    const float xf = (float)x;
    const float dr_x = fmaf(a01, xf, b0f), dc_x = fmaf(a11, xf, b1f);
    if (interior) {
        // every sample of this tile is well inside the layer
        const float *qb = &Q[0][0] - br0 * (kBox + 1) - bc0;
        for (int yi = threadIdx.y; yi < kTile; yi += blockDim.y) {
            const int y = y0 + yi;
            if (y >= L) break;
            const float yf = (float)y;
            const float dr = fmaf(a00, yf, dr_x), dc = fmaf(a10, yf, dc_x);
            const float fdr = floorf(dr), fdc = floorf(dc);
            const float fr = dr - fdr, fc = dc - fdc;
            const float *p = qb + (y + (int)fdr) * (kBox + 1) + x + (int)fdc;
            const float q00 = p[0], q01 = p[1], q10 = p[kBox + 1], q11 = p[kBox + 2];
            const float top = fmaf(fc, q01 - q00, q00);
            const float bot = fmaf(fc, q11 - q10, q10);
            out[(size_t)y * L] = __fmul_rn(fmaf(fr, bot - top, top), scale);
        }
        return;
    }
    // tiles near the layer edge: only the edge test (sample outside [0, L-1]
    // gives 0) is discontinuous; within 1e-4 px of an edge it is redone with
    // SciPy's exact float64 expression (m00*y + m01*x) + off0
    const float Lm1 = (float)(L - 1);
    for (int yi = threadIdx.y; yi < kTile; yi += blockDim.y) {
        const int y = y0 + yi;
        if (y >= L) break;
        float v;
        const float yf = (float)y;
        const float dr = fmaf(a00, yf, dr_x), dc = fmaf(a10, yf, dc_x);
        const float irf = yf + dr, icf = xf + dc;
        bool inside = irf >= 0.f && irf <= Lm1 && icf >= 0.f && icf <= Lm1;
        const float eps = 1e-4f;
        if (irf < eps || irf > Lm1 - eps || icf < eps || icf > Lm1 - eps) {
            const double yd = (double)y, xd = (double)x;
            const double ir = __dadd_rn(__dadd_rn(__dmul_rn(ly.m00, yd), __dmul_rn(ly.m01, xd)), ly.off0);
            const double ic = __dadd_rn(__dadd_rn(__dmul_rn(ly.m10, yd), __dmul_rn(ly.m11, xd)), ly.off1);
            inside = ir >= 0.0 && ir <= (double)(L - 1) && ic >= 0.0 && ic <= (double)(L - 1);
        }
        if (!inside) {
            v = 0.0f;
        } else {
            const float fdr = floorf(dr), fdc = floorf(dc);
            int r0 = y + (int)fdr, c0 = x + (int)fdc;
            float fr = dr - fdr, fc = dc - fdc;
            // clamp to the grid (only reachable within 1e-4 px of an edge)
            if (r0 < 0) { r0 = 0; fr = 0.f; }
            if (c0 < 0) { c0 = 0; fc = 0.f; }
            if (r0 > L - 1) { r0 = L - 1; fr = 0.f; }
            if (c0 > L - 1) { c0 = L - 1; fc = 0.f; }
            const int qr = r0 - br0, qc = c0 - bc0;
            const bool rin = r0 + 1 < L, cin = c0 + 1 < L;
            const float q00 = Q[qr][qc];
            const float q01 = cin ? Q[qr][qc + 1] : 0.0f;
            const float q10 = rin ? Q[qr + 1][qc] : 0.0f;
            const float q11 = (rin && cin) ? Q[qr + 1][qc + 1] : 0.0f;
            const float top = fmaf(fc, q01 - q00, q00);
            const float bot = fmaf(fc, q11 - q10, q10);
            v = fmaf(fr, bot - top, top);
        }
        out[(size_t)y * L] = __fmul_rn(v, scale);   // atmo_evolution.py:294
    }
}

struct PropArgs {
    sb_prop_layer layer[SB_MAX_LAYERS];
    int n, pupil;
};

__global__ void __launch_bounds__(256) propagate_kernel(PropArgs a, float *__restrict__ A, float *__restrict__ P) {
    const int n = a.pupil * a.pupil;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int r = e / a.pupil, c = e - r * a.pupil;
        float amp = 1.0f, ph = 0.0f;                       // ElectricField.reset()
        for (int k = 0; k < a.n; ++k) {
            const sb_prop_layer &l = a.layer[k];
            const size_t g = (size_t)(r + l.top) * l.ld + (c + l.left);
            if (l.A) amp = __fmul_rn(amp, l.A[g]);
            if (l.phase) ph = __fadd_rn(ph, l.phase[g]);
        }
        A[e] = amp;
        P[e] = ph;
    }
}

}  // namespace

extern "C" int sb_atmo_evolve(const sb_atmo_layer *layers, int n_layers, int L, double *positions, void *stream) {
    sb::clear_error();
    if (!layers || !positions || n_layers < 0 || L < 1) return sb::fail(SB_EINVAL, "sb_atmo_evolve: bad args");
    if (n_layers > SB_MAX_LAYERS) return sb::fail(SB_ESHAPE, "sb_atmo_evolve: at most %d layers", SB_MAX_LAYERS);
    if (n_layers == 0) return SB_OK;
    EvolveArgs a;
    for (int k = 0; k < n_layers; ++k) {
        const sb_atmo_layer &l = layers[k];
        // the window [pos, pos + L] must stay inside the strip for every
        // position the cycling rule allows: pos + L < screen_cols
        if (!l.screen || !l.out || l.screen_cols < L + 1 || l.screen_ld < l.screen_cols || l.rot90 < 0 ||
            l.rot90 > 3 || !(l.delta >= 0.0))
            return sb::fail(SB_EINVAL, "sb_atmo_evolve: layer %d: bad screen window", k);
        // element offsets inside the strip window are 32-bit
        if ((long long)L * l.screen_ld + l.screen_cols >= (1LL << 31))
            return sb::fail(SB_ESHAPE, "sb_atmo_evolve: layer %d: strip too large", k);
        // the fractional-degree rotation is below 1 degree: the staged
        // footprint of a tile is sized for that
        if (l.rotate && !(fabs(l.m01) < 0.0175 && fabs(l.m10) < 0.0175 && l.m00 > 0.9998 && l.m11 > 0.9998))
            return sb::fail(SB_EINVAL, "sb_atmo_evolve: layer %d: rotation must be below one degree", k);
        a.layer[k] = l;
    }
    a.n = n_layers;
    a.L = L;
    a.pos = positions;
    cudaStream_t st = sb::as_stream(stream);
    atmo_advance_kernel<<<1, 32, 0, st>>>(a);
    int rc = sb::check_launch("atmo_advance_kernel");
    if (rc) return rc;
    dim3 block(32, 8), grid((L + kTile - 1) / kTile, (L + kTile - 1) / kTile, n_layers);
    atmo_evolve_kernel<<<grid, block, 0, st>>>(a);
    return sb::check_launch("atmo_evolve_kernel");
}

extern "C" int sb_propagate_on_axis(const sb_prop_layer *layers, int n_layers, int pupil, float *A_out,
                                    float *phase_out, void *stream) {
    sb::clear_error();
    if (!layers || !A_out || !phase_out || n_layers < 0 || pupil < 1)
        return sb::fail(SB_EINVAL, "sb_propagate_on_axis: bad args");
    if (n_layers > SB_MAX_LAYERS) return sb::fail(SB_ESHAPE, "sb_propagate_on_axis: at most %d layers", SB_MAX_LAYERS);
    PropArgs a;
    for (int k = 0; k < n_layers; ++k) {
        if (layers[k].top < 0 || layers[k].left < 0 || layers[k].ld < pupil + layers[k].left)
            return sb::fail(SB_EINVAL, "sb_propagate_on_axis: layer %d: bad crop", k);
        a.layer[k] = layers[k];
    }
    a.n = n_layers;
    a.pupil = pupil;
    int nblk = (pupil * pupil + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    propagate_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(a, A_out, phase_out);
    return sb::check_launch("propagate_kernel");
}
