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
#include <new>
#include <vector>

#include "sb_common.cuh"
#include "sb_mc.cuh"

namespace {

// per-step layer parameters (atmo_evolution.py:262-294)
struct LayerDyn {
    double delta;
    double m00, m01, m10, m11, off0, off1;
    int rot90, rotate;
    float scale;
};

// per-layer device pointers: the layer's seeing / wind inputs and position
struct LayerPtrs {
    const double *seeing, *wind_speed, *wind_direction;
    double *pos;
};

template <int CAP>
struct EvolveArgsT {
    sb_atmo_layer layer[CAP];
    LayerPtrs ptr[CAP];
    int n, L;
    // constants of the per-step parameters (its pointers are not read here)
    sb_atmo_inputs in;
    // per-step parameters computed on the device from the inputs (NULL: the
    // delta / rot90 / rotation / scale fields of layer[] are used)
    LayerDyn *dyn;
};
constexpr int kBatchLayers = 64;   // layers per batched launch

// Per-step layer parameters from device-resident seeing / wind inputs, with
// the reference's float64 / float32 arithmetic (atmo_evolution.py:262-294):
// r0 = 0.9759*0.5/(seeing*4.848) * airmass^(-3/5) and the r0 scale in float32
// (NumPy promotes the Python-float products to the float32 airmass), shift
// wind_speed*dt/pitch, rot90 by trunc(dir/90) mod 4 and the fractional-degree
// rotation about the layer centre (scipy.ndimage.rotate's output->input map).
__device__ LayerDyn layer_dyn(const sb_atmo_inputs &in, const LayerPtrs &p, int L) {
    LayerDyn d;
    const double seeing = p.seeing[0];
    const double ws = p.wind_speed[0];
    const double wd = p.wind_direction[0];
    const double r0d = __ddiv_rn(__dmul_rn(0.9759, 0.5), __dmul_rn(seeing, 4.848));
    const float r0 = __fmul_rn((float)r0d, in.airmass_pow);
    const float r0l = __fmul_rn(r0, in.lambda_factor);
    const float x = __fdiv_rn(in.pixel_pitch_f, r0l);
    d.scale = (float)pow((double)x, (double)(5.0f / 6.0f));
    d.delta = __ddiv_rn(__dmul_rn(ws, in.delta_time), in.pixel_pitch);
    const double q90 = trunc(__ddiv_rn(wd, 90.0));
    int k90 = (int)fmod(q90, 4.0);
    d.rot90 = k90 < 0 ? k90 + 4 : k90;
    const double frac = wd - trunc(wd);
    d.rotate = frac != 0.0;
    double c = 1.0, sn = 0.0;
    if (d.rotate) {
        const double t = __ddiv_rn(frac, 180.0);
        c = cospi(t);
        sn = sinpi(t);
    }
    const double ctr = (L - 1) / 2.0;
    d.m00 = c; d.m01 = sn; d.m10 = -sn; d.m11 = c;
    d.off0 = __dsub_rn(ctr, __dadd_rn(__dmul_rn(c, ctr), __dmul_rn(sn, ctr)));
    d.off1 = __dsub_rn(ctr, __dadd_rn(__dmul_rn(-sn, ctr), __dmul_rn(c, ctr)));
    return d;
}

__device__ __forceinline__ LayerDyn static_dyn(const sb_atmo_layer &l) {
    LayerDyn d;
    d.delta = l.delta;
    d.m00 = l.m00; d.m01 = l.m01; d.m10 = l.m10; d.m11 = l.m11; d.off0 = l.off0; d.off1 = l.off1;
    d.rot90 = l.rot90;
    d.rotate = l.rotate;
    d.scale = l.scale;
    return d;
}

// new = last + delta; cycle to 0 when new + L reaches the strip width;
// float64 like the reference's NumPy arithmetic (atmo_evolution.py:269-277)
template <int CAP>
__global__ void atmo_advance_kernel(EvolveArgsT<CAP> a) {
    const int k = threadIdx.x;
    if (k >= a.n) return;
    double delta = a.layer[k].delta;
    if (a.dyn) {
        const LayerDyn d = layer_dyn(a.in, a.ptr[k], a.L);
        a.dyn[k] = d;
        delta = d.delta;
    }
    double *pos = a.ptr[k].pos;
    double np = __dadd_rn(*pos, delta);
    if (__dadd_rn(np, (double)a.L) >= (double)a.layer[k].screen_cols) np = 0.0;
    *pos = np;
}

// Output tiles of 32 x 32 pixels per CTA (32 x 8 threads, 4 rows each).
// The tile's footprint in the rot90'd, lerped layer is staged in shared
// memory first: that read is ordered so consecutive threads touch
// consecutive screen columns whatever the rot90 quarter, which keeps the
// strip reads coalesced (a direct gather is column-strided for odd k).
constexpr int kTile = 32;
constexpr int kBox = kTile + 8;   // footprint of a tile rotated by < 1 degree, plus the bilinear +1
constexpr int kRowStep = 8;       // blockDim.y: output rows advance by 8 per thread

// floor(v) for |v| < 2^22 on the FMA and integer pipes instead of the
// conversion unit: the round-down sum with C = 1.5 * 2^23 lands on the
// integer grid (spacing 1 in [2^23, 2^24)) at exactly C + floor(v), so
// (sum - C) is floor(v) as a float and the bit difference is floor(v) as an
// integer.
__device__ __forceinline__ int floor_small(float v, float &fl) {
    constexpr float C = 12582912.0f;
    const float t = __fadd_rd(v, C);
    fl = __fsub_rn(t, C);
    return __float_as_int(t) - __float_as_int(C);
}
__device__ __forceinline__ int floor_small(float v) {
    float fl;
    return floor_small(v, fl);
}

// The pieces of one 32 x 32 output tile of layer li.  tile_footprint (one
// thread) fixes the layer's per-step parameters and the footprint of the tile
// in the rot90'd, lerped layer; tile_load issues this thread's share of the
// footprint reads; tile_stage writes them into the shared staging Q;
// tile_values (after a barrier) produces rows y0 + ty + 8 j (j < 4) of column
// x0 + tx and hands each value to sink(j, y, x, value).
struct TileFootprint {
    int br0, br1, bc0, bc1, interior;
};

// the layer a tile is cut from: its record, position, per-step parameters
// (NULL: the record's static ones), side and the tile's origin
struct TileSrc {
    const sb_atmo_layer *layer;
    const double *pos;
    const LayerDyn *dyn;
    int L, x0, y0;
};

template <int CAP>
__device__ __forceinline__ TileSrc tile_src(const EvolveArgsT<CAP> &a, int li) {
    return {&a.layer[li], a.ptr[li].pos, a.dyn ? a.dyn + li : nullptr, a.L, (int)blockIdx.x * kTile,
            (int)blockIdx.y * kTile};
}

__device__ __forceinline__ void tile_footprint(const TileSrc &src, LayerDyn &lyd, TileFootprint &fp) {
    lyd = src.dyn ? *src.dyn : static_dyn(*src.layer);
    const LayerDyn &ly = lyd;
    const int L = src.L;
    const int x0 = src.x0, y0 = src.y0;
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
    fp.br0 = br0; fp.br1 = br1; fp.bc0 = bc0; fp.bc1 = bc1; fp.interior = interior;
}

constexpr int kStagePer = (kBox * kBox + 255) / 256;   // footprint elements per thread

// this thread's footprint reads: the strip's two neighbouring columns of each
// element (v0, v1), its place in Q (qo, -1: none) and the lerp weights
struct TileLoads {
    float v0[kStagePer], v1[kStagePer];
    int qo[kStagePer];
    float w0, frac;
};

__device__ __forceinline__ void tile_load(const TileSrc &src, const LayerDyn &ly, const TileFootprint &fp, int tid,
                                          TileLoads &t) {
    const sb_atmo_layer &lys = *src.layer;
    const int L = src.L;
    // integer position and float32 remainder (atmo_evolution.py:278-279)
    const double np = *src.pos;
    const double q = floor(np);
    const float *row0 = lys.screen + (long long)q;
    const int ld = lys.screen_ld;
    t.frac = (float)(np - q);
    t.w0 = __fsub_rn(1.0f, t.frac);
    const int k = ly.rot90;
    const int br0 = fp.br0, br1 = fp.br1, bc0 = fp.bc0, bc1 = fp.bc1;
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
    // Q strides of the fast and slow walk: Q[sl][fa] for even k, Q[fa][sl] for odd k
    const int qs_fast = odd ? kBox + 1 : 1, qs_slow = odd ? 1 : kBox + 1;
    // the footprint walked as one flat range e = sl * n_fast + fa, every
    // lane busy; sl = floor((e + 0.5) / n_fast) in float32 is exact here
    // (e < 1600, n_fast <= 40: the quotient is >= 0.0125 from an integer,
    // the float32 error below 5e-6)
    const int n_el = n_fast * n_slow;
    const float inv_nf = 1.0f / (float)n_fast;
    const float e_half = (float)tid + 0.5f;
#pragma unroll
    for (int j = 0; j < kStagePer; ++j) {
        const int e = tid + 256 * j;
        t.qo[j] = -1;
        if (e < n_el) {
            const int sl = floor_small((e_half + 256.0f * j) * inv_nf);
            const int fa = e - sl * n_fast;
            const float *p = row0 + (b0 + sl * d_slow + fa * d_fast);
            t.v0[j] = p[0];
            t.v1[j] = p[1];
            t.qo[j] = sl * qs_slow + fa * qs_fast;
        }
    }
}

__device__ __forceinline__ void tile_stage(float (&Q)[kBox][kBox + 1], const TileLoads &t) {
    float *qbase = &Q[0][0];
#pragma unroll
    for (int j = 0; j < kStagePer; ++j)
        if (t.qo[j] >= 0) qbase[t.qo[j]] = __fadd_rn(__fmul_rn(t.w0, t.v0[j]), __fmul_rn(t.frac, t.v1[j]));
}

template <class Sink>
__device__ __forceinline__ void tile_values(int L, int x0, int y0, const float (&Q)[kBox][kBox + 1],
                                            const LayerDyn &ly, const TileFootprint &fp, Sink &&sink) {
    const int br0 = fp.br0, bc0 = fp.bc0;
    const bool interior = fp.interior != 0;
    const int x = x0 + threadIdx.x;
    if (x >= L) return;
    const float scale = ly.scale;
    if (!ly.rotate) {
#pragma unroll
        for (int j = 0; j < kTile / kRowStep; ++j) {
            const int y = y0 + (int)threadIdx.y + kRowStep * j;
            if (y < L) sink(j, y, x, __fmul_rn(Q[y - br0][x - bc0], scale));   // atmo_evolution.py:294
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
        float yf = (float)(y0 + (int)threadIdx.y);
#pragma unroll
        for (int j = 0; j < kTile / kRowStep; ++j, yf += (float)kRowStep) {
            const int y = y0 + (int)threadIdx.y + kRowStep * j;
            if (y >= L) break;
            const float dr = fmaf(a00, yf, dr_x), dc = fmaf(a10, yf, dc_x);
            float fdr, fdc;
            const int idr = floor_small(dr, fdr), idc = floor_small(dc, fdc);
            const float fr = dr - fdr, fc = dc - fdc;
            const float *p = qb + (y + idr) * (kBox + 1) + x + idc;
            const float q00 = p[0], q01 = p[1], q10 = p[kBox + 1], q11 = p[kBox + 2];
            const float top = fmaf(fc, q01 - q00, q00);
            const float bot = fmaf(fc, q11 - q10, q10);
            sink(j, y, x, __fmul_rn(fmaf(fr, bot - top, top), scale));
        }
        return;
    }
    // tiles near the layer edge: only the edge test (sample outside [0, L-1]
    // gives 0) is discontinuous; within 1e-4 px of an edge it is redone with
    // SciPy's exact float64 expression (m00*y + m01*x) + off0
    const float Lm1 = (float)(L - 1);
#pragma unroll
    for (int j = 0; j < kTile / kRowStep; ++j) {
        const int y = y0 + (int)threadIdx.y + kRowStep * j;
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
        sink(j, y, x, __fmul_rn(v, scale));   // atmo_evolution.py:294
    }
}

// One whole tile (every thread of the CTA must call it: it holds two CTA
// barriers); Q, fp and lyd are the CTA's shared staging.
template <class Sink>
__device__ __forceinline__ void evolve_tile(const TileSrc &src, float (&Q)[kBox][kBox + 1], TileFootprint &fp,
                                            LayerDyn &lyd, Sink &&sink) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) tile_footprint(src, lyd, fp);
    __syncthreads();                      // lyd and fp written by thread 0
    TileLoads t;
    tile_load(src, lyd, fp, tid, t);
    tile_stage(Q, t);
    __syncthreads();
    tile_values(src.L, src.x0, src.y0, Q, lyd, fp, sink);
}

template <int CAP>
__global__ void __launch_bounds__(256) atmo_evolve_kernel(EvolveArgsT<CAP> a) {
    __shared__ float Q[kBox][kBox + 1];
    __shared__ TileFootprint fp;          // footprint of the tile and the interior flag
    __shared__ LayerDyn lyd;              // this layer's per-step parameters
    float *out = a.layer[blockIdx.z].out;
    const int L = a.L;
    evolve_tile(tile_src(a, blockIdx.z), Q, fp, lyd, [&](int, int y, int x, float v) { out[(size_t)y * L + x] = v; });
}

// The on-axis propagation of pupil-sized layers fused in: blockIdx.z is a
// realisation whose n_atm layers are layer[z * n_atm ...]; each layer is
// written as by atmo_evolve_kernel and summed in registers in layer order,
// then the stop and mirror layers are applied in propagate_batched_kernel's
// operation order and the field written (the same bits as the two launches).
constexpr int kFusedMaxLayers = SB_MAX_LAYERS;   // turbulence layers per realisation in the fused kernel

struct FusedPropArgs {
    const float *stop_A, *stop_phase, *dm_A, *dm_phase;
    long long dm_stride, out_stride;
    float *A, *P;
    int n_atm, real0;   // layers per realisation; index of this launch's first realisation
};

template <int CAP>
__global__ void __launch_bounds__(256, 4) atmo_propagate_kernel(EvolveArgsT<CAP> a, FusedPropArgs f) {
    // layers are software-pipelined: the footprint reads of layer k+1 are in
    // flight while layer k's values are computed from the other staging buffer
    __shared__ float Q[2][kBox][kBox + 1];
    __shared__ TileFootprint fp[kFusedMaxLayers];
    __shared__ LayerDyn lyd[kFusedMaxLayers];
    const int L = a.L;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int n = f.n_atm, l0 = blockIdx.z * n;
    if (tid < n) tile_footprint(tile_src(a, l0 + tid), lyd[tid], fp[tid]);
    float acc[kTile / kRowStep];
#pragma unroll
    for (int j = 0; j < kTile / kRowStep; ++j) acc[j] = 0.0f;          // ElectricField.reset()
    __syncthreads();
    TileLoads t;
    tile_load(tile_src(a, l0), lyd[0], fp[0], tid, t);
    for (int k = 0; k < n; ++k) {
        tile_stage(Q[k & 1], t);
        if (k + 1 < n) tile_load(tile_src(a, l0 + k + 1), lyd[k + 1], fp[k + 1], tid, t);
        // staging k complete; the buffer of layer k+1 was last read at layer
        // k-1, before this barrier's predecessor
        __syncthreads();
        float *out = a.layer[l0 + k].out;
        tile_values(L, (int)blockIdx.x * kTile, (int)blockIdx.y * kTile, Q[k & 1], lyd[k], fp[k],
                    [&](int j, int y, int x, float v) {
            out[(size_t)y * L + x] = v;
            acc[j] = __fadd_rn(acc[j], v);
        });
    }
    const int x = blockIdx.x * kTile + threadIdx.x;
    if (x >= L) return;
    const long long b = f.real0 + blockIdx.z;
#pragma unroll
    for (int j = 0; j < kTile / kRowStep; ++j) {
        const int y = blockIdx.y * kTile + (int)threadIdx.y + kRowStep * j;
        if (y >= L) break;
        const long long e = (long long)y * L + x;
        float amp = 1.0f, ph = acc[j];
        if (f.stop_A) amp = __fmul_rn(amp, f.stop_A[e]);
        if (f.stop_phase) ph = __fadd_rn(ph, f.stop_phase[e]);
        if (f.dm_phase) {                 // NULL: the mirror term is left to the consumer
            if (f.dm_A) amp = __fmul_rn(amp, f.dm_A[e]);
            ph = __fadd_rn(ph, f.dm_phase[b * f.dm_stride + e]);
        }
        f.A[b * f.out_stride + e] = amp;
        f.P[b * f.out_stride + e] = ph;
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

namespace {

// the checks every layer passes before a launch reads it
int check_layer(const char *who, int k, const sb_atmo_layer &l, const LayerPtrs &ptr, int L, bool inputs) {
    // the window [pos, pos + L] must stay inside the strip for every
    // position the cycling rule allows: pos + L < screen_cols
    if (!l.screen || !l.out || l.screen_cols < L + 1 || l.screen_ld < l.screen_cols || !ptr.pos ||
        (!inputs && (l.rot90 < 0 || l.rot90 > 3 || !(l.delta >= 0.0))))
        return sb::fail(SB_EINVAL, "%s: layer %d: bad screen window", who, k);
    if (inputs && (!ptr.seeing || !ptr.wind_speed || !ptr.wind_direction))
        return sb::fail(SB_EINVAL, "%s: layer %d: null input pointer", who, k);
    // element offsets inside the strip window are 32-bit
    if ((long long)L * l.screen_ld + l.screen_cols >= (1LL << 31))
        return sb::fail(SB_ESHAPE, "%s: layer %d: strip too large", who, k);
    // the fractional-degree rotation is below 1 degree: the staged
    // footprint of a tile is sized for that
    if (!inputs && l.rotate && !(fabs(l.m01) < 0.0175 && fabs(l.m10) < 0.0175 && l.m00 > 0.9998 && l.m11 > 0.9998))
        return sb::fail(SB_EINVAL, "%s: layer %d: rotation must be below one degree", who, k);
    return SB_OK;
}

template <int CAP>
int launch_evolve_t(const char *who, const sb_atmo_layer *layers, const LayerPtrs *ptrs, int n_layers, int L,
                    const sb_atmo_inputs *in, LayerDyn *dyn, void *stream, const FusedPropArgs *fuse = nullptr) {
    EvolveArgsT<CAP> a;
    for (int k = 0; k < n_layers; ++k) {
        const int rc = check_layer(who, k, layers[k], ptrs[k], L, in != nullptr);
        if (rc) return rc;
        a.layer[k] = layers[k];
        a.ptr[k] = ptrs[k];
    }
    a.n = n_layers;
    a.L = L;
    a.dyn = dyn;
    if (in) a.in = *in;
    cudaStream_t st = sb::as_stream(stream);
    atmo_advance_kernel<CAP><<<1, CAP < 32 ? 32 : CAP, 0, st>>>(a);
    int rc = sb::check_launch("atmo_advance_kernel");
    if (rc) return rc;
    if (fuse) {
        dim3 block(32, kRowStep), grid((L + kTile - 1) / kTile, (L + kTile - 1) / kTile, n_layers / fuse->n_atm);
        atmo_propagate_kernel<CAP><<<grid, block, 0, st>>>(a, *fuse);
        return sb::check_launch("atmo_propagate_kernel");
    }
    dim3 block(32, kRowStep), grid((L + kTile - 1) / kTile, (L + kTile - 1) / kTile, n_layers);
    atmo_evolve_kernel<CAP><<<grid, block, 0, st>>>(a);
    return sb::check_launch("atmo_evolve_kernel");
}

int launch_evolve(const char *who, const sb_atmo_layer *layers, int n_layers, int L, double *positions,
                  const sb_atmo_inputs *in, LayerDyn *dyn, void *stream) {
    if (!layers || !positions || n_layers < 0 || L < 1) return sb::fail(SB_EINVAL, "%s: bad args", who);
    if (n_layers > SB_MAX_LAYERS) return sb::fail(SB_ESHAPE, "%s: at most %d layers", who, SB_MAX_LAYERS);
    if (n_layers == 0) return SB_OK;
    LayerPtrs ptrs[SB_MAX_LAYERS];
    for (int k = 0; k < n_layers; ++k) {
        ptrs[k].pos = positions + k;
        ptrs[k].seeing = in ? in->seeing : nullptr;
        ptrs[k].wind_speed = in ? in->wind_speed + (in->n_wind_speed > 1 ? k : 0) : nullptr;
        ptrs[k].wind_direction = in ? in->wind_direction + (in->n_wind_direction > 1 ? k : 0) : nullptr;
    }
    return launch_evolve_t<SB_MAX_LAYERS>(who, layers, ptrs, n_layers, L, in, dyn, stream);
}

// One realisation's field, elements e0, e0 + step, ... (the order of the sums
// does not depend on the split)
__device__ __forceinline__ void propagate_field(const float *__restrict__ at, int n_atm, long long atm_layer_stride,
                                                const float *__restrict__ stop_A,
                                                const float *__restrict__ stop_phase,
                                                const float *__restrict__ dm_A, const float *__restrict__ dp, int n,
                                                float *__restrict__ Ao, float *__restrict__ Po, int e0, int step) {
    for (int e = e0; e < n; e += step) {
        float amp = 1.0f, ph = 0.0f;
        for (int k = 0; k < n_atm; ++k) ph = __fadd_rn(ph, at[k * atm_layer_stride + e]);
        if (stop_A) amp = __fmul_rn(amp, stop_A[e]);
        if (stop_phase) ph = __fadd_rn(ph, stop_phase[e]);
        if (dm_A) amp = __fmul_rn(amp, dm_A[e]);
        ph = __fadd_rn(ph, dp[e]);
        Ao[e] = amp;
        Po[e] = ph;
    }
}

// Batched on-axis propagation of realisations with the same layer structure:
// n_atm unit-amplitude turbulence layers (rows of a stack), one shared
// amplitude/phase layer (the pupil stop) and a mirror layer with a shared
// amplitude and a per-realisation phase; same operation order as
// propagate_kernel, every layer pupil-sized (no crop).
__global__ void __launch_bounds__(256) propagate_batched_kernel(const float *__restrict__ atm, int n_atm,
                                                                long long atm_layer_stride,
                                                                long long atm_real_stride,
                                                                const float *__restrict__ stop_A,
                                                                const float *__restrict__ stop_phase,
                                                                const float *__restrict__ dm_A,
                                                                const float *__restrict__ dm_phase,
                                                                long long dm_stride, int n, float *__restrict__ A,
                                                                float *__restrict__ P, long long out_stride) {
    const long long b = blockIdx.y;
    propagate_field(atm + b * atm_real_stride, n_atm, atm_layer_stride, stop_A, stop_phase, dm_A,
                    dm_phase + b * dm_stride, n, A + b * out_stride, P + b * out_stride,
                    blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

}  // namespace

extern "C" int sb_propagate_batched(const float *atm, int n_atm, long long atm_layer_stride, long long atm_real_stride,
                                    const float *stop_A, const float *stop_phase, const float *dm_A,
                                    const float *dm_phase, long long dm_stride, int n_batch, int pupil, float *A_out,
                                    float *phase_out, long long out_stride, void *stream) {
    sb::clear_error();
    const long long n = (long long)pupil * pupil;
    if ((n_atm > 0 && !atm) || !dm_phase || !A_out || !phase_out || n_atm < 0 || n_batch < 1 || n_batch > 65535 ||
        pupil < 1 || atm_layer_stride < (n_atm > 0 ? n : 0) || dm_stride < n || out_stride < n)
        return sb::fail(SB_EINVAL, "sb_propagate_batched: bad args");
    int nblk = (int)((n + 255) / 256);
    nblk = nblk > 296 ? 296 : nblk;
    propagate_batched_kernel<<<dim3(nblk, n_batch), 256, 0, sb::as_stream(stream)>>>(
        atm, n_atm, atm_layer_stride, atm_real_stride, stop_A, stop_phase, dm_A, dm_phase, dm_stride, (int)n, A_out,
        phase_out, out_stride);
    return sb::check_launch("propagate_batched_kernel");
}

extern "C" int sb_atmo_evolve(const sb_atmo_layer *layers, int n_layers, int L, double *positions, void *stream) {
    sb::clear_error();
    return launch_evolve("sb_atmo_evolve", layers, n_layers, L, positions, nullptr, nullptr, stream);
}

extern "C" size_t sb_atmo_work_bytes(int n_layers) {
    if (n_layers < 0 || n_layers > SB_MAX_LAYERS) return 0;
    return ((size_t)n_layers * sizeof(LayerDyn) + 255) & ~(size_t)255;
}

extern "C" int sb_atmo_evolve_inputs(const sb_atmo_layer *layers, int n_layers, int L, double *positions,
                                     const sb_atmo_inputs *in, void *work, size_t work_bytes, void *stream) {
    sb::clear_error();
    if (!in || !in->seeing || !in->wind_speed || !in->wind_direction || in->n_wind_speed < 1 ||
        in->n_wind_direction < 1 || !(in->pixel_pitch > 0.0) || !(in->delta_time >= 0.0))
        return sb::fail(SB_EINVAL, "sb_atmo_evolve_inputs: bad inputs");
    if ((in->n_wind_speed != 1 && in->n_wind_speed != n_layers) ||
        (in->n_wind_direction != 1 && in->n_wind_direction != n_layers))
        return sb::fail(SB_ESHAPE, "sb_atmo_evolve_inputs: wind vectors must have 1 or %d values", n_layers);
    if (!work || work_bytes < sb_atmo_work_bytes(n_layers))
        return sb::fail(SB_ESCRATCH, "sb_atmo_evolve_inputs: work needs %zu bytes", sb_atmo_work_bytes(n_layers));
    return launch_evolve("sb_atmo_evolve_inputs", layers, n_layers, L, positions, in,
                         static_cast<LayerDyn *>(work), stream);
}

extern "C" int sb_atmo_evolve_batched(const sb_atmo_layer *layers, const sb_atmo_layer_inputs *inputs, int n_layers,
                                      int L, const sb_atmo_inputs *constants, void *work, size_t work_bytes,
                                      void *stream) {
    sb::clear_error();
    if (!layers || !inputs || !constants || n_layers < 0 || L < 1 || !(constants->pixel_pitch > 0.0) ||
        !(constants->delta_time >= 0.0))
        return sb::fail(SB_EINVAL, "sb_atmo_evolve_batched: bad args");
    if (n_layers == 0) return SB_OK;
    if (!work || work_bytes < (size_t)n_layers * sizeof(LayerDyn))
        return sb::fail(SB_ESCRATCH, "sb_atmo_evolve_batched: work needs %zu bytes", (size_t)n_layers * sizeof(LayerDyn));
    LayerPtrs ptrs[kBatchLayers];
    for (int k0 = 0; k0 < n_layers; k0 += kBatchLayers) {
        const int n = n_layers - k0 < kBatchLayers ? n_layers - k0 : kBatchLayers;
        for (int k = 0; k < n; ++k) {
            const sb_atmo_layer_inputs &li = inputs[k0 + k];
            ptrs[k].seeing = li.seeing;
            ptrs[k].wind_speed = li.wind_speed;
            ptrs[k].wind_direction = li.wind_direction;
            ptrs[k].pos = li.position;
        }
        const int rc = launch_evolve_t<kBatchLayers>("sb_atmo_evolve_batched", layers + k0, ptrs, n, L, constants,
                                                     static_cast<LayerDyn *>(work) + k0, stream);
        if (rc) return rc;
    }
    return SB_OK;
}

extern "C" int sb_atmo_propagate_batched(const sb_atmo_layer *layers, const sb_atmo_layer_inputs *inputs, int n_atm,
                                         int n_batch, int L, const sb_atmo_inputs *constants, void *work,
                                         size_t work_bytes, const float *stop_A, const float *stop_phase,
                                         const float *dm_A, const float *dm_phase, long long dm_stride, float *A_out,
                                         float *phase_out, long long out_stride, void *stream) {
    sb::clear_error();
    const long long n = (long long)L * L;
    if (!layers || !inputs || !constants || n_atm < 1 || n_atm > kBatchLayers || n_batch < 1 || L < 1 ||
        !(constants->pixel_pitch > 0.0) || !(constants->delta_time >= 0.0) || !A_out || !phase_out ||
        (dm_phase && dm_stride < n) || out_stride < n)
        return sb::fail(SB_EINVAL, "sb_atmo_propagate_batched: bad args");
    if (n_atm > kFusedMaxLayers)
        return sb::fail(SB_ESHAPE, "sb_atmo_propagate_batched: at most %d layers per realisation", kFusedMaxLayers);
    const int n_layers = n_atm * n_batch;
    if (!work || work_bytes < (size_t)n_layers * sizeof(LayerDyn))
        return sb::fail(SB_ESCRATCH, "sb_atmo_propagate_batched: work needs %zu bytes",
                        (size_t)n_layers * sizeof(LayerDyn));
    // whole realisations per launch
    const int per = (kBatchLayers / n_atm) * n_atm;
    LayerPtrs ptrs[kBatchLayers];
    for (int k0 = 0; k0 < n_layers; k0 += per) {
        const int nl = n_layers - k0 < per ? n_layers - k0 : per;
        for (int k = 0; k < nl; ++k) {
            const sb_atmo_layer_inputs &li = inputs[k0 + k];
            ptrs[k].seeing = li.seeing;
            ptrs[k].wind_speed = li.wind_speed;
            ptrs[k].wind_direction = li.wind_direction;
            ptrs[k].pos = li.position;
        }
        FusedPropArgs f;
        f.stop_A = stop_A;
        f.stop_phase = stop_phase;
        f.dm_A = dm_A;
        f.dm_phase = dm_phase;
        f.dm_stride = dm_stride;
        f.out_stride = out_stride;
        f.A = A_out;
        f.P = phase_out;
        f.n_atm = n_atm;
        f.real0 = k0 / n_atm;
        const int rc = launch_evolve_t<kBatchLayers>("sb_atmo_propagate_batched", layers + k0, ptrs, nl, L, constants,
                                                     static_cast<LayerDyn *>(work) + k0, stream, &f);
        if (rc) return rc;
    }
    return SB_OK;
}

// ---------------------------------------------------------------------------
// Monte-Carlo step, stages 1-3: every turbulence layer of every realisation of
// every group.  The layer records live in the workspace; a CTA finds its
// group from the block prefix in the kernel arguments, then its layer and
// tile, and runs the same tile code as atmo_evolve_kernel.
// ---------------------------------------------------------------------------
namespace {

struct McAtmoLayer {
    sb_atmo_layer layer;
    LayerPtrs ptr;
};

struct McAtmoGroup {
    sb_atmo_inputs in;               // constants (pointers unused)
    int layer0, n_layers, L, tiles;  // first layer in the table, count, side, tiles per side
};

struct McAtmoArgs {
    const McAtmoLayer *layers;
    LayerDyn *dyn;
    int n_groups, n_layers;
    McAtmoGroup g[sb::kMcMaxGroups];
    int blk0[sb::kMcMaxGroups + 1];   // evolve CTAs before each group
    int fblk0[sb::kMcMaxGroups + 1];  // fused evolve + propagation CTAs before each group
};

struct McPropGroup {
    const float *atm;
    long long atm_real_stride, atm_layer_stride;
    const float *stop_A, *stop_phase, *dm_A;
    const float *dm_phase[2];        // the mirror-phase buffers (the second may be NULL)
    long long dm_stride;
    float *A, *P;
    long long out_stride;
    int n_atm, n;
};

struct McPropArgs {
    int n_groups, sel;               // sel: the mirror-phase buffer read
    McPropGroup g[sb::kMcMaxGroups];
    int real0[sb::kMcMaxGroups + 1];  // realisations before each group
};

struct McAtmoBlob {
    McAtmoArgs atmo;
    McPropArgs prop;
    int evolve_blocks, prop_blocks, n_real, fused_blocks, fused;
};

__global__ void __launch_bounds__(256) mc_atmo_advance_kernel(McAtmoArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n_layers) return;
    int g = 0;
    while (g + 1 < a.n_groups && k >= a.g[g + 1].layer0) ++g;
    const McAtmoLayer &ly = a.layers[k];
    const int L = a.g[g].L;
    // as atmo_advance_kernel with device inputs
    const LayerDyn d = layer_dyn(a.g[g].in, ly.ptr, L);
    a.dyn[k] = d;
    double *pos = ly.ptr.pos;
    double np = __dadd_rn(*pos, d.delta);
    if (__dadd_rn(np, (double)L) >= (double)ly.layer.screen_cols) np = 0.0;
    *pos = np;
}

__global__ void __launch_bounds__(256) mc_atmo_evolve_kernel(McAtmoArgs a) {
    __shared__ float Q[kBox][kBox + 1];
    __shared__ TileFootprint fp;
    __shared__ LayerDyn lyd;
    const int blk = blockIdx.x;
    int g = 0;
    while (g + 1 < a.n_groups && blk >= a.blk0[g + 1]) ++g;
    const int tiles = a.g[g].tiles, L = a.g[g].L;
    const int t2 = tiles * tiles, local = blk - a.blk0[g];
    const int kl = local / t2, tt = local - kl * t2;
    const int ty = tt / tiles, tx = tt - ty * tiles;
    const int li = a.g[g].layer0 + kl;
    const McAtmoLayer &ly = a.layers[li];
    const TileSrc src{&ly.layer, ly.ptr.pos, a.dyn + li, L, tx * kTile, ty * kTile};
    float *out = ly.layer.out;
    evolve_tile(src, Q, fp, lyd, [&](int, int y, int x, float v) { out[(size_t)y * L + x] = v; });
}

// Layers and field in one launch: a CTA is one 32 x 32 tile of one
// realisation; its layers are evaluated in turn, software-pipelined and
// written as in atmo_propagate_kernel, and summed in registers in layer
// order, then the stop and mirror terms are applied in propagate_field's
// order (the same bits as mc_atmo_evolve_kernel + mc_propagate_kernel).
__global__ void __launch_bounds__(256, 3) mc_atmo_propagate_kernel(McAtmoArgs a, McPropArgs f) {
    __shared__ float Q[2][kBox][kBox + 1];
    __shared__ TileFootprint fp[kFusedMaxLayers];
    __shared__ LayerDyn lyd[kFusedMaxLayers];
    const int blk = blockIdx.x;
    int g = 0;
    while (g + 1 < a.n_groups && blk >= a.fblk0[g + 1]) ++g;
    const int tiles = a.g[g].tiles, L = a.g[g].L;
    const int t2 = tiles * tiles, local = blk - a.fblk0[g];
    const int b = local / t2, tt = local - b * t2;
    const int ty = tt / tiles, tx = tt - ty * tiles;
    const int x0 = tx * kTile, y0 = ty * kTile;
    const McPropGroup &G = f.g[g];
    const int n = G.n_atm, l0 = a.g[g].layer0 + b * n;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    auto src = [&](int li) {
        const McAtmoLayer &ly = a.layers[li];
        return TileSrc{&ly.layer, ly.ptr.pos, a.dyn + li, L, x0, y0};
    };
    if (tid < n) tile_footprint(src(l0 + tid), lyd[tid], fp[tid]);
    float acc[kTile / kRowStep];
#pragma unroll
    for (int j = 0; j < kTile / kRowStep; ++j) acc[j] = 0.0f;
    __syncthreads();
    if (n > 0) {
        TileLoads t;
        tile_load(src(l0), lyd[0], fp[0], tid, t);
        for (int k = 0; k < n; ++k) {
            tile_stage(Q[k & 1], t);
            if (k + 1 < n) tile_load(src(l0 + k + 1), lyd[k + 1], fp[k + 1], tid, t);
            __syncthreads();
            float *out = a.layers[l0 + k].layer.out;
            tile_values(L, x0, y0, Q[k & 1], lyd[k], fp[k], [&](int j, int y, int x, float v) {
                out[(size_t)y * L + x] = v;
                acc[j] = __fadd_rn(acc[j], v);
            });
        }
    }
    const int x = x0 + threadIdx.x;
    if (x >= L) return;
    const float *dp = G.dm_phase[f.sel] + b * G.dm_stride;
#pragma unroll
    for (int j = 0; j < kTile / kRowStep; ++j) {
        const int y = y0 + (int)threadIdx.y + kRowStep * j;
        if (y >= L) break;
        const long long e = (long long)y * L + x;
        float amp = 1.0f, ph = acc[j];
        if (G.stop_A) amp = __fmul_rn(amp, G.stop_A[e]);
        if (G.stop_phase) ph = __fadd_rn(ph, G.stop_phase[e]);
        if (G.dm_A) amp = __fmul_rn(amp, G.dm_A[e]);
        ph = __fadd_rn(ph, dp[e]);
        G.A[b * G.out_stride + e] = amp;
        G.P[b * G.out_stride + e] = ph;
    }
}

__global__ void __launch_bounds__(256) mc_propagate_kernel(McPropArgs a) {
    const int r = blockIdx.y;
    int g = 0;
    while (g + 1 < a.n_groups && r >= a.real0[g + 1]) ++g;
    const McPropGroup &G = a.g[g];
    const long long b = r - a.real0[g];
    propagate_field(G.atm ? G.atm + b * G.atm_real_stride : nullptr, G.n_atm, G.atm_layer_stride, G.stop_A,
                    G.stop_phase, G.dm_A, G.dm_phase[a.sel] + b * G.dm_stride, G.n, G.A + b * G.out_stride,
                    G.P + b * G.out_stride, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

}  // namespace

namespace sb {

size_t mc_atmo_workspace(const sb_mc_group *gs, int n) {
    size_t nl = 0;
    for (int g = 0; g < n; ++g) nl += (size_t)gs[g].n_batch * gs[g].n_atm;
    return mc_align(nl * sizeof(McAtmoLayer)) + mc_align(nl * sizeof(LayerDyn));
}

int mc_atmo_prepare(const sb_mc_group *gs, int n, void *ws, McBlob &blob, cudaStream_t st) {
    static_assert(sizeof(McAtmoBlob) <= sizeof(McBlob), "atmosphere stage arguments exceed the blob");
    static_assert(sizeof(McAtmoArgs) <= 4096 && sizeof(McPropArgs) <= 4096, "kernel arguments above 4 KB");
    const char *who = "sb_mc_create";
    McAtmoBlob *B = new (blob.b) McAtmoBlob();
    size_t nl = 0;
    for (int g = 0; g < n; ++g) nl += (size_t)gs[g].n_batch * gs[g].n_atm;
    std::vector<McAtmoLayer> tab(nl);
    McAtmoArgs &a = B->atmo;
    McPropArgs &p = B->prop;
    a.layers = static_cast<const McAtmoLayer *>(ws);
    a.dyn = reinterpret_cast<LayerDyn *>(static_cast<unsigned char *>(ws) + mc_align(nl * sizeof(McAtmoLayer)));
    a.n_groups = p.n_groups = n;
    a.n_layers = (int)nl;
    int k = 0, blocks = 0, real = 0, max_n = 1, fblocks = 0, fused = 1;
    for (int g = 0; g < n; ++g) {
        const sb_mc_group &G = gs[g];
        const int L = G.L, cnt = G.n_batch * G.n_atm;
        const sb_atmo_inputs &in = G.constants;
        if (!(in.pixel_pitch > 0.0) || !(in.delta_time >= 0.0) || L < 1 || G.n_atm < 0 || (cnt && (!G.layers || !G.inputs)))
            return fail(SB_EINVAL, "%s: group %d: bad atmosphere", who, g);
        const int tiles = (L + kTile - 1) / kTile;
        a.g[g].in = in;
        a.g[g].layer0 = k;
        a.g[g].n_layers = cnt;
        a.g[g].L = L;
        a.g[g].tiles = tiles;
        a.blk0[g] = blocks;
        a.fblk0[g] = fblocks;
        fblocks += G.n_batch * tiles * tiles;
        fused &= G.n_atm <= kFusedMaxLayers;
        for (int j = 0; j < cnt; ++j, ++k) {
            const sb_atmo_layer_inputs &li = G.inputs[j];
            tab[k].layer = G.layers[j];
            tab[k].ptr.seeing = li.seeing;
            tab[k].ptr.wind_speed = li.wind_speed;
            tab[k].ptr.wind_direction = li.wind_direction;
            tab[k].ptr.pos = li.position;
            const int rc = check_layer(who, j, tab[k].layer, tab[k].ptr, L, true);
            if (rc) return rc;
            // the layers are the rows of atm, as the propagation reads them
            const float *want = G.atm + (j / G.n_atm) * G.atm_real_stride + (long long)(j % G.n_atm) * L * L;
            if (tab[k].layer.out != want)
                return fail(SB_EINVAL, "%s: group %d: layer %d does not write its row of atm", who, g, j);
        }
        blocks += cnt * tiles * tiles;
        McPropGroup &q = p.g[g];
        const long long nn = (long long)L * L;
        if (!G.dm_phase || !G.field_A || !G.field_phase || G.dm_stride < nn || G.field_stride < nn ||
            (G.n_atm > 0 && (!G.atm || G.atm_real_stride < G.n_atm * nn)))
            return fail(SB_EINVAL, "%s: group %d: bad propagation buffers", who, g);
        q.atm = G.atm;
        q.atm_real_stride = G.atm_real_stride;
        q.atm_layer_stride = nn;
        q.stop_A = G.stop_A;
        q.stop_phase = G.stop_phase;
        q.dm_A = G.dm_A;
        q.dm_phase[0] = G.dm_phase;
        q.dm_phase[1] = G.dm_phase_alt;
        q.dm_stride = G.dm_stride;
        q.A = G.field_A;
        q.P = G.field_phase;
        q.out_stride = G.field_stride;
        q.n_atm = G.n_atm;
        q.n = (int)nn;
        p.real0[g] = real;
        real += G.n_batch;
        max_n = nn > max_n ? (int)nn : max_n;
    }
    a.blk0[n] = blocks;
    a.fblk0[n] = fblocks;
    p.real0[n] = real;
    B->fused_blocks = fblocks;
    B->fused = fused;
    B->evolve_blocks = blocks;
    B->n_real = real;
    const int nblk = (max_n + 255) / 256;
    B->prop_blocks = nblk > 296 ? 296 : nblk;
    if (real > 65535) return fail(SB_ESHAPE, "%s: at most 65535 realisations", who);
    if (nl) {
        const cudaError_t e = cudaMemcpyAsync(ws, tab.data(), nl * sizeof(McAtmoLayer), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(SB_ECUDA, "%s: layer table copy: %s", who, cudaGetErrorString(e));
    }
    return SB_OK;
}

int mc_atmo_launch(const McBlob &blob, int sel, cudaStream_t st) {
    const McAtmoBlob *B = reinterpret_cast<const McAtmoBlob *>(blob.b);
    McPropArgs p = B->prop;
    p.sel = sel;
    for (int g = 0; g < p.n_groups; ++g)
        if (!p.g[g].dm_phase[sel]) return fail(SB_EINVAL, "sb_mc_stage: group %d has no second mirror buffer", g);
    if (B->atmo.n_layers > 0) {
        mc_atmo_advance_kernel<<<(B->atmo.n_layers + 255) / 256, 256, 0, st>>>(B->atmo);
        const int rc = check_launch("mc_atmo_advance_kernel");
        if (rc) return rc;
    }
    if (B->fused) {
        mc_atmo_propagate_kernel<<<B->fused_blocks, dim3(32, kRowStep), 0, st>>>(B->atmo, p);
        return check_launch("mc_atmo_propagate_kernel");
    }
    // a group with more layers than the fused kernel stages: layers, then the field
    if (B->atmo.n_layers > 0) {
        mc_atmo_evolve_kernel<<<B->evolve_blocks, dim3(32, kRowStep), 0, st>>>(B->atmo);
        const int rc = check_launch("mc_atmo_evolve_kernel");
        if (rc) return rc;
    }
    mc_propagate_kernel<<<dim3(B->prop_blocks, B->n_real), 256, 0, st>>>(p);
    return check_launch("mc_propagate_kernel");
}

}  // namespace sb

namespace {
struct PropSampArgs {
    sb_prop_sampling layer[SB_MAX_LAYERS];
    int n, pupil;
};

// bilinear at (y, x) on the integer grid, in double (RegularGridInterpolator)
__device__ __forceinline__ float bilinear(const float *v, int ld, int rows, int cols, double y, double x) {
    int y0 = (int)floor(y), x0 = (int)floor(x);
    y0 = max(0, min(y0, rows - 2));
    x0 = max(0, min(x0, cols - 2));
    const double fy = y - y0, fx = x - x0;
    const size_t i00 = (size_t)y0 * ld + x0;
    return (float)(v[i00] * ((1 - fy) * (1 - fx)) + v[i00 + 1] * ((1 - fy) * fx) + v[i00 + ld] * (fy * (1 - fx)) +
                   v[i00 + ld + 1] * (fy * fx));
}

__global__ void __launch_bounds__(256) propagate_sampling_kernel(PropSampArgs a, float *__restrict__ A,
                                                                 float *__restrict__ P) {
    const int n = a.pupil * a.pupil;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int r = e / a.pupil, c = e - r * a.pupil;
        float amp = 1.0f, ph = 0.0f;                       // ElectricField.reset()
        for (int k = 0; k < a.n; ++k) {
            const sb_prop_sampling &l = a.layer[k];
            if (l.yy) {
                const double y = l.yy[e], x = l.xx[e];
                if (l.A) amp = __fmul_rn(amp, bilinear(l.A, l.ld, l.rows, l.cols, y, x));
                if (l.phase) ph = __fadd_rn(ph, bilinear(l.phase, l.ld, l.rows, l.cols, y, x));
            } else {
                const size_t g = (size_t)(r + l.top) * l.ld + (c + l.left);
                if (l.A) amp = __fmul_rn(amp, l.A[g]);
                if (l.phase) ph = __fadd_rn(ph, l.phase[g]);
            }
        }
        A[e] = amp;
        P[e] = ph;
    }
}
}  // namespace

extern "C" int sb_propagate(const sb_prop_sampling *layers, int n_layers, int pupil, float *A_out, float *phase_out,
                            void *stream) {
    sb::clear_error();
    if (!layers || !A_out || !phase_out || n_layers < 0 || pupil < 1)
        return sb::fail(SB_EINVAL, "sb_propagate: bad args");
    if (n_layers > SB_MAX_LAYERS) return sb::fail(SB_ESHAPE, "sb_propagate: at most %d layers", SB_MAX_LAYERS);
    PropSampArgs a;
    for (int k = 0; k < n_layers; ++k) {
        const sb_prop_sampling &l = layers[k];
        if (l.yy || l.xx) {
            if (!l.yy || !l.xx || l.rows < 2 || l.cols < 2 || l.ld < l.cols)
                return sb::fail(SB_EINVAL, "sb_propagate: layer %d: bad sampling grid", k);
        } else if (l.top < 0 || l.left < 0 || l.ld < pupil + l.left || (l.rows && l.rows < pupil + l.top)) {
            return sb::fail(SB_EINVAL, "sb_propagate: layer %d: bad crop", k);
        }
        a.layer[k] = l;
    }
    a.n = n_layers;
    a.pupil = pupil;
    int nblk = (pupil * pupil + 255) / 256;
    nblk = nblk > 1184 ? 1184 : nblk;
    propagate_sampling_kernel<<<nblk, 256, 0, sb::as_stream(stream)>>>(a, A_out, phase_out);
    return sb::check_launch("propagate_sampling_kernel");
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
