/*
 * specula_b200.h — C ABI of the B200 closed-loop Shack-Hartmann step.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), launches its kernels on that stream and returns an int
 * status (SB_OK == 0, negative on error; sb_last_error() describes the last
 * failure of the calling thread).  No entry point allocates device memory or
 * synchronises the host, so a sequence of calls can be captured in a CUDA
 * graph.  Work buffers ("scratch") are passed in by the caller; their size is
 * given by the matching *_scratch_bytes() query.
 *
 * Each function cites the reference (SPECULA) code it replaces; paths are
 * relative to the SPECULA project root.  The Python processing objects of
 * the package (specula_b200.processing_objects.*) call these through ctypes
 * from their trigger_code().
 */
#ifndef SPECULA_B200_H
#define SPECULA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB_OK 0
#define SB_EINVAL (-1)        /* bad pointer or parameter value            */
#define SB_ESHAPE (-2)        /* sizes outside what the kernels support     */
#define SB_ECUDA (-3)         /* a CUDA launch or query failed              */
#define SB_ESCRATCH (-4)      /* scratch buffer missing or too small        */
#define SB_ETIMEOUT (-5)      /* a bounded device-side wait gave up         */
#define SB_EUNSUPPORTED (-6)  /* option not implemented on this path        */

/* ABI version (major*100 + minor). */
int sb_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char *sb_last_error(void);

/* ------------------------------------------------------------------------
 * SH sensor forward model
 * replaces specula/processing_objects/sh.py:348-420 (trigger_code: field
 * build, zero-padded FFT, |E|^2, fftshift, field-stop mask, FoV cut, mosaic)
 * + specula/lib/toccd.py:33-113 (LCM area rebin)
 * + specula/processing_objects/sh.py:422-428 (post_trigger photon
 * normalisation i *= S0*masked_area/sum(i)).
 *
 * Geometry integers come from the host-side solve that restates
 * sh.py:112-323.  The DFT is evaluated only on the cut window and only from
 * the np x np non-zero samples of each zero-padded sub-aperture.
 * ---------------------------------------------------------------------- */
typedef struct sb_sh_plan {
    int n_lenses;        /* sub-apertures per side (Lenslet.dimx == dimy)      */
    int np_sub;          /* field samples per sub-aperture side (ovs_np_sub)   */
    int cutsize;         /* focal-plane samples kept per side (fft - cut)      */
    int subap_npx;       /* detector pixels per sub-aperture side              */
    int field_ld;        /* row stride (elements) of A and phase               */
    float phase_to_rad;  /* float32(2*pi/lambda_nm)                            */
    /* device tables, all float32, prepared once at setup */
    const float *twiddle;  /* [cutsize][np_sub][2]: exp(-2*pi*i*k_b*c/fft)    */
    const float *tilt;     /* [np_sub][np_sub][2]: half-pixel tilt (sh.py:469) */
    const float *fp_mask;  /* [cutsize][cutsize]: field stop on the cut window */
    const float *rebin;    /* [subap_npx][cutsize]: LCM overlap / dx_out       */
} sb_sh_plan;

size_t sb_sh_scratch_bytes(const sb_sh_plan *plan);

/*
 * A, phase_nm: the sampled field, (n_lenses*np_sub) rows of field_ld floats.
 * A_norm: amplitude of the field the SH object received (n_norm floats; the
 *   same pointer as A unless the field was resampled).
 * photon_scale: S0 * pixel_pitch^2 of that field.
 * intensity: (n_lenses*subap_npx)^2 float32, row-major, scaled so that its
 *   sum equals photon_scale * sum(A_norm) (sh.py:425-427).
 */
int sb_sh_forward(const sb_sh_plan *plan, const float *A, const float *phase_nm,
                  const float *A_norm, int n_norm, float photon_scale, float *intensity,
                  void *scratch, size_t scratch_bytes, void *stream);

/*
 * No counterpart in the reference.  Same computation as sb_sh_forward, for
 * callers that cannot allocate device memory: a real-time control thread
 * that must not allocate once the loop runs, or a foreign-language binding
 * that holds device buffers for its inputs and outputs but has no CUDA
 * allocator of its own.  The caller still passes inputs and outputs; the
 * scratch is a file-scope device array of SB_SH_STATIC_SCRATCH_BYTES bytes
 * (every GPU that loads the library keeps it until the process exits).
 * Geometries whose sb_sh_scratch_bytes() exceeds that size are rejected with
 * SB_ESCRATCH.  The first call on a device resolves the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  The address is kept for the life of the
 * process, so the device must not be reset (cudaDeviceReset) after that first
 * call.  With the default 64 KB the largest grid is 128 x 128 lenslets
 * (sb_sh_scratch_bytes sizes for two sub-apertures per CTA:
 * ceil(n/2) * n * 8 bytes).  All calls share the array: the kernels
 * overwrite every partial sum they read, so no clearing is needed, but calls
 * that overlap on the GPU (different streams, or concurrent graphs) race on
 * it and must be serialised by the caller.
 */
#define SB_SH_STATIC_SCRATCH_BYTES (64 * 1024)
int sb_sh_forward_static(const sb_sh_plan *plan, const float *A, const float *phase_nm,
                         const float *A_norm, int n_norm, float photon_scale, float *intensity,
                         void *stream);

/* Batched form for Monte-Carlo realisations sharing one plan: realisation b
 * (blockIdx.z) reads A + b*A_stride, phase_nm + b*phase_stride, A_norm +
 * b*A_norm_stride (strides in floats; 0 shares one array) and writes its
 * normalised frame at intensity + b*intensity_stride.  scratch: n_batch *
 * sb_sh_scratch_bytes(plan) bytes.  Each frame equals sb_sh_forward's. */
int sb_sh_forward_batched(const sb_sh_plan *plan, const float *A, long long A_stride, const float *phase_nm,
                          long long phase_stride, const float *A_norm, long long A_norm_stride, int n_norm,
                          float photon_scale, float *intensity, long long intensity_stride, int n_batch,
                          void *scratch, size_t scratch_bytes, void *stream);

/* Split-BF16 tensor-core form of sb_sh_forward / sb_sh_forward_batched (same
 * arguments, scratch and outputs; the reference computes the same quantity
 * in sh.py:348-428 with complex64 FFTs).  Both small DFT products run on
 * the tcgen05 tensor cores with every operand split into bf16 hi + lo parts
 * and hi*hi + lo*hi + hi*lo accumulated in FP32 (relative error of order
 * 1e-5 of the field, against about 1e-7 for the FP32 form).  Geometries:
 * np_sub 8 with (cutsize, subap_npx) in (12,6) (8,8) (12,8) (14,8) (16,8);
 * others return SB_EUNSUPPORTED.  A timed-out wait on the tensor cores is
 * reported by sb_device_status. */
int sb_sh_split_bf16_supported(const sb_sh_plan *plan);
int sb_sh_forward_split_bf16(const sb_sh_plan *plan, const float *A, const float *phase_nm,
                             const float *A_norm, int n_norm, float photon_scale, float *intensity,
                             void *scratch, size_t scratch_bytes, void *stream);
int sb_sh_forward_split_bf16_batched(const sb_sh_plan *plan, const float *A, long long A_stride,
                                     const float *phase_nm, long long phase_stride, const float *A_norm,
                                     long long A_norm_stride, int n_norm, float photon_scale, float *intensity,
                                     long long intensity_stride, int n_batch, void *scratch,
                                     size_t scratch_bytes, void *stream);

/* Laser-guide-star SH (replaces the kernel branch of sh.py:382-394 with the
 * kernel spectra of data_objects/convolution_kernel.py:260-276): per
 * sub-aperture the unshifted |FFT|^2 of the tilted, zero-padded field on
 * the full fft_size grid is correlated with the sub-aperture's sodium-spot
 * kernel, psf = Re(IFFT(FFT(|F|^2) * K)) with an unnormalised inverse, then
 * field stop, cut, rebin and photon normalisation as in sb_sh_forward.
 * Tables (complex64, host-built): w_full_t[c][k] = exp(-2 pi i k c / N)
 * (np_sub x N), w_dft[u][x] = exp(-2 pi i u x / N) (N x N), v_inv_t[u][a] =
 * exp(+2 pi i (a + cutpixels/2) u / N) (N x cutsize); kernel_spectra: one
 * N x N spectrum per lenslet, lenslet row-major.  Geometries: np_sub 8 with
 * (N, cutsize, npx) in (16,12,6) (32,12,6) (16,14,8) (32,16,8). */
typedef struct sb_sh_lgs_tables {
    int fft_size;
    const void *w_full_t;
    const void *w_dft;
    const void *v_inv_t;
    const void *kernel_spectra;
} sb_sh_lgs_tables;
int sb_sh_lgs_supported(const sb_sh_plan *plan, int fft_size);
int sb_sh_forward_lgs(const sb_sh_plan *plan, const sb_sh_lgs_tables *lgs, const float *A, const float *phase_nm,
                      const float *A_norm, int n_norm, float photon_scale, float *intensity, void *scratch,
                      size_t scratch_bytes, void *stream);

/* replaces specula/lib/extrapolate_edge_pixel.py:4-28.
 * out[p] = phase[p] if src1[p] < 0; phase[src1[p]] if src2[p] < 0;
 * else 2*phase[src1[p]] - phase[src2[p]].  Tables from the host restatement
 * of specula/lib/extrapolate_edge_pixel_mat_define.py:5-143. */
int sb_edge_extrapolate(const float *phase, const int32_t *src1, const int32_t *src2,
                        int n_pixels, float *out, void *stream);

/* replaces specula/lib/interp2d.py:95-122 for the SH oversampling
 * (sh.py:353-357): bilinear resampling of A and phase at precomputed,
 * clamped coordinates yy/xx (float32, n_out entries) of an in_rows x in_cols
 * input; the last input row is handled like the reference kernel
 * (interp2d.py:31-38). */
int sb_interp2d_field(const float *A_in, const float *phase_in, int in_rows, int in_cols,
                      const float *yy, const float *xx, int n_out,
                      float *A_out, float *phase_out, void *stream);

/* ------------------------------------------------------------------------
 * CCD — replaces specula/processing_objects/ccd.py:198-287 (integration,
 * binning 1, QE, background/dark, Poisson photon noise, Gaussian readout,
 * ADU quantisation).  Noise is drawn from a counter-based Philox4x32-10
 * stream keyed by (seed, frame, pixel): deterministic and reproducible.
 * ---------------------------------------------------------------------- */
typedef struct sb_ccd_state {   /* device-resident, zero-initialised      */
    uint64_t frame_index;   /* frames read so far: the RNG counter            */
    int n_integrated;       /* loop steps integrated into the open frame      */
    unsigned int blocks_done;  /* internal: completion count of the last launch */
} sb_ccd_state;

typedef struct sb_ccd_params {
    int n_pixels;
    int frames_per_read;    /* detector dt / loop dt (ccd.py:59-63,207)       */
    float rate;             /* loop_dt_s * bandw (ccd.py:205)                 */
    float qe;
    float bg_plus_dark;     /* added when background or dark noise is on      */
    int photon_noise;
    int readout_noise;
    float readout_level;
    float adu_gain;
    float adu_bias;
    float dark_level;       /* subtracted after ADU when dark noise is on     */
    int dark_noise;
    uint64_t photon_seed;
    uint64_t readout_seed;
    sb_ccd_state *state;    /* device pointer; advanced by the kernel itself  */
    /* detector-structure options (ccd.py:223-245), in the reference's order
     * around the photon and read-out noise; all zero / NULL: off */
    int cic_noise;          /* + Bernoulli(cic_level) electrons before the photon noise */
    float cic_level;
    int excess_noise;       /* EMCCD after the photon noise: n -> Gamma(delta n,
                             * emccd_gain) / delta, then / emccd_gain after ADU */
    float excess_delta;
    float emccd_gain;
    uint64_t excess_seed;
    const float *pixel_gains;  /* per-pixel gains after the read-out noise */
    const float *qe_map;       /* per-pixel QE applied with qe (notUniformQe) */
    int qe_map_normalise;      /* divide by qe_map after the noise */
} sb_ccd_params;

/* One loop step: integrate; when the frame closes, read it out into
 * `pixels` (otherwise `pixels` is left untouched).  The frame counter and
 * the integration count live in *state, so repeated calls (or replays of a
 * captured graph) draw fresh noise every frame. */
int sb_ccd_step(const sb_ccd_params *p, const float *intensity, float *integrated,
                float *pixels, void *stream);

/* CCD with b x b binning (ccd.py:198-216, 262-280): p->n_pixels is the full
 * rows x cols frame, integrated every step; on a readout step the block sums
 * S are formed and scaled as the reference does, S * b^2 * (sum(frame) /
 * sum(S)), and the QE / noise / ADU model of sb_ccd_step runs on the
 * (rows/b) x (cols/b) binned pixels (RNG counter: the binned index).
 * Scratch: sb_ccd_binned_scratch_bytes (0 when the frame is not divisible). */
size_t sb_ccd_binned_scratch_bytes(int rows, int cols, int binning);
int sb_ccd_step_binned(const sb_ccd_params *p, int rows, int cols, int binning, const float *intensity,
                       float *integrated, float *pixels, void *scratch, size_t scratch_bytes, void *stream);

/* CCD step with charge-transfer inefficiency (ccd.py:223-224): on a
 * read-out step the frame after QE and background becomes cte0 * frame *
 * cte1 (row-major side x side matrices, FP32 products) before the noise and
 * the ADU model of sb_ccd_step; no binning.  scratch:
 * sb_ccd_cte_scratch_bytes(side) bytes. */
size_t sb_ccd_cte_scratch_bytes(int side);
int sb_ccd_step_cte(const sb_ccd_params *p, int side, const float *cte0, const float *cte1, const float *intensity,
                    float *integrated, float *pixels, void *scratch, size_t scratch_bytes, void *stream);

/* Batched CCD step: n_batch frames of p->n_pixels each, contiguous in
 * intensity / integrated / pixels; frame b draws its noise with
 * photon_seeds[b] / readout_seeds[b] (device arrays) and its own pixel
 * indices, so it equals sb_ccd_step with those seeds.  One frame state
 * (p->state) for all: the realisations integrate and read out in step. */
int sb_ccd_step_batched(const sb_ccd_params *p, const uint64_t *photon_seeds, const uint64_t *readout_seeds,
                        int n_batch, const float *intensity, float *integrated, float *pixels, void *stream);

/* Raw Philox4x32-10 stream, for determinism tests: out[4*i..4*i+3] is the
 * block for counter (i, c1, c2, c3) under key (key0, key1). */
int sb_philox_raw(uint32_t key0, uint32_t key1, uint32_t c1, uint32_t c2, uint32_t c3,
                  int n_blocks, uint32_t *out, void *stream);

/* ------------------------------------------------------------------------
 * ShSlopec — replaces specula/processing_objects/sh_slopec.py:308-438
 * (calc_slopes_nofor: gather, threshold, clamp, CoG with the
 * 1e-3*mean(flux) cut-off) with weights from sh_slopec.py:86-132.
 * slopes = [sx(0..n-1), sy(0..n-1)] (slopes.py:26-33).
 * ---------------------------------------------------------------------- */
typedef struct sb_slopec_plan {
    int n_subaps;
    int npx2;               /* pixels per sub-aperture (np_sub^2)             */
    float thr;              /* subtracted then clamped at 0 (0: no threshold) */
    const int32_t *idxs;    /* [n_subaps][npx2] flat indices into the frame   */
    const float *xw;        /* [npx2] x weights                               */
    const float *yw;        /* [npx2] y weights                               */
    const float *mw;        /* [npx2] mask weights                            */
    /* options of calc_slopes_nofor (sh_slopec.py:356-420); zero / NULL: off  */
    int thr_pedestal;       /* pixels below thr set to 0, the others kept     */
    float thr_ratio;        /* > 0: each sub-aperture's thr = thr_ratio * its
                             * largest (windowed) pixel                        */
    const float *window;    /* [npx2][n_subaps] weights after the flux sums   */
    float mult;             /* != 0: slopes *= mult                           */
} sb_slopec_plan;

size_t sb_slopec_scratch_bytes(const sb_slopec_plan *plan);
int sb_slopec(const sb_slopec_plan *plan, const float *pixels, float *slopes, float *flux,
              void *scratch, size_t scratch_bytes, void *stream);

/* Batched: frame b at pixels + b*frame_stride, slopes at slopes +
 * b*slopes_stride, flux at flux + b*flux_stride; scratch n_batch *
 * sb_slopec_scratch_bytes(plan) bytes. */
int sb_slopec_batched(const sb_slopec_plan *plan, const float *pixels, long long frame_stride, float *slopes,
                      int slopes_stride, float *flux, int flux_stride, int n_batch, void *scratch,
                      size_t scratch_bytes, void *stream);

/*
 * One loop step's per-sub-aperture chain, SH forward to slopes, in two
 * launches: the SH forward of sb_sh_forward (dft_mode 0) or
 * sb_sh_forward_split_bf16 (dft_mode 1) without its normalisation launch,
 * then one kernel that applies the photon normalisation (sh.py:425-427),
 * runs the detector of sb_ccd_step (ccd.py:198-287) and the CoG of sb_slopec
 * (sh_slopec.py:308-438) on each lenslet's pixels while they are in shared
 * memory, and lets its last CTA apply the 1e-3 * mean flux cut-off and
 * advance the detector frame state.  Replaces the five launches of
 * sb_sh_forward + sb_ccd_step + sb_slopec in the loop step
 * (SH.trigger_code, CCD.trigger_code, ShSlopec.trigger_code) with the same
 * results bit for bit: intensity (normalised), integrated, pixels, slopes
 * (the [sx..., sy...] layout) and flux are written as those calls write them.
 * Conditions: the detector reads out every loop step (frames_per_read 1) at
 * the SH frame size with no binning, subap_npx <= 16, and the sub-aperture
 * table lists each valid lenslet's npx x npx box row-major;
 * lenslet_subap[i * n_lenses + j] is the valid sub-aperture index of lenslet
 * (row i, column j) or -1.  scratch: sb_sh_ccd_slopec_scratch_bytes(sh,
 * n_subaps) bytes, no initialisation needed.
 * mirror_A / mirror_phase (dft_mode 0 only; NULL: none): the last layer of
 * the on-axis propagation (atmo_propagation.py:105-144), applied while the
 * field is read: the SH sees amplitude A * mirror_A and phase phase_nm +
 * mirror_phase (A, phase_nm then hold the product and sum of the other
 * layers, in their order), the photon normalisation uses that amplitude
 * (A_norm must be A, n_norm the whole field), and the field is written to
 * field_A / field_phase (the AtmoPropagation output) when they are given.
 * So the turbulence of a step can be computed before the mirror of the
 * previous step is known.
 */
size_t sb_sh_ccd_slopec_scratch_bytes(const sb_sh_plan *sh, int n_subaps);
int sb_sh_ccd_slopec(const sb_sh_plan *sh, int dft_mode, const float *A, const float *phase_nm,
                     const float *A_norm, int n_norm, const float *mirror_A, const float *mirror_phase,
                     float *field_A, float *field_phase, float photon_scale, float *intensity,
                     const sb_ccd_params *ccd, float *integrated, float *pixels,
                     const sb_slopec_plan *slopec, const int32_t *lenslet_subap, float *slopes,
                     float *flux, void *scratch, size_t scratch_bytes, void *stream);

/* One SCAO system split over GPUs by bands of lenslet rows (the reference
 * steps the whole pupil in one process; a band is rows row0 .. row0+n_rows-1
 * of the lenslet grid).  Per step on every GPU:
 *   sb_sh_forward_rows   the band's SH frame rows, unnormalised, and the
 *                        per-CTA partial sums in the WHOLE grid's layout
 *                        (2 x sb_sh_rows_parts floats at the start of
 *                        scratch: frame sums, then A_norm sums), written for
 *                        the band's CTAs only
 *   [sum the bands' partial arrays: zero outside each band, so the sum is
 *    the array of one whole-grid launch, bit for bit]
 *   sb_ccd_slopec_rows   photon normalisation from the summed partials, CCD and
 *                        CoG of the band: its pixels, and tot / sxn / syn
 *                        (work: 3 x n_valid floats) / flux / slopes of its
 *                        valid sub-apertures at their places
 *   [sum the bands' slope, flux and work vectors]
 *   sb_slopec_cutoff     the flux cut-off on the summed vectors
 * then the reconstructor on the whole slope vector and the mirror on the
 * band's influence-function columns (sb_dm_project on a column range).
 * The results are those of sb_sh_ccd_slopec on the whole system, bit for
 * bit (the CCD draws use the whole frame's pixel indices).  Compile-time SH
 * geometries; the detector read out every step without binning. */
int sb_sh_rows_parts(const sb_sh_plan *plan, int dft_mode);
int sb_sh_forward_rows(const sb_sh_plan *plan, int dft_mode, int row0, int n_rows, const float *A,
                       const float *phase_nm, const float *A_norm, int n_norm, float *intensity, void *scratch,
                       size_t scratch_bytes, void *stream);
int sb_ccd_slopec_rows(const sb_sh_plan *sh, const float *parts, int nparts, float photon_scale, int row0,
                       int n_rows, float *intensity, const sb_ccd_params *ccd, float *integrated, float *pixels,
                       const sb_slopec_plan *slopec, const int32_t *lenslet_subap, float *slopes, float *flux,
                       float *work, void *stream);
int sb_slopec_cutoff(const float *tot, const float *sxn, const float *syn, int n_valid, float *slopes,
                     void *stream);

/* ------------------------------------------------------------------------
 * Modalrec — replaces specula/processing_objects/modalrec.py:159
 * (modes = R @ slopes), R row-major (n_modes x n_slopes).
 * ---------------------------------------------------------------------- */
int sb_modalrec(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes,
                float *modes, void *stream);

/* ------------------------------------------------------------------------
 * Integrator — replaces specula/processing_objects/iir_filter.py:100-211
 * for the 2-tap filters built by iir_filter_data.py:264-292 (num=[0,g],
 * den=[-ff,1]); state is (n x total) with total = ceil(delay)+1, ist/ost are
 * (n x 2, or n x n_num / n x n_den for general filters of up to 8 taps).
 * Output = state[:, delay] (integer delay) or the fractional mix.
 * ---------------------------------------------------------------------- */
typedef struct sb_iir_plan {
    int n;
    int total;              /* state columns (ceil(delay) + 1)                */
    int shift;              /* delay > 0: shift the state buffer first        */
    int k_out;              /* state column read (int(delay) or ceil(delay))  */
    float rem;              /* delay % 1 (0: integer delay)                   */
    float one_minus_rem;    /* 1 - (delay % 1), rounded once on the host      */
    const float *num;       /* [n][2] */
    const float *den;       /* [n][2] */
    float *ist;             /* [n][2] */
    float *ost;             /* [n][2] */
    float *state;           /* [n][total] */
    float *out_next;        /* optional [n]: the output the NEXT step will
                               emit (state[:, k_out-1] after this update),
                               for integer delays >= 1; NULL to skip.  Lets a
                               caller start the next step's DM projection
                               before that step's integrator runs.          */
    int n_num, n_den;       /* taps of num / den (and of ist / ost), 2..8;
                               0 means 2 (the integrator)                    */
} sb_iir_plan;

int sb_integrator(const sb_iir_plan *plan, const float *delta, float *out, void *stream);

/* Modalrec followed by the Integrator in one launch (modalrec.py:159 then
 * iir_filter.py:100-211): modes = R @ slopes, then the filter of mode m
 * consumes modes[m].  Results are identical to sb_modalrec + sb_integrator;
 * used when both objects are captured in one loop graph. */
int sb_modalrec_integrator(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes,
                           float *modes, const sb_iir_plan *plan, float *out, void *stream);

/* ------------------------------------------------------------------------
 * DM — replaces specula/processing_objects/dm.py:72-86:
 * phase[mask_idx[p]] = sum_m (sign * cmd[m]) * IF[m][p]; IF row-major
 * (n_modes x n_valid) with row stride ld_if >= n_valid.  Pixels outside the
 * mask are not written.  With 16-byte aligned rows and up to 4096 modes the
 * influence functions are streamed by 2-D TMA loads (one CTA per SM, small
 * register and shared-memory footprint so concurrent kernels co-reside).
 * ---------------------------------------------------------------------- */
int sb_dm_project(const float *ifunc, int n_modes, int n_valid, int ld_if,
                  const float *cmd, int n_cmd, float sign, const int32_t *mask_idx,
                  float *phase, void *stream);

/* Batched form for Monte-Carlo realisations sharing one mirror: for
 * b < n_batch, phase[b * phase_stride + mask_idx[p]] =
 * sum_m (sign * cmd[b * ld_cmd + m]) * IF[m][p].  Each influence-function
 * element is read once per 16 realisations (same TMA pipeline as
 * sb_dm_project, 5 stages); up to 1024 modes, 16-byte aligned IF rows. */
int sb_dm_project_batched(const float *ifunc, int n_modes, int n_valid, int ld_if, const float *cmd,
                          int ld_cmd, int n_batch, float sign, const int32_t *mask_idx, float *phase,
                          long long phase_stride, void *stream);

/* Batched Modalrec (modalrec.py:159) for realisations sharing one
 * reconstructor: modes[b * ldm + m] = sum_j R[m][j] * slopes[b * lds + j];
 * R is read once per 16 realisations. */
int sb_modalrec_batched(const float *R, int n_modes, int n_slopes, int ldr, const float *slopes, int lds,
                        int n_batch, float *modes, int ldm, void *stream);

/* ------------------------------------------------------------------------
 * Tile-shape tuning (an addition; the reference has no tuned kernels).  A
 * tunable kernel family has several compiled tile shapes ("variants"); a
 * launch uses the variant registered for its shape key, variant 0 when none
 * is.  specula_b200.autotune times every variant on the caller's shapes and
 * registers the fastest.  Registration is host state read when a launch is
 * made (so a captured graph keeps the variant it was captured with).
 *   SB_TUNE_DM_BATCHED  sb_dm_project_batched; key sb_tune_key(n_modes, n_valid, n_batch);
 *                       realisations per pass (16, 8, 4) x mode rows of a stage split over 1 or 2 warp groups
 *                       (variants 0-5), or the register-blocked form (4 columns x 8 or 16 realisations
 *                       per thread) with 8 (6-8) or 16 (9-11) realisations per pass in 1024-, 512- or
 *                       256-column tiles
 *   SB_TUNE_SH_FP32     sb_sh_forward / sb_sh_forward_batched; key sb_tune_key(n_lenses, cutsize, n_batch);
 *                       sub-apertures per CTA (8, 4, 2) with each CTA's field tile staged in shared
 *                       memory by 2-D TMA loads where the launch allows it (variants 0-2: a single
 *                       field without the mirror term, 16-byte aligned rows), or read directly
 *                       (variants 3-5, and every other launch); same frames for the same CTA size
 *   SB_TUNE_MODALREC_BATCHED  sb_modalrec_batched; key sb_tune_key(n_modes, n_slopes, n_batch);
 *                       reconstructor rows per CTA (2, 1, 4)
 * ------------------------------------------------------------------------ */
#define SB_TUNE_DM_BATCHED 0
#define SB_TUNE_SH_FP32 1
#define SB_TUNE_MODALREC_BATCHED 2
int sb_tune_variants(int family);                         /* 0 for an unknown family */
const char *sb_tune_variant_name(int family, int variant);
unsigned long long sb_tune_key(int a, int b, int c);
int sb_tune_set(int family, unsigned long long key, int variant);   /* variant < 0: remove */
int sb_tune_get(int family, unsigned long long key);               /* -1 for an unknown family */

/* Diagnostics: SB_OK, or SB_ETIMEOUT when a bounded wait inside a kernel
 * (the shared-memory pipeline of sb_dm_project, the tensor-core waits of
 * sb_sh_forward_split_bf16) gave up since the last call;
 * reading clears it.  Synchronous (waits for the device); not for the step. */
int sb_device_status(void);

/* ------------------------------------------------------------------------
 * Adjoint of the noise-free SH -> ShSlopec chain, and the interaction
 * matrix built from it.  No counterpart in the reference, which measures
 * the interaction matrix by push-pull (im_rec_calibrator.py:42-71 with
 * lib/modal_pushpull_signal.py:35-65: 2 x n_modes forward loop steps).
 *
 * A linear detector (no noise) leaves the CoG slopes of a sub-aperture a
 * function of that sub-aperture's phase samples only; the photon
 * normalisation (sh.py:426-427) cancels in the CoG (sh_slopec.py:392-404).
 * So d(slopes)/d(phase) is a 2 x np_sub^2 block per valid sub-aperture.
 *   lenslet[s]  lenslet index (row * n_lenses + column) of valid
 *               sub-aperture s, in slope order
 *   xw/yw/mw    the ShSlopec weights (subap_npx^2 each)
 *   active[s]   nonzero where the reference keeps the sub-aperture
 *               (1/flux <= 1/(1e-3 * mean flux), sh_slopec.py:400) at the
 *               linearisation point; zero rows stay zero.  NULL: every
 *               sub-aperture with flux (then apply the cut-off from
 *               tot_out, as sb_intmat_contract does)
 * Threshold 0 only (the thresholded CoG is not differentiable).
 * Geometries (np_sub, cutsize, subap_npx): (8, 12, 6), (8, 14, 8),
 * (8, 16, 8), (8, 8, 8) and (16, 16, 8), the 2x-resampled 8-pixel lenslets
 * of fov_ovs != 1 geometries (A and phase_nm are then the SH's resampled
 * field; the host carries the resampling's transpose).
 * ---------------------------------------------------------------------- */

/* jac[axis][s][r * np_sub + c] = d slope(axis, s) / d phase_nm at pixel
 * (r, c) of sub-aperture s; axis 0 = x, 1 = y.  tot_out (optional,
 * n_valid): each sub-aperture's CoG denominator, sum_px D * mw, at the
 * linearisation point (unnormalised: only ratios are meaningful). */
int sb_sh_slopes_jacobian(const sb_sh_plan *plan, const float *A, const float *phase_nm, int n_valid,
                          const int32_t *lenslet, const float *xw, const float *yw, const float *mw,
                          const float *active, float *jac, float *tot_out, void *stream);

/* Vector-Jacobian product: grad_phase[pixel] = sum_j seed[j] d slope_j /
 * d phase_nm[pixel], seed laid out like the slopes ([sx..., sy...]).
 * Writes the pixels of the valid sub-apertures only (grad_phase has the
 * field's row stride plan->field_ld; clear it first). */
int sb_sh_slopes_vjp(const sb_sh_plan *plan, const float *A, const float *phase_nm, int n_valid,
                     const int32_t *lenslet, const float *xw, const float *yw, const float *mw,
                     const float *active, const float *seed, float *grad_phase, void *stream);

/* intmat[m][j] = scale * sum_px jac[j][px] * ifunc[m][pix2col[px]] over the
 * pixels of slope j's sub-aperture.  slot[i * n_lenses + j]: valid
 * sub-aperture index of lenslet (i, j) or -1; pix2col: field pixel ->
 * influence-function column, -1 outside the mirror's mask (field row
 * stride field_ld).  tot (optional): the sb_sh_slopes_jacobian flux; when
 * given, sub-apertures below the CoG cut-off get zero columns.  intmat is
 * n_modes x (2 n_valid), row-major.  With scale = 2 * sign this is the
 * reference's push-pull matrix (s+ - s-)/a in the limit of small a (DM
 * phase = sign * cmd @ IF, dm.py:72-86).  np_sub in {4, 8, 16};
 * n_lenses * np_sub <= 1024 (512 for np_sub = 16). */
int sb_intmat_contract(const float *jac, const float *tot, int n_valid, int np_sub, int n_lenses, int field_ld,
                       const int32_t *slot, const int32_t *pix2col, const float *ifunc, int n_modes,
                       int ld_if, float scale, float *intmat, void *stream);

/* sb_intmat_contract with the influence functions streamed by TMA (the same
 * contraction as im_rec_calibrator.py:58-63 in its small-amplitude limit; the
 * same matrix bit for bit).  The mirror's columns enumerate its pixels
 * row-major, so the np_sub field rows of lenslet row li lie in one column
 * range: row_seg[2*li] = first column, row_seg[2*li+1] = number of columns
 * (both multiples of 32, covering every column under a valid sub-aperture of
 * that row; 0 columns for a row without any), seg_max = the largest count
 * (<= 7168).  A work unit (lenslet row, 4 modes) is one stage of a
 * shared-memory ring (about 100 KB per CTA), loaded as 256-column x 4-mode
 * 2-D TMA boxes.  Needs ld_if a
 * multiple of 32, a 16-byte aligned ifunc, np_sub 4 or 8 and at most 992
 * field columns; a segment that is misaligned or misses a column is skipped
 * and reported by sb_device_status (SB_EINVAL), as are timed-out waits
 * (SB_ETIMEOUT). */
int sb_intmat_contract_rows(const float *jac, const float *tot, int n_valid, int np_sub, int n_lenses,
                            int field_ld, const int32_t *slot, const int32_t *pix2col, const int32_t *row_seg,
                            int seg_max, const float *ifunc, int n_modes, int ld_if, float scale, float *intmat,
                            void *stream);

/* The same contraction (im_rec_calibrator.py:58-63 in its small-amplitude
 * limit) in two steps, for a mirror whose interaction matrix is computed
 * more than once (at several operating points, or each calibration).
 * sb_intmat_lenslet_ifunc copies, once per mirror and column map, the
 * influence-function samples under the valid sub-apertures into a
 * lenslet-major array: ifl[m][s][c][r] = ifunc[m * ld_if + col] with col =
 * pix2col[(li * np_sub + r) * field_ld + lj * np_sub + c], 0 where col < 0,
 * lenslet[s] = li * n_lenses + lj the lenslet of valid sub-aperture s
 * (n_modes * n_valid * np_sub^2 floats, 16-byte aligned).
 * sb_intmat_contract_lenslets then reads that array once per matrix (one
 * contiguous np_sub^2 run per mode and sub-aperture) with jac, tot and
 * scale as in sb_intmat_contract, and writes the same matrix bit for bit
 * (the same products, summed in the same order).  The mean flux of the CoG
 * cut-off is summed over another thread grouping, so a sub-aperture whose
 * flux lies within a rounding of the cut-off could be decided the other
 * way.  np_sub 4 or 8. */
int sb_intmat_lenslet_ifunc(const float *ifunc, int n_modes, int ld_if, const int32_t *lenslet, int n_valid,
                            int np_sub, int n_lenses, int field_ld, const int32_t *pix2col, float *ifl,
                            void *stream);
int sb_intmat_contract_lenslets(const float *jac, const float *tot, int n_valid, int np_sub, const float *ifl,
                                int n_modes, float scale, float *intmat, void *stream);

/* ------------------------------------------------------------------------
 * AtmoEvolution — replaces specula/processing_objects/atmo_evolution.py:
 * 286-294: per layer, (1-f)*P[:, q:q+L] + f*P[:, q+1:q+1+L], rot90 by k,
 * order-1 rotation by the fractional part of the wind direction in degrees
 * (scipy.ndimage.rotate(reshape=False, order=1, mode='constant')), times
 * the r0 scale.  One launch updates every layer.
 * ---------------------------------------------------------------------- */
#define SB_MAX_LAYERS 16
typedef struct sb_atmo_layer {
    const float *screen;    /* strip, rows = L, row stride screen_ld          */
    int screen_ld;
    int screen_cols;        /* strip width: positions cycle to 0 beyond it    */
    double delta;           /* wind_speed * delta_time / pixel_pitch (float64) */
    int rot90;              /* k in 0..3                                      */
    int rotate;             /* nonzero: apply the fractional-degree rotation  */
    double m00, m01, m10, m11, off0, off1;  /* scipy affine map (output->input) */
    float scale;            /* (pitch / r0_lambda)^(5/6)                      */
    float *out;             /* L x L, row-major                               */
} sb_atmo_layer;

/* positions: device float64[n_layers], the layers' last positions (pixels);
 * the call advances them by `delta` (cycling to 0 when pos + L reaches the
 * strip width, atmo_evolution.py:269-279) and then writes every layer. */
int sb_atmo_evolve(const sb_atmo_layer *layers, int n_layers, int L, double *positions,
                   void *stream);

/* Device-resident per-step inputs of AtmoEvolution (the seeing and wind
 * FuncGenerator outputs) and the constants of atmo_evolution.py:262-294. */
typedef struct sb_atmo_inputs {
    const double *seeing;          /* device, 1 value [arcsec]                          */
    const double *wind_speed;      /* device, n_wind_speed values [m/s] (1: all layers)  */
    const double *wind_direction;  /* device, n_wind_direction values [deg]              */
    int n_wind_speed;
    int n_wind_direction;
    double delta_time;             /* [s] since the previous step                        */
    double pixel_pitch;            /* [m]                                                */
    float pixel_pitch_f;           /* the pitch rounded to float32 (r0-scale arithmetic) */
    float airmass_pow;             /* float32(airmass) ** (-3/5), as NumPy computes it   */
    float lambda_factor;           /* float32((wavelength_nm / 500) ** (6/5))            */
} sb_atmo_inputs;

size_t sb_atmo_work_bytes(int n_layers);

/* sb_atmo_evolve with each layer's shift, rot90, fractional rotation and r0
 * scale computed on the device from device-resident inputs (the delta,
 * rot90, rotate, m.., off.. and scale fields of layers[] are not read), so
 * a captured CUDA graph of this call follows new seeing / wind values.
 * work: device scratch of sb_atmo_work_bytes(n_layers) bytes. */
int sb_atmo_evolve_inputs(const sb_atmo_layer *layers, int n_layers, int L, double *positions,
                          const sb_atmo_inputs *in, void *work, size_t work_bytes, void *stream);

/* Batched form: many layers (of many realisations) in one launch (chunks of
 * 64), each with its own device pointers to its seeing value, wind speed,
 * wind direction and position; the constants (delta_time, pitch, airmass,
 * wavelength factor) are shared and constants' pointers are not read.
 * work: n_layers * sb_atmo_work_bytes(1) bytes or more. */
typedef struct sb_atmo_layer_inputs {
    const double *seeing;
    const double *wind_speed;
    const double *wind_direction;
    double *position;
} sb_atmo_layer_inputs;

int sb_atmo_evolve_batched(const sb_atmo_layer *layers, const sb_atmo_layer_inputs *inputs, int n_layers, int L,
                           const sb_atmo_inputs *constants, void *work, size_t work_bytes, void *stream);

/* ------------------------------------------------------------------------
 * AtmoPropagation, on-axis branch — replaces
 * specula/processing_objects/atmo_propagation.py:105-125 with
 * electric_field.py:35-43,77-82: reset, then A *= layer.A[crop],
 * phase += layer.phase[crop] for each layer in order.
 * ---------------------------------------------------------------------- */
typedef struct sb_prop_layer {
    const float *A;         /* NULL: all ones                                 */
    const float *phase;     /* NULL: all zeros                                */
    int ld;
    int top, left;          /* crop offsets                                   */
} sb_prop_layer;

int sb_propagate_on_axis(const sb_prop_layer *layers, int n_layers, int pupil,
                         float *A_out, float *phase_out, void *stream);

/* General propagation (atmo_propagation.py:104-209 with lib/interp2d.py):
 * like sb_propagate_on_axis, but a layer with yy / xx set is resampled at
 * those per-output-pixel coordinates (row, column; clamped by the caller)
 * by bilinear interpolation in float64 on its rows x cols grid, as the
 * reference's Interp2D (off-axis sources, LGS cone effect, shifted, rotated
 * or magnified layers); the interpolated values are rounded to float32
 * before A *= ..., phase += ... */
typedef struct sb_prop_sampling {
    const float *A;         /* NULL: all ones                                 */
    const float *phase;     /* NULL: all zeros                                */
    int ld;
    int rows, cols;         /* layer size                                     */
    int top, left;          /* crop offsets (yy == NULL)                      */
    const float *yy, *xx;   /* pupil x pupil sample coordinates, or NULL      */
} sb_prop_sampling;
int sb_propagate(const sb_prop_sampling *layers, int n_layers, int pupil, float *A_out, float *phase_out,
                 void *stream);

/* Batched propagation of realisations sharing the layer structure of the
 * SCAO chain: n_atm unit-amplitude turbulence layers (realisation b's layer k
 * at atm + b*atm_real_stride + k*atm_layer_stride), the pupil stop (stop_A,
 * stop_phase, shared; either may be NULL) and the mirror (dm_A shared or
 * NULL, phase at dm_phase + b*dm_stride); all pupil x pupil, no crop.
 * Outputs at A_out / phase_out + b*out_stride.  Same operation order as
 * sb_propagate_on_axis over [turbulence..., stop, mirror]. */
int sb_propagate_batched(const float *atm, int n_atm, long long atm_layer_stride, long long atm_real_stride,
                         const float *stop_A, const float *stop_phase, const float *dm_A, const float *dm_phase,
                         long long dm_stride, int n_batch, int pupil, float *A_out, float *phase_out,
                         long long out_stride, void *stream);

/* sb_atmo_evolve_batched followed by sb_propagate_batched in one launch
 * (replaces atmo_evolution.py:258-300 then atmo_propagation.py:105-144 for
 * realisations whose n_atm layers are pupil-sized): layers / inputs hold
 * n_atm * n_batch entries, realisation b's layer k at index b * n_atm + k;
 * every layer is still written to its `out`, its values summed in layer
 * order and the field formed as sb_propagate_batched does, with the same
 * bits as the two calls.  n_batch = 1 serves a single system (the pipelined
 * SCAO step graph calls it so).  dm_phase NULL: no mirror term (dm_A is not
 * read); the outputs then hold the product and sum of the turbulence and the
 * stop, for a consumer that applies the mirror itself (sb_sh_ccd_slopec),
 * so the turbulence of a step need not wait for the previous mirror;
 * at most 16 layers per realisation. */
int sb_atmo_propagate_batched(const sb_atmo_layer *layers, const sb_atmo_layer_inputs *inputs, int n_atm, int n_batch,
                              int L, const sb_atmo_inputs *constants, void *work, size_t work_bytes,
                              const float *stop_A, const float *stop_phase, const float *dm_A, const float *dm_phase,
                              long long dm_stride, float *A_out, float *phase_out, long long out_stride,
                              void *stream);

/* ------------------------------------------------------------------------
 * PSF — replaces specula/processing_objects/psf.py:56-137 (PSF.calc_psf,
 * the Strehl ratio of trigger_code and the integration of post_trigger).
 * scratch: sb_psf_scratch_bytes() bytes, zero-filled before the first call
 * (the Strehl reduction keeps a completion counter there and resets it).
 * ---------------------------------------------------------------------- */
size_t sb_psf_scratch_bytes(void);

/* sr = |sum A e^{i phi}|^2 / (sum A)^2 with phi = phase_nm * phase_to_rad,
 * which equals the reference's centre pixel of the normalised, fftshift-ed
 * PSF over the flat-phase reference (Parseval); float64 accumulation.
 * integrate != 0: int_sr[0] += sr, int_sr[1] += 1 (device float64 pair). */
int sb_strehl(const float *A, const float *phase_nm, int n_pixels, float phase_to_rad, float *sr,
              double *int_sr, int integrate, void *scratch, size_t scratch_bytes, void *stream);

/* field[e] = A[e] * exp(i * phase_nm[e] * phase_to_rad) as complex64
 * (interleaved re, im): the input of the PSF's two DFT products. */
int sb_psf_field(const float *A, const float *phase_nm, int n_pixels, float phase_to_rad, void *field,
                 void *stream);

/* psf = |F|^2 / sum |F|^2 from the focal-plane field F (complex64), and,
 * when int_psf is not NULL, int_psf += psf. */
int sb_psf_finish(const void *focal_field, long long n_pixels, float *psf, float *int_psf, void *scratch,
                  size_t scratch_bytes, void *stream);

/* The PSF image on the tensor cores (replaces psf.py:56-96: the zero-padded
 * field's |fftshift(fft2)|^2 normalised to unit sum, for an m x m field and
 * the padded size n = round(m nd / 2) * 2).  F = W u W^T with the n x m DFT
 * matrix W (rows in fftshift order) as two real GEMMs on tcgen05 with
 * split-BF16 operands (hi*hi + lo*hi + hi*lo, FP32 accumulation in tensor
 * memory); the normalisation uses Parseval's total n^2 sum |u|^2.
 *   sb_psf_tc_prepare  builds the DFT operand once (dft: sb_psf_tc_dft_bytes,
 *                      256-byte aligned)
 *   sb_psf_tc          one PSF: psf (n x n float32), int_psf += psf when not
 *                      NULL; scratch: sb_psf_tc_scratch_bytes, 256-byte
 *                      aligned, zero-filled before the first call
 * Three launches (field, W u^T, W G); bounded waits, reported by
 * sb_device_status. */
size_t sb_psf_tc_dft_bytes(int m, int n);
int sb_psf_tc_prepare(int m, int n, void *dft, size_t dft_bytes, void *stream);
size_t sb_psf_tc_scratch_bytes(int m, int n);
int sb_psf_tc(const float *A, const float *phase_nm, int m, int n, float phase_to_rad, const void *dft, float *psf,
              float *int_psf, void *scratch, size_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Monte-Carlo step over geometry groups — the loop step of many independent
 * SCAO realisations of uneven pupil / sub-aperture counts (the reference
 * steps each through its own LoopControl.iter, loop_control.py:83-123).
 * A group is realisations that share the pupil, sub-aperture grid,
 * wavelength, reconstructor and mirror, with their own atmospheres and
 * detector seeds; each stage of the step is ONE launch over every
 * realisation of every group:
 *   1 layer positions + per-step parameters    (atmo_evolution.py:258-277)
 *   2 every turbulence layer and the on-axis field
 *                                                (atmo_evolution.py:278-294,
 *                                                 atmo_propagation.py:105-144)
 *   3 SH forward, unnormalised + partial sums    (sh.py:348-420)
 *   4 photon normalisation, CCD, CoG slopes, flux cut-off, detector state
 *                                                (sh.py:422-428, ccd.py:198-287,
 *                                                 sh_slopec.py:308-438)
 *   5 reconstructor rows + integrators           (modalrec.py:114-162,
 *                                                 iir_filter.py:100-211)
 *   6 mirror projection                          (dm.py:72-86)
 * (stage 2 is two launches when a group has more than 16 layers)
 * Each stage computes what the group-by-group batched calls compute
 * (sb_atmo_evolve_batched, sb_propagate_batched, sb_sh_forward[_split_bf16]_batched,
 * sb_ccd_step_batched, sb_slopec_batched, sb_modalrec_batched,
 * sb_integrator, sb_dm_project_batched with one mode-row group), bit for bit.
 * Per group: SH geometries with a compile-time kernel, every frame read out
 * each step (frames_per_read 1, no binning, no charge-transfer matrices),
 * the slope computer with thr_value only, sub-aperture boxes listed
 * row-major (lenslet_subap maps lenslet i*n+j to its valid sub-aperture or
 * -1), at most 1024 modes.  The frames of a group are rows of stacks:
 * intensity, integrated and pixels share frame_stride; the turbulence
 * layers' outputs (layers[].out) are rows of atm.
 *   sb_mc_workspace_bytes  device workspace for the groups (256-byte aligned,
 *                          zero-filled before sb_mc_create)
 *   sb_mc_create           validates the groups, copies their tables into the
 *                          workspace (on stream) and returns a host handle;
 *                          the host arrays may be freed afterwards
 *   sb_mc_step             one step: SB_MC_LAUNCHES launches on stream, no
 *                          allocation, no synchronisation (graph-capturable)
 *   sb_mc_destroy          frees the handle
 * ---------------------------------------------------------------------- */
#define SB_MC_MAX_GROUPS 8
#define SB_MC_LAUNCHES 6

typedef struct sb_mc_group {
    int n_batch;                        /* realisations                                */
    /* atmosphere: n_batch * n_atm layers, realisation-major (host arrays) */
    int n_atm;
    int L;                              /* pupil side [px]                             */
    const sb_atmo_layer *layers;
    const sb_atmo_layer_inputs *inputs;
    sb_atmo_inputs constants;           /* its pointers are not read                   */
    /* propagation: layer k of realisation b is atm + b*atm_real_stride + k*L*L */
    const float *atm;
    long long atm_real_stride;
    const float *stop_A, *stop_phase;   /* pupil stop (shared; NULL: none)             */
    const float *dm_A;                  /* mirror amplitude (shared; NULL: none)       */
    float *dm_phase;                    /* per-realisation mirror phase, stride dm_stride */
    long long dm_stride;
    float *field_A, *field_phase;       /* per-realisation field, stride field_stride   */
    long long field_stride;
    /* SH: dft_mode 0 FP32, 1 split-BF16 */
    sb_sh_plan sh;
    int dft_mode;
    float photon_scale;
    /* detector and slopes */
    float *intensity, *integrated, *pixels;
    long long frame_stride;
    sb_ccd_params ccd;                  /* shared parameters and frame state (one per group) */
    const uint64_t *photon_seeds;       /* device [n_batch]                            */
    const uint64_t *readout_seeds;      /* device [n_batch]                            */
    sb_slopec_plan slopec;
    const int32_t *lenslet_subap;       /* device [n_lenses^2]                         */
    float *slopes;                      /* [n_batch][slopes_stride]                    */
    int slopes_stride;
    float *flux;                        /* [n_batch][flux_stride]                      */
    int flux_stride;
    /* reconstructor and integrators */
    const float *R;
    int n_modes, n_slopes, ldr;
    float *modes;                       /* [n_batch][n_modes]                          */
    sb_iir_plan iir;                    /* n = n_batch * n_modes, element b*n_modes+m  */
    float *commands;                    /* [n_batch][n_modes]: the integrators' output */
    /* mirror: phase[b][mask_idx[p]] = dm_sign * sum_m commands[b][m] IF[m][p] */
    const float *ifunc;                 /* 16-byte aligned rows                        */
    int n_valid, ld_if;
    const int32_t *mask_idx;
    float dm_sign;
    /* pipelined stages (NULL: sb_mc_stage takes parity -1 only): a second
     * mirror-phase buffer (stride dm_stride) and the integrators' next
     * output, which iir.out_next must point to */
    float *dm_phase_alt;
    float *commands_next;
} sb_mc_group;

typedef struct sb_mc_handle sb_mc_handle;

size_t sb_mc_workspace_bytes(const sb_mc_group *groups, int n_groups);
int sb_mc_create(const sb_mc_group *groups, int n_groups, void *workspace, size_t workspace_bytes,
                 sb_mc_handle **handle, void *stream);
int sb_mc_step(const sb_mc_handle *handle, void *stream);
void sb_mc_destroy(sb_mc_handle *handle);

/* One stage of the step on a stream of the caller's choice, so that the
 * mirror projection of step t can overlap the other stages of step t (the
 * integrators' output for step t is known after step t-1, for integer
 * delays >= 1).  parity -1: the stages of sb_mc_step (the field takes
 * dm_phase, the mirror writes it from commands).  parity p = t % 2, with
 * dm_phase_alt and commands_next set: SB_MC_ATMO's field takes buffer p ^ 1
 * and SB_MC_DM writes buffer p (0: dm_phase, 1: dm_phase_alt) from
 * commands_next.  Step t then runs, with DM(t) on a second stream:
 *   second stream: wait for REC(t-1); DM(t)
 *   first stream:  ATMO, SH, CHAIN; wait for DM(t); REC
 * after one sb_mc_step (which fills commands_next and dm_phase) as step
 * t = 0, i.e. parities 1, 0, 1, ...  The results equal sb_mc_step's. */
#define SB_MC_ATMO 0    /* stages 1-2 (two launches) */
#define SB_MC_SH 1
#define SB_MC_CHAIN 2
#define SB_MC_REC 3
#define SB_MC_DM 4
int sb_mc_stage(const sb_mc_handle *handle, int stage, int parity, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SPECULA_B200_H */
