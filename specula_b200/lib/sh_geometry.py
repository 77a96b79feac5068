"""Host-side SH geometry solve and the device tables derived from it.

The integer geometry (sub-aperture sampling, FFT size, FoV oversampling,
cut) follows specula/processing_objects/sh.py:112-237 (set_in_ef) and
:239-282 (calc_trigger_geometry) operation for operation, including the
float round trips through radians, because Python ``round`` decisions depend
on them.  One deliberate difference: ``cutpixels == 0`` (detector FoV equal
to the FFT FoV) is treated as "no cut"; the reference slices ``[0:-0]`` there
and fails.

The device tables replace the reference's per-row FFT/fftshift/cut/toccd
sequence (sh.py:364-420, toccd.py:33-63) by an equivalent pruned DFT:
  * twiddle[b][c] = exp(-2*pi*i * k_b * c / fft) for the cut window's
    frequencies k_b = (cut//2 + b - fft//2) mod fft (fftshift) and the np_sub
    non-zero input samples c;
  * fp_mask restricted to the cut window;
  * rebin[p][a] = |[p*dxo, (p+1)*dxo) ∩ a-th input cell| / dxo, the LCM area
    rebin per sub-aperture (the mosaic of toccd never mixes sub-apertures
    because lcm(n*cs, n*npx) = n*lcm(cs, npx)).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from specula_b200 import RAD2ASEC
from specula_b200.lib.make_mask import make_mask


@dataclass
class SHGeometry:
    n_lenses: int
    np_sub: int
    ovs_np_sub: int
    fov_ovs: float
    scale_ovs: int
    fft_size: int
    cutpixels: int
    cutsize: int
    subap_npx: int
    sensor_pxscale: float           # radians, updated by set_in_ef
    fov_complete: float             # radians
    fp_diaratio: float
    squaremask: bool
    xy_shift: tuple
    rot_angle: float
    do_interpolation: bool
    wf1_pixel_pitch: float
    extra: dict = field(default_factory=dict)

    @property
    def ccd_side(self):
        return self.subap_npx * self.n_lenses


def solve(wavelengthInNm, subap_wanted_fov, sensor_pxscale, subap_on_diameter, subap_npx, ef_size,
          pixel_pitch, FoVres30mas=False, squaremask=True, fov_ovs_coeff=0, xShiftPhInPixel=0,
          yShiftPhInPixel=0, aXShiftPhInPixel=0, aYShiftPhInPixel=0, rotAnglePhInDeg=0,
          aRotAnglePhInDeg=0, do_not_double_fov_ovs=False, set_fov_res_to_turbpxsc=False):
    """Geometry of an SH with the reference constructor's arguments (angles in
    arcsec) looking at a square field of ``ef_size`` pixels of ``pixel_pitch`` m."""
    n = int(subap_on_diameter)
    lens_size = 2.0 / n
    wanted_rad = subap_wanted_fov / RAD2ASEC
    pxs_rad = sensor_pxscale / RAD2ASEC
    fov_res = 0.03 if FoVres30mas else 0
    coeff = fov_ovs_coeff

    # ---- set_in_ef (sh.py:112-237) ----
    np_sub_int = max([1, round((ef_size * lens_size) / 2.0)])
    if np_sub_int * n > ef_size:
        np_sub_int -= 1
    np_sub_f = (ef_size * lens_size) / 2.0
    pxs_arcsec = pxs_rad * RAD2ASEC
    turb = wavelengthInNm * 1e-9 / (np_sub_f * pixel_pitch) * RAD2ASEC
    wanted_arcsec = wanted_rad * RAD2ASEC
    real_arcsec = pxs_rad * subap_npx * RAD2ASEC

    if fov_res == 0:
        if set_fov_res_to_turbpxsc:
            if turb >= pxs_arcsec:
                raise ValueError('set_fov_res_to_turbpxsc property should be set to one only if '
                                 'turb. pix. sc. is < sensor pix. sc.')
            fov_res = turb
        elif turb < pxs_arcsec and pxs_arcsec / 2.0 > 0.5:
            fov_res = turb * 0.5
        else:
            i = 0
            while turb / (i + 2) >= pxs_arcsec:
                i += 1
            cand = np.arange(10)
            res_try = np.array([turb / (i + k + 2) for k in cand])
            scale_try = np.array([round(turb / r) for r in res_try], dtype=float)
            fft_scale = np.array([wavelengthInNm / 1e9 * n / (ef_size * pixel_pitch * s) * RAD2ASEC
                                  for s in scale_try])
            real_try = np.array([round(wanted_arcsec / fs / 2.0) * 2 for fs in fft_scale], dtype=float)
            mcm_try = np.array([np.lcm(int(subap_npx), int(r)) for r in real_try], dtype=float)
            err = np.abs(real_try * fft_scale - wanted_arcsec) / wanted_arcsec
            good = np.where(err < 0.02)[0]
            if len(good) == 0:
                good = np.arange(10)
            best = np.argmin(mcm_try[good] / scale_try[good])
            if good[best] != 0 and mcm_try[good[0]] / mcm_try[good[best]] > scale_try[good[best]] / scale_try[good[0]]:
                fov_res = res_try[good[best]]
            else:
                fov_res = res_try[good[0]]

    scale_ovs = round(turb / fov_res)
    fft_px_arcsec = wavelengthInNm * 1e-9 / (ef_size * pixel_pitch * scale_ovs / n) * RAD2ASEC
    real_pix = round(real_arcsec / fft_px_arcsec / 2.0) * 2.0
    real_arcsec = real_pix * fft_px_arcsec
    turb_fov_pix = int(scale_ovs * np_sub_f)

    if turb_fov_pix > 2 * real_pix:
        fov_ovs = coeff if coeff != 0.0 else 1
    else:
        ratio = float(real_pix) / float(turb_fov_pix)
        np_factor = 1 if abs(np_sub_f - int(np_sub_f)) < 1e-3 else int(np_sub_f)
        if do_not_double_fov_ovs and coeff == 0.0:
            fov_ovs = np.ceil(np_factor * ratio / 2.0) * 2.0 / float(np_factor)
        else:
            if coeff == 0.0:
                coeff = 2.0
            if ratio < 2:
                fov_ovs = np.ceil(np_factor * coeff) / float(np_factor)
            else:
                fov_ovs = np.ceil(np_factor * ratio * coeff) / float(np_factor)

    pxs_rad = real_arcsec / subap_npx / RAD2ASEC
    ovs_np_sub = int(ef_size * fov_ovs * lens_size * 0.5)
    fft_size = ovs_np_sub * scale_ovs
    chk = (ef_size * round(fov_ovs) * lens_size) / 2.0
    if abs(chk - round(chk)) > 1e-4:
        raise ValueError(f'ERROR: interpolated input phase size {ef_size} * {round(fov_ovs)} is not divisible '
                         f'by {n} subapertures.')

    # ---- calc_trigger_geometry (sh.py:239-282) ----
    rot = rotAnglePhInDeg + aRotAnglePhInDeg
    shift = np.round(np.array([xShiftPhInPixel + aXShiftPhInPixel,
                               yShiftPhInPixel + aYShiftPhInPixel]) * fov_ovs).astype(int)
    do_interp = bool(fov_ovs != 1 or rot != 0 or np.sum(np.abs(shift)) != 0)
    wf1_pitch = pixel_pitch / fov_ovs if do_interp else pixel_pitch
    fp4_pitch = wavelengthInNm / 1e9 / (wf1_pitch * fft_size)
    fov_complete = fft_size * fp4_pitch
    cutpixels = int(np.round((fov_complete - pxs_rad * subap_npx) / fp4_pitch) / 2 * 2)
    if cutpixels < 0:
        raise ValueError(f'detector FoV ({subap_npx} px) is wider than the FFT FoV ({fft_size} samples)')
    return SHGeometry(n_lenses=n, np_sub=int(np_sub_int), ovs_np_sub=int(ovs_np_sub), fov_ovs=fov_ovs,
                      scale_ovs=int(scale_ovs), fft_size=int(fft_size), cutpixels=cutpixels,
                      cutsize=int(fft_size - cutpixels), subap_npx=int(subap_npx), sensor_pxscale=pxs_rad,
                      fov_complete=fov_complete, fp_diaratio=wanted_rad / fov_complete,
                      squaremask=squaremask, xy_shift=(int(shift[0]), int(shift[1])), rot_angle=rot,
                      do_interpolation=do_interp, wf1_pixel_pitch=wf1_pitch)


def tilt_table(p, fft_size):
    """Half-pixel tilt exp(-2*pi*i*(x+y)/(2*fft)) on the p x p sub-aperture
    grid, x, y in [-p//2, p//2) (sh.py:469-477), as complex64."""
    a = np.arange(-p // 2, p // 2)
    g = a[None, :] + a[:, None]
    return np.exp(-2j * np.pi * g / (2 * fft_size)).astype(np.complex64)


def cut_frequencies(fft_size, cutpixels):
    """Unshifted FFT bins of the cut window after fftshift (sh.py:396,405)."""
    cs = fft_size - cutpixels
    lo = cutpixels // 2
    return (lo + np.arange(cs) - fft_size // 2) % fft_size


def twiddle_table(p, fft_size, cutpixels):
    """W[b][c] = exp(-2*pi*i*k_b*c/fft), float64 phases rounded once to complex64."""
    k = cut_frequencies(fft_size, cutpixels)
    c = np.arange(p)
    ph = (np.outer(k, c) % fft_size) * (-2.0 * np.pi / fft_size)
    return np.exp(1j * ph).astype(np.complex64)


def field_stop_cut(g: SHGeometry):
    """Field-stop mask (sh.py:282) restricted to the cut window, float32."""
    m = make_mask(g.fft_size, diaratio=g.fp_diaratio, square=g.squaremask).astype(np.float32)
    lo = g.cutpixels // 2
    return np.ascontiguousarray(m[lo:lo + g.cutsize, lo:lo + g.cutsize])


def rebin_table(cutsize, npx):
    """R[p][a]: overlap of output pixel p with input cell a on the LCM grid,
    divided by the output width (toccd.py:55-61 per sub-aperture)."""
    L = math.lcm(cutsize, npx)
    dxi, dxo = L // cutsize, L // npx
    R = np.zeros((npx, cutsize), dtype=np.float64)
    for m in range(L):
        R[m // dxo, m // dxi] += 1.0
    return (R / dxo).astype(np.float32)
