"""Oracle: Shack-Hartmann sensor forward model (test infrastructure only).

Restates specula/processing_objects/sh.py (geometry solve :112-323, trigger
:348-420, photon normalisation :422-428, tilt :469-477), specula/lib/toccd.py
(CPU branch :33-63 with specula/lib/rebin.py), specula/lib/interp2d.py
(:48-122, CPU branch) and specula/lib/extrapolate_edge_pixel*.py; the
laser-guide-star branch (sh.py:289-321 and :382-394) with the kernel maps
of specula/data_objects/convolution_kernel.py:14-131 (lgs_map_sh) and
:260-276 (process_kernels).

Everything is vectorised over all sub-apertures at once; per-sub-aperture
arithmetic follows the reference's dtype rules at ``precision=1`` (float32 /
complex64) or ``precision=0`` (float64 / complex128).
"""
import math
from dataclasses import dataclass

import numpy as np

from .masks import RAD2ASEC, make_mask


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
    ccd_side: int
    xy_shift: tuple
    rot_angle: float
    do_interp: bool
    wf1_pitch: float
    fp_diaratio: float
    squaremask: bool
    sensor_pxscale_rad: float


def sh_geometry(wavelength_nm, subap_wanted_fov, sensor_pxscale, subap_on_diameter,
                subap_npx, ef_size, pixel_pitch, fov_ovs_coeff=0.0, FoVres30mas=False,
                squaremask=True, do_not_double_fov_ovs=False, set_fov_res_to_turbpxsc=False,
                xShiftPhInPixel=0, yShiftPhInPixel=0, aXShiftPhInPixel=0, aYShiftPhInPixel=0,
                rotAnglePhInDeg=0, aRotAnglePhInDeg=0):
    """Geometry integers and scalars of the SH (sh.py:112-237 set_in_ef and
    sh.py:239-282 calc_trigger_geometry).  The float round trips through
    radians are kept because ``round`` boundaries depend on them."""
    n = int(subap_on_diameter)
    lens_size = 2.0 / n                      # Lenslet(n).get(0,0)[2]
    sub_wanted_rad = subap_wanted_fov / RAD2ASEC
    sensor_rad = sensor_pxscale / RAD2ASEC
    fov_res = 0.03 if FoVres30mas else 0
    coeff = fov_ovs_coeff

    np_sub_int = max([1, round((ef_size * lens_size) / 2.0)])
    if np_sub_int * n > ef_size:
        np_sub_int -= 1
    np_sub = (ef_size * lens_size) / 2.0

    sensor_pxscale_arcsec = sensor_rad * RAD2ASEC
    d_sub = np_sub * pixel_pitch
    turb_px = wavelength_nm * 1e-9 / d_sub * RAD2ASEC
    wanted_arcsec = sub_wanted_rad * RAD2ASEC
    real_fov_arcsec = sensor_rad * subap_npx * RAD2ASEC

    if fov_res == 0:
        if set_fov_res_to_turbpxsc:
            if turb_px >= sensor_pxscale_arcsec:
                raise ValueError('set_fov_res_to_turbpxsc needs turbulence px scale < sensor px scale')
            fov_res = turb_px
        elif turb_px < sensor_pxscale_arcsec and sensor_pxscale_arcsec / 2.0 > 0.5:
            fov_res = turb_px * 0.5
        else:
            i = 0
            while turb_px / (i + 2) >= sensor_pxscale_arcsec:
                i += 1
            i_min = i
            ntry = 10
            res_try = np.zeros(ntry)
            scale_try = np.zeros(ntry)
            fft_scale_try = np.zeros(ntry)
            sub_real_try = np.zeros(ntry)
            mcm_try = np.zeros(ntry)
            for k in range(ntry):
                res_try[k] = turb_px / (i_min + k + 2)
                scale_try[k] = round(turb_px / res_try[k])
                fft_scale_try[k] = wavelength_nm / 1e9 * n / (ef_size * pixel_pitch * scale_try[k]) * RAD2ASEC
                sub_real_try[k] = round(wanted_arcsec / fft_scale_try[k] / 2.0) * 2
                mcm_try[k] = np.lcm(int(subap_npx), int(sub_real_try[k]))
            fov = sub_real_try * fft_scale_try
            err = np.abs(fov - wanted_arcsec) / wanted_arcsec
            good = np.where(err < 0.02)[0]
            if len(good) == 0:
                good = np.arange(ntry)
            ratio_mcm = mcm_try[good] / scale_try[good]
            imin = np.argmin(ratio_mcm)
            if good[imin] != 0 and mcm_try[good[0]] / mcm_try[good[imin]] > scale_try[good[imin]] / scale_try[good[0]]:
                fov_res = res_try[good[imin]]
            else:
                fov_res = res_try[good[0]]

    scale_ovs = round(turb_px / fov_res)
    d_sub_padded = ef_size * pixel_pitch * scale_ovs / n
    fft_px_arcsec = wavelength_nm * 1e-9 / d_sub_padded * RAD2ASEC
    real_fov_pix = round(real_fov_arcsec / fft_px_arcsec / 2.0) * 2.0
    real_fov_arcsec = real_fov_pix * fft_px_arcsec
    turb_fov_pix = int(scale_ovs * np_sub)

    if turb_fov_pix > 2 * real_fov_pix:
        fov_ovs = 1
        if coeff != 0.0:
            fov_ovs = coeff
    else:
        ratio = float(real_fov_pix) / float(turb_fov_pix)
        np_factor = 1 if abs(np_sub - int(np_sub)) < 1e-3 else int(np_sub)
        if do_not_double_fov_ovs and coeff == 0.0:
            coeff = 1.0
            fov_ovs = np.ceil(np_factor * ratio / 2.0) * 2.0 / float(np_factor)
        else:
            if coeff == 0.0:
                coeff = 2.0
            if ratio < 2:
                fov_ovs = np.ceil(np_factor * coeff) / float(np_factor)
            else:
                fov_ovs = np.ceil(np_factor * ratio * coeff) / float(np_factor)

    sensor_rad = real_fov_arcsec / subap_npx / RAD2ASEC
    ovs_np_sub = int(ef_size * fov_ovs * lens_size * 0.5)
    fft_size = ovs_np_sub * scale_ovs

    chk = (ef_size * round(fov_ovs) * lens_size) / 2.0
    if abs(chk - round(chk)) > 1e-4:
        raise ValueError('interpolated input phase size is not divisible by the number of subapertures')

    # calc_trigger_geometry (sh.py:239-282)
    rot = rotAnglePhInDeg + aRotAnglePhInDeg
    shift = np.round(np.array([xShiftPhInPixel + aXShiftPhInPixel,
                               yShiftPhInPixel + aYShiftPhInPixel]) * fov_ovs).astype(int)
    do_interp = fov_ovs != 1 or rot != 0 or np.sum(np.abs(shift)) != 0
    wf1_pitch = pixel_pitch / fov_ovs if do_interp else pixel_pitch
    fp4_pitch = wavelength_nm / 1e9 / (wf1_pitch * fft_size)
    fov_complete = fft_size * fp4_pitch
    fov_cut = fov_complete - sensor_rad * subap_npx
    cutpixels = int(np.round(fov_cut / fp4_pitch) / 2 * 2)
    if cutpixels < 0:
        raise ValueError('detector field of view is larger than the FFT field of view')
    cutsize = fft_size - cutpixels
    return SHGeometry(n_lenses=n, np_sub=int(np_sub_int), ovs_np_sub=ovs_np_sub, fov_ovs=fov_ovs,
                      scale_ovs=int(scale_ovs), fft_size=int(fft_size), cutpixels=cutpixels,
                      cutsize=int(cutsize), subap_npx=int(subap_npx), ccd_side=int(subap_npx) * n,
                      xy_shift=(int(shift[0]), int(shift[1])), rot_angle=rot, do_interp=bool(do_interp),
                      wf1_pitch=wf1_pitch, fp_diaratio=sub_wanted_rad / fov_complete,
                      squaremask=squaremask, sensor_pxscale_rad=sensor_rad)


def tilt_factor(p, c, cdtype=np.complex64):
    """Half-pixel tilt exp(-2*pi*i*(x+y)/(2*(p+c))) on a p x p grid (sh.py:469-477)."""
    a = np.arange(-p // 2, p // 2)
    xx, yy = np.meshgrid(a, a)
    return np.exp(-2 * np.pi * 1j * (xx + yy) / (2 * (p + c)), dtype=cdtype)


def _rebin_sample(a, shape):
    """IDL-style nearest-sample upsampling (rebin.py:14-19)."""
    sl = [slice(0, old, float(old) / new) for old, new in zip(a.shape, shape)]
    idx = np.mgrid[sl].astype(np.int32)
    return a[tuple(idx)]


def _rebin_mean(a, shape):
    """Integer-factor block average (rebin.py:21-27)."""
    M, N = a.shape
    m, n = shape
    return a.reshape((m, M // m, n, N // n)).mean(3).mean(1)


def toccd(a, newshape):
    """LCM area rebin, CPU branch (toccd.py:33-63)."""
    if a.shape == tuple(newshape):
        return a
    total = a.sum()
    mx = math.lcm(a.shape[0], newshape[0])
    my = math.lcm(a.shape[1], newshape[1])
    t = a if (mx, a.shape[1]) == a.shape else _rebin_sample(a, (mx, a.shape[1]))
    t = t if (newshape[0], a.shape[1]) == t.shape else _rebin_mean(t, (newshape[0], a.shape[1]))
    t = t if (newshape[0], my) == t.shape else _rebin_sample(t, (newshape[0], my))
    t = t if tuple(newshape) == t.shape else _rebin_mean(t, tuple(newshape))
    return t / t.sum() * total


def interp2d_coords(in_shape, out_shape, rot_deg=0.0, row_shift=0, col_shift=0, dtype=np.float32):
    """Sampling coordinates of Interp2D without explicit xx/yy (interp2d.py:48-93)."""
    yy, xx = map(dtype, np.mgrid[0:out_shape[0], 0:out_shape[1]])
    yy *= (in_shape[0] - 1) / out_shape[0]
    xx *= (in_shape[1] - 1) / out_shape[1]
    if rot_deg != 0:
        yc = in_shape[0] / 2 - 0.5
        xc = in_shape[1] / 2 - 0.5
        c = np.cos(rot_deg * 3.1415 / 180.0)
        s = np.sin(rot_deg * 3.1415 / 180.0)
        xr = (xx - xc) * c - (yy - yc) * s
        yr = (xx - xc) * s + (yy - yc) * c
        xx = xr + xc
        yy = yr + yc
    if row_shift != 0 or col_shift != 0:
        yy += row_shift
        xx += col_shift
    yy[yy < 0] = 0
    xx[xx < 0] = 0
    yy[yy > in_shape[0] - 1] = in_shape[0] - 1
    xx[xx > in_shape[1] - 1] = in_shape[1] - 1
    return np.array(yy, dtype=dtype).ravel(), np.array(xx, dtype=dtype).ravel()


def interp2d(value, yy, xx, out_shape, dtype=np.float32):
    """Bilinear sampling at (yy, xx), as RegularGridInterpolator(method='linear')
    on the integer grid (interp2d.py:117-122); coordinates are already clamped
    into the grid.  Computed in float64 like SciPy, then cast."""
    v = value.astype(np.float64)
    ny, nx = v.shape
    y = yy.astype(np.float64)
    x = xx.astype(np.float64)
    y0 = np.clip(np.floor(y).astype(np.int64), 0, ny - 2)
    x0 = np.clip(np.floor(x).astype(np.int64), 0, nx - 2)
    fy = y - y0
    fx = x - x0
    out = (v[y0, x0] * (1 - fy) * (1 - fx) + v[y0, x0 + 1] * (1 - fy) * fx +
           v[y0 + 1, x0] * fy * (1 - fx) + v[y0 + 1, x0 + 1] * fy * fx)
    return out.reshape(out_shape).astype(dtype)


def extrapol_tables(mask, do_ext_2_pix=True):
    """Edge-extrapolation index tables (extrapolate_edge_pixel_mat_define.py:5-143).
    Returns (s1, s2, idx_1pix, idx_2pix): flattened source indices for every
    pixel (-1 when none), the (row, col) arrays of extrapolated pixels and the
    positions within them that use the two-pixel linear rule."""
    shape = mask.shape
    fm = mask.astype(float)
    s1 = np.full(shape, -1.0)
    s2 = np.full(shape, -1.0)
    lin = np.zeros_like(fm)
    inside = np.where(mask)
    lin[inside] = np.ravel_multi_index(inside, shape)
    near1 = (np.roll(fm, 1, 0) + np.roll(fm, -1, 0) + np.roll(fm, 1, 1) + np.roll(fm, -1, 1)) * (1.0 - fm)
    near2 = (np.roll(fm, 2, 0) + np.roll(fm, -2, 0) + np.roll(fm, 2, 1) + np.roll(fm, -2, 1)) * (1.0 - fm)
    ring1 = np.where(near1 > 0)
    ring2 = np.where((near2 > 0) & (near1 == 0))

    def visit(r, c, d):
        # the four directions are tried in the order +col, -col, +row, -row;
        # `d` is the distance of the first in-pupil neighbour (1 or 2)
        test = -1
        for dr, dc in ((0, 1), (0, -1), (1, 0), (-1, 0)):
            ra, ca = r + dr * d, c + dc * d
            rb, cb = r + dr * (d + 1), c + dc * (d + 1)
            if dr == 0:
                lim_ok_a = (ca < shape[1] - 1) if dc > 0 else (ca > 0)
                lim_ok_b = (cb < shape[1] - 1) if dc > 0 else (cb > 0)
            else:
                lim_ok_a = (ra < shape[0] - 1) if dr > 0 else (ra > 0)
                lim_ok_b = (rb < shape[0] - 1) if dr > 0 else (rb > 0)
            own = s1 if d == 1 else s2
            if lim_ok_a and own[r, c] == -1 and fm[ra, ca] > 0:
                if lim_ok_b and fm[rb, cb] > 0:
                    s2[r, c] = lin[rb, cb]
                    s1[r, c] = lin[ra, ca]
                else:
                    test = lin[ra, ca]
        if s1[r, c] == -1 and test >= 0:
            s1[r, c] = test

    for r, c in zip(*ring1):
        visit(r, c, 1)
    if do_ext_2_pix:
        for r, c in zip(*ring2):
            visit(r, c, 2)
    idx_1pix = np.where(s1 >= 0)
    idx_2pix = np.where(s2[idx_1pix] >= 0)
    return s1.astype(np.int32), s2.astype(np.int32), idx_1pix, idx_2pix


def extrapolate_edge(phase, s1, s2, idx_1pix, idx_2pix):
    """Fill pixels just outside the pupil from their neighbours
    (extrapolate_edge_pixel.py:4-28)."""
    out = phase.copy()
    flat = phase.ravel()
    v1 = flat[s1[idx_1pix]]
    v2 = flat[s2[idx_1pix]]
    v1[idx_2pix] = 2 * v1[idx_2pix] - v2[idx_2pix]
    out[idx_1pix] = v1
    return out


class SHOracle:
    """Forward SH model on one electric field (sh.py:348-428)."""

    def __init__(self, geom: SHGeometry, wavelength_nm, ef_A_for_tables=None, precision=1):
        self.g = geom
        self.lam = wavelength_nm
        self.dtype = np.float32 if precision == 1 else np.float64
        self.cdtype = np.complex64 if precision == 1 else np.complex128
        g = geom
        self.tltf = tilt_factor(g.ovs_np_sub, g.fft_size - g.ovs_np_sub, self.cdtype)
        self.fp_mask = make_mask(g.fft_size, diaratio=g.fp_diaratio, square=g.squaremask)
        self.tables = None
        if g.do_interp:
            if ef_A_for_tables is None:
                raise ValueError('the interpolating geometry needs the pupil amplitude for its tables')
            self.tables = extrapol_tables(np.asarray(ef_A_for_tables), do_ext_2_pix=True)

    def psf_cut(self, A, phase, kernels_fft=None):
        """Masked, cut focal-plane cube (n*n, cutsize, cutsize) before toccd.
        ``kernels_fft`` (n*n, fft, fft): the LGS branch, where the unshifted
        |FFT|^2 goes through fft2, times the kernel spectrum, and an
        unnormalised inverse (sh.py:382-394) instead of the fftshift."""
        g = self.g
        A = np.asarray(A, dtype=self.dtype)
        phase = np.asarray(phase, dtype=self.dtype)
        if g.do_interp:
            pe = extrapolate_edge(phase, *self.tables)
            M = int(A.shape[0] * g.fov_ovs)
            yy, xx = interp2d_coords(A.shape, (M, M), g.rot_angle, g.xy_shift[0], g.xy_shift[1], self.dtype)
            A = interp2d(A, yy, xx, (M, M), self.dtype)
            phase = interp2d(pe, yy, xx, (M, M), self.dtype)
        n, p, N = g.n_lenses, g.ovs_np_sub, g.fft_size
        phi = phase * ((2 * np.pi) / self.lam)
        ef = np.exp(1j * phi, dtype=self.cdtype)
        ef *= A
        c = g.cutpixels
        cs = N - c
        out = None
        # a few lenslet rows at a time, as the reference's row loop
        # (sh.py:364-413) does: every sub-aperture's transform is independent,
        # so the chunking changes no value, only the working-set size
        rows = 1
        wf3 = np.zeros((rows * n, N, N), dtype=self.cdtype)   # the padding stays zero
        for r0 in range(0, n, rows):
            r1 = min(n, r0 + rows)
            cube = ef[r0 * p:r1 * p, :n * p].reshape(r1 - r0, p, n, p).transpose(0, 2, 1, 3).reshape(-1, p, p)
            wf3[:, :p, :p] = cube * self.tltf[np.newaxis]
            fp4 = np.fft.fft2(wf3, axes=(1, 2))
            psf = np.real(fp4 * np.conj(fp4))
            if kernels_fft is None:
                psf = np.fft.fftshift(psf, axes=(1, 2))
            else:
                spec = np.fft.fft2(psf, axes=(1, 2)) * np.asarray(kernels_fft)[r0 * n:r1 * n]
                psf = np.real(np.fft.ifft2(spec, axes=(1, 2), norm='forward')).astype(self.dtype)
            psf *= self.fp_mask[np.newaxis]
            if c > 0:
                psf = psf[:, c // 2: -c // 2, c // 2: -c // 2]
            if out is None:
                out = np.empty((n * n, cs if c > 0 else N, cs if c > 0 else N), dtype=psf.dtype)
            out[r0 * n:r1 * n] = psf
        return out

    def forward(self, A, phase, S0, pixel_pitch, kernels_fft=None):
        """Normalised detector-plane intensity (ccd_side x ccd_side)."""
        g = self.g
        n = g.n_lenses
        psf = self.psf_cut(A, phase, kernels_fft)
        cs = psf.shape[1]
        img = psf.reshape(n, n, cs, cs).transpose(0, 2, 1, 3).reshape(n * cs, n * cs)
        out = toccd(img, (g.ccd_side, g.ccd_side)).astype(self.dtype)
        A = np.asarray(A, dtype=self.dtype)
        phot = S0 * ((pixel_pitch ** 2) * np.sum(A))
        out *= (phot / out.sum())
        return out


ASEC2RAD = 1.0 / RAD2ASEC


def lgs_map_sh(nsh, diam, rl, zb, dz, profz, fwhmb, ps, ssp, theta=(0.0, 0.0)):
    """Geometric sodium-beacon images behind an nsh x nsh lenslet array
    (convolution_kernel.py:14-131, Gaussian radial profile, oversampling 1,
    no pupil weighting), in float64.  Returns (nsh*nsh, ssp, ssp) with
    index (lenslet column) * nsh + (lenslet row), as the reference's cube.

    For lenslet centre s, focal-plane sample f (angle times zb) and the
    on-axis point at distance dz from zb, the distance of the point seen from
    s to the beacon axis (launched from rl towards zb with tip-tilt theta):
    d2 = |f + dz (f - s)/zb - (b + dz e)|^2, e = (zb k + b - rl) / (zb + b_z - rl_z);
    each sample sums profz * exp(-d2 / (2 sigma^2)) / (sigma pi sqrt 2)."""
    s_ax = np.linspace(-diam / 2, diam / 2, nsh)
    f_ax = np.linspace(-ssp * ps / 2, ssp * ps / 2, ssp) * ASEC2RAD * zb
    sigma = fwhmb * ASEC2RAD * zb / (2 * np.sqrt(2 * np.log(2)))
    b = np.array([theta[0] * ASEC2RAD * zb, theta[1] * ASEC2RAD * zb, 0.0])
    axis = np.array([0.0, 0.0, float(zb)]) + b - np.broadcast_to(np.asarray(rl, dtype=np.float64), (3,))
    e = axis / axis[2]
    # full grid: rows = (lenslet row, sample row), columns = (lenslet column, sample column)
    fx = np.tile(f_ax, nsh)[np.newaxis, :]
    fy = np.tile(f_ax, nsh)[:, np.newaxis]
    sx = np.repeat(s_ax, ssp)[np.newaxis, :]
    sy = np.repeat(s_ax, ssp)[:, np.newaxis]
    fmap = np.zeros((nsh * ssp, nsh * ssp))
    gnorm = 1.0 / (sigma * np.pi * np.sqrt(2.0))
    for z, w in zip(np.atleast_1d(dz), np.atleast_1d(profz)):
        if w <= 0:
            continue
        dx = fx + z * (fx - sx) / zb - (b[0] + z * e[0])
        dy = fy + z * (fy - sy) / zb - (b[1] + z * e[1])
        dzz = z - (b[2] + z * e[2])
        fmap += gnorm * w * np.exp(-(dx * dx + dy * dy + dzz * dzz) / (2 * sigma ** 2))
    cube = fmap.reshape(nsh, ssp, nsh, ssp).transpose(2, 0, 1, 3).reshape(nsh * nsh, ssp, ssp)
    return cube


def lgs_kernel_spectra(real_kernels, nsh):
    """Per lenslet (row-major) the spectrum the SH multiplies by
    (convolution_kernel.py:260-276): each map normalised to unit sum and
    transformed with the normalised inverse FFT; map (column c, row r) goes
    to lenslet (r, c)."""
    rk = np.asarray(real_kernels, dtype=np.float64)
    out = np.zeros(rk.shape, dtype=np.complex128)
    for c in range(nsh):
        for r in range(nsh):
            k = rk[c * nsh + r]
            t = k.sum()
            if t > 0:
                k = k / t
            out[r * nsh + c] = np.fft.ifft2(k)
    return out
