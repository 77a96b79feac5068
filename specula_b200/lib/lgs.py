"""Laser-guide-star pieces of the SH (sh.py:289-321, 382-394;
data_objects/convolution_kernel.py): the geometric sodium-beacon maps on the
device, their spectra, and the DFT tables of sb_sh_forward_lgs.

``lgs_map_sh`` follows convolution_kernel.py:14-131 (Gaussian radial
profile): for lenslet centre s, focal-plane sample f (angle x zb) and the
beacon point at distance dz from zb along the launch axis,
d2 = |f + dz (f - s)/zb - (b + dz e)|^2 with e the launch direction scaled to
unit z; every sample sums profz * exp(-d2 / (2 sigma^2)) / (sigma pi sqrt 2).
The geometry runs in float64 on the device and the maps are stored in
float32, as the reference's.
"""
import math

import numpy as np
import torch

from specula_b200 import ASEC2RAD


def lgs_map_sh(nsh, diam, rl, zb, dz, profz, fwhmb, ps, ssp, overs=1, theta=(0.0, 0.0), rprof_type=0,
               device='cuda'):
    """(nsh*nsh, ssp, ssp) float32 maps, index (lenslet column) * nsh +
    (lenslet row), as the reference's cube."""
    if overs != 1:
        raise NotImplementedError('lgs_map_sh: oversampling other than 1 is not on the specula_b200 path')
    if rprof_type not in (0, 1):
        raise ValueError('Unsupported radial profile type')
    f64 = dict(dtype=torch.float64, device=device)
    s_ax = torch.linspace(-diam / 2, diam / 2, nsh, **f64)
    f_ax = torch.linspace(-ssp * ps / 2, ssp * ps / 2, ssp, **f64) * (ASEC2RAD * zb)
    sigma = fwhmb * ASEC2RAD * zb / (2 * math.sqrt(2 * math.log(2)))
    th = np.asarray(theta, dtype=np.float64)
    b = np.array([th[0] * ASEC2RAD * zb, th[1] * ASEC2RAD * zb, 0.0])
    axis = np.array([0.0, 0.0, float(zb)]) + b - np.broadcast_to(np.asarray(rl, dtype=np.float64), (3,))
    e = axis / axis[2]
    fx = f_ax.repeat(nsh).view(1, -1)
    fy = f_ax.repeat(nsh).view(-1, 1)
    sx = s_ax.repeat_interleave(ssp).view(1, -1)
    sy = s_ax.repeat_interleave(ssp).view(-1, 1)
    fmap = torch.zeros((nsh * ssp, nsh * ssp), **f64)
    if rprof_type == 0:
        gnorm = 1.0 / (sigma * math.pi * math.sqrt(2.0))
    else:
        gnorm = 1.0 / (math.pi / 4 * (fwhmb * ASEC2RAD * zb) ** 2)
    for z, w in zip(np.atleast_1d(np.asarray(dz, dtype=np.float64)), np.atleast_1d(np.asarray(profz, np.float64))):
        if w <= 0:
            continue
        dx = fx + z * (fx - sx) / zb - (b[0] + z * e[0])
        dy = fy + z * (fy - sy) / zb - (b[1] + z * e[1])
        dzz = z - (b[2] + z * e[2])
        d2 = dx * dx + dy * dy + dzz * dzz
        if rprof_type == 0:
            fmap += (gnorm * w) * torch.exp(-d2 / (2 * sigma ** 2))
        else:
            fmap += (gnorm * w) * (d2 / sigma ** 2 <= 1.0).to(torch.float64)
    cube = fmap.view(nsh, ssp, nsh, ssp).permute(2, 0, 1, 3).reshape(nsh * nsh, ssp, ssp)
    return cube.to(torch.float32).contiguous()


def kernel_spectra(real_kernels, nsh, out=None):
    """Per lenslet (row-major) the spectrum the SH multiplies by
    (convolution_kernel.py:260-276): each map normalised to unit sum, then the
    normalised inverse FFT; map (column c, row r) goes to lenslet (r, c).
    Written into ``out`` (complex64, same address every update) when given."""
    rk = real_kernels.to(torch.float64)
    tot = rk.sum(dim=(1, 2), keepdim=True)
    rk = torch.where(tot > 0, rk / torch.where(tot > 0, tot, torch.ones_like(tot)), rk)
    spec = torch.fft.ifft2(rk.to(torch.float32)).to(torch.complex64)
    n, s1, s2 = spec.shape
    spec = spec.view(nsh, nsh, s1, s2).transpose(0, 1).reshape(n, s1, s2)
    if out is None:
        return spec.contiguous()
    out.copy_(spec)
    return out


def _phase_table(rows, cols, n, sign, row_offset=0):
    """exp(sign * 2 pi i ((r + row_offset) c mod n) / n), complex64, from float64 phases."""
    r = (np.arange(rows) + row_offset)[:, None]
    c = np.arange(cols)[None, :]
    ph = sign * (2.0 * np.pi / n) * ((r * c) % n)
    return (np.cos(ph) + 1j * np.sin(ph)).astype(np.complex64)


def lgs_tables(np_sub, fft_size, cutpixels, cutsize):
    """Host tables of sb_sh_forward_lgs: (w_full_t [np_sub][N], w_dft [N][N],
    v_inv_t [N][cutsize]), complex64."""
    N = int(fft_size)
    w_full_t = _phase_table(N, np_sub, N, -1.0).T.copy()        # [c][k]
    w_dft = _phase_table(N, N, N, -1.0)
    v_inv_t = _phase_table(cutsize, N, N, +1.0, row_offset=cutpixels // 2).T.copy()   # [u][a]
    return w_full_t, w_dft, v_inv_t
