"""Zernike influence functions on a pupil mask (host, setup time).

Restates specula/lib/compute_zern_ifunc.py:6-29 with the polynomials of
specula/lib/zernike_generator.py:142-190,192-246 (Noll ordering, index 1 =
piston, normalisation sqrt(2(n+1)), sqrt(n+1) for m = 0) evaluated at pixel
centres of a dim x dim grid with the unit disk of radius dim/2 centred at
dim/2; modes 2..nzern+1 sampled on the mask pixels, orthonormalised by a QR
decomposition (specula/lib/utils.py:51-84), then made zero-mean and unit-RMS.
"""
import numpy as np
from scipy.special import factorial

from specula_b200.lib.make_mask import make_mask


def radial_order(j):
    """Radial order n of Noll index j (zernike_generator.py:404-419)."""
    return np.ceil(0.5 * (np.sqrt(8 * np.array(j) + 1) - 3)).astype(int)


def degree(j):
    """(n, m) of Noll index j (zernike_generator.py:142-151)."""
    n = int(radial_order(j))
    cn = n * (n + 1) / 2 + 1
    if n % 2 == 0:
        m = int(j - cn + 1) // 2 * 2
    else:
        m = int(j - cn) // 2 * 2 + 1
    return n, m


def radial(n, m, rho, dtype):
    """R_n^m(rho) by the explicit factorial sum (float64 terms: the
    coefficients are float64 scalars)."""
    if (n - m) % 2 or abs(m) > n:
        raise ValueError(f'invalid Zernike degree ({n}, {m})')
    if n == 0 and m == 0:
        return np.ones(rho.shape, dtype=dtype)
    rho = np.where(rho < 0, 0, rho)
    out = np.zeros(rho.shape, dtype=dtype)
    for s in range((n - abs(m)) // 2 + 1):
        c = (-1) ** s * factorial(n - s) / (factorial(s) * factorial(-s + (n + abs(m)) / 2) *
                                            factorial(-s + (n - abs(m)) / 2))
        out = out + c * rho ** (n - 2 * s)
    return out


def polar_grid(dim, dtype):
    """rho, theta at pixel centres: unit disk of radius dim/2 centred at dim/2
    (the centre is held in ``dtype``; the grid itself is float64)."""
    sz = int(np.ceil(dim))
    c = np.ones(2, dtype=dtype) * (sz / 2)
    y, x = np.mgrid[0.5:sz + 0.5:1, 0.5:sz + 0.5:1]
    X = (x - c[1]) / (dim / 2)
    Y = (y - c[0]) / (dim / 2)
    return np.sqrt(X ** 2 + Y ** 2), np.arctan2(Y, X)


def zernike(j, rho, theta, dtype):
    n, m = degree(j)
    r = radial(n, m, rho, dtype)
    nc = np.sqrt(2 * (n + 1))
    if m == 0:
        return np.sqrt(0.5) * nc * r
    if j % 2 == 0:
        return nc * r * np.cos(m * theta)
    return nc * r * np.sin(m * theta)


def compute_zern_ifunc(dim, nzern, obsratio=0.0, diaratio=1.0, start_mode=0, mask=None, dtype=np.float32):
    """(nzern - start_mode) x n_mask orthonormalised Zernike modes (Noll
    2..nzern+1) on ``mask`` (default: make_mask(dim, obsratio, diaratio)),
    and the mask as ``dtype``."""
    if mask is None:
        mask = make_mask(dim, 0.0 if obsratio is None else obsratio, 1.0 if diaratio is None else diaratio)
    mask = np.asarray(mask).astype(float)
    idx = np.where(mask)
    mask = mask.astype(dtype)
    rho, theta = polar_grid(dim, dtype)
    # evaluated in float64, stored as dtype (zernike_generator.py:257-267)
    modes = np.stack([zernike(j, rho, theta, dtype).astype(dtype) for j in range(2, nzern + 2)])[start_mode:]
    z2 = np.array([m[idx] for m in modes], dtype=dtype)
    if z2.shape[1] > z2.shape[0]:
        q, _ = np.linalg.qr(z2.T)
        q = q.T
    else:
        q, _ = np.linalg.qr(z2)
    z2 = np.asarray(q, dtype=dtype)
    z2 = z2 - np.mean(z2, axis=1, keepdims=True)
    z2 = z2 / np.std(z2, axis=1, keepdims=True)
    return z2, mask
