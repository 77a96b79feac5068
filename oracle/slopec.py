"""Oracle: Shack-Hartmann slope computer (test infrastructure only).

Restates specula/processing_objects/sh_slopec.py:86-132 (weights) and
:308-438 (calc_slopes_nofor), plus the sub-aperture detection of
specula/processing_objects/sh_subap_calibrator.py:46-92.
"""
import numpy as np


def xy_weights(np_sub, exp_weight=1.0, precision=1):
    """CoG weights; x varies along columns (sh_slopec.py:98-132, no windowing).
    x/y stay float64 as in the reference, the mask takes the object dtype."""
    x, y = np.meshgrid(np.linspace(-1, 1, np_sub), np.linspace(-1, 1, np_sub))
    x = np.where(x > 0, np.power(x, exp_weight), -np.power(np.abs(x), exp_weight))
    y = np.where(y > 0, np.power(y, exp_weight), -np.power(np.abs(y), exp_weight))
    mask = np.ones((np_sub, np_sub), dtype=np.float32 if precision == 1 else np.float64)
    return x, y, mask


def sh_slopes(pixels, idxs, thr_value=-1, exp_weight=1.0, precision=1):
    """Returns (slopes [sx..., sy...], flux per sub-aperture).
    idxs: (n_subaps, np_sub**2) flattened indices into ``pixels``."""
    dtype = np.float32 if precision == 1 else np.float64
    n_sub, npx2 = idxs.shape
    np_sub = int(round(np.sqrt(npx2)))
    xw, yw, mw = xy_weights(np_sub, exp_weight, precision)
    ncols = pixels.shape[1]
    rows = idxs // ncols
    cols = idxs - rows * ncols
    p = pixels[rows, cols].T                     # (npx2, n_sub)
    flux = np.sum(p, axis=0)
    thr = thr_value if thr_value > 0 else 0
    p = p - thr
    p = np.where(p < 0, 0, p)
    tot = np.sum(p * mw.reshape(npx2, 1), axis=0)
    mean_tot = np.mean(tot)
    with np.errstate(divide='ignore'):
        factor = 1.0 / tot
    factor = np.where(factor > 1.0 / (mean_tot * 1e-3), 0, factor)
    sx = np.sum(p * xw.reshape(npx2, 1) * factor[np.newaxis, :], axis=0)
    sy = np.sum(p * yw.reshape(npx2, 1) * factor[np.newaxis, :], axis=0)
    slopes = np.zeros(2 * n_sub, dtype=dtype)
    slopes[:n_sub] = sx
    slopes[n_sub:] = sy
    return slopes, flux


def detect_subaps(image, n_lenses, energy_th):
    """Valid sub-aperture pixel tables (sh_subap_calibrator.py:46-92).
    Returns (idxs int64 (n_valid, np_sub**2), display_map int64 (n_valid,))."""
    npix = image.shape[0]
    step = 2.0 / n_lenses
    centres = (np.arange(n_lenses) - (n_lenses - 1) / 2.0) / (n_lenses / 2.0)   # make_xy vector
    np_sub = round(npix / 2.0 * step)
    spot = np.zeros((n_lenses, n_lenses))
    boxes = {}
    for i in range(n_lenses):
        for j in range(n_lenses):
            # Lenslet.get(i, j) = [x[i, j], y[i, j], size] with x varying along j
            lx = centres[j]
            ly = centres[i]
            xc = npix / 2.0 * (1 + lx)
            yc = npix / 2.0 * (1 + ly)
            r0, r1 = int(np.round(xc - np_sub / 2)), int(np.round(xc + np_sub / 2))
            c0, c1 = int(np.round(yc - np_sub / 2)), int(np.round(yc + np_sub / 2))
            boxes[(i, j)] = (r0, r1, c0, c1)
            spot[i, j] = np.sum(image[r0:r1, c0:c1])
    idxs, dmap = [], []
    for i in range(n_lenses):
        for j in range(n_lenses):
            if spot[i, j] > energy_th * np.max(spot):
                r0, r1, c0, c1 = boxes[(i, j)]
                rr, cc = np.meshgrid(np.arange(r0, r1), np.arange(c0, c1), indexing='ij')
                idxs.append(np.ravel_multi_index((rr.ravel(), cc.ravel()), image.shape))
                dmap.append(j * n_lenses + i)
    if not idxs:
        raise ValueError('no subapertures selected')
    return np.array(idxs, dtype=np.int64), np.array(dmap, dtype=np.int64)
