"""Oracle: Shack-Hartmann slope computer (test infrastructure only).

Restates specula/processing_objects/sh_slopec.py:86-132 (weights) and
:308-438 (calc_slopes_nofor), plus the sub-aperture detection of
specula/processing_objects/sh_subap_calibrator.py:46-92.
"""
import numpy as np


def xy_weights(np_sub, exp_weight=1.0, precision=1, quadcell_mode=False, weighted_pix_rad=0.0, windowing=False):
    """CoG weights; x varies along columns (sh_slopec.py:98-132).
    x/y stay float64 as in the reference, the mask takes the object dtype.
    quadcell_mode: weights are the signs (:101-104).  weighted_pix_rad != 0
    with windowing: a circular window of diameter 2 * weighted_pix_rad pixels
    (:117-119, make_mask); without windowing a Gaussian of FWHM
    weighted_pix_rad on the [-1, 1] grid normalised to its peak (the
    psf_gaussian of :440-445 that :121 means to call); entries below 1e-6 are
    zeroed and the x/y weights multiplied by the mask (:125-128)."""
    from oracle.masks import make_mask
    dtype = np.float32 if precision == 1 else np.float64
    x, y = np.meshgrid(np.linspace(-1, 1, np_sub), np.linspace(-1, 1, np_sub))
    if quadcell_mode:
        x = np.where(x > 0, 1.0, -1.0)
        y = np.where(y > 0, 1.0, -1.0)
    else:
        x = np.where(x > 0, np.power(x, exp_weight), -np.power(np.abs(x), exp_weight))
        y = np.where(y > 0, np.power(y, exp_weight), -np.power(np.abs(y), exp_weight))
    if weighted_pix_rad != 0:
        if windowing:
            mask = make_mask(np_sub, diaratio=2.0 * weighted_pix_rad / np_sub).astype(np.float64)
        else:
            g, h = np.meshgrid(np.linspace(-1, 1, np_sub), np.linspace(-1, 1, np_sub))
            mask = np.exp(-4 * np.log(2) * (g ** 2 + h ** 2) / weighted_pix_rad ** 2, dtype=dtype)
            mask = mask / np.max(mask)
        mask[mask < 1e-6] = 0.0
        x = x * mask.astype(dtype)
        y = y * mask.astype(dtype)
    else:
        mask = np.ones((np_sub, np_sub), dtype=dtype)
    return x, y, mask


def sh_slopes(pixels, idxs, thr_value=-1, exp_weight=1.0, precision=1, thr_pedestal=False, thr_ratio_value=0.0,
              win_mat=None, mult_factor=0.0, weights=None):
    """Returns (slopes [sx..., sy...], flux per sub-aperture).
    idxs: (n_subaps, np_sub**2) flattened indices into ``pixels``.
    Options (sh_slopec.py:364-418): win_mat (np_sub, np_sub, n_subaps)
    multiplies the pixels after the flux sums; thr_ratio_value > 0 sets each
    sub-aperture's threshold to that fraction of its largest windowed pixel
    (the per-sub-aperture loop, :215-232, the form of it that runs); thr_pedestal
    zeroes the pixels below the threshold instead of subtracting it;
    mult_factor != 0 scales the slopes.  weights: (x, y, mask) from
    xy_weights, default the exponential-law weights."""
    dtype = np.float32 if precision == 1 else np.float64
    n_sub, npx2 = idxs.shape
    np_sub = int(round(np.sqrt(npx2)))
    xw, yw, mw = weights if weights is not None else xy_weights(np_sub, exp_weight, precision)
    ncols = pixels.shape[1]
    rows = idxs // ncols
    cols = idxs - rows * ncols
    p = pixels[rows, cols].T                     # (npx2, n_sub)
    flux = np.sum(p, axis=0)
    if win_mat is not None:
        p = p * np.asarray(win_mat).reshape(npx2, n_sub)
    if thr_value > 0 and thr_ratio_value > 0:
        raise ValueError('thr_value and thr_ratio_value are exclusive')
    if thr_ratio_value > 0:
        thr = thr_ratio_value * np.max(p, axis=0, keepdims=True)
    elif thr_pedestal or thr_value > 0:
        thr = thr_value
    else:
        thr = 0
    if thr_pedestal:
        p = np.where(p < thr, 0, p)
    else:
        p = p - thr
        p = np.where(p < 0, 0, p)
    tot = np.sum(p * mw.reshape(npx2, 1), axis=0)
    mean_tot = np.mean(tot)
    with np.errstate(divide='ignore'):
        factor = 1.0 / tot
    factor = np.where(factor > 1.0 / (mean_tot * 1e-3), 0, factor)
    sx = np.sum(p * xw.reshape(npx2, 1) * factor[np.newaxis, :], axis=0)
    sy = np.sum(p * yw.reshape(npx2, 1) * factor[np.newaxis, :], axis=0)
    if mult_factor != 0:
        sx = sx * mult_factor
        sy = sy * mult_factor
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
