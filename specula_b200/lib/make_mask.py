"""Sampling grids and masks (same results as specula/lib/make_xy.py:1-186 for
the plain cartesian grid and specula/lib/make_mask.py:7-146 without spiders)."""
import numpy as np


def make_xy(sampling, ratio, dtype=None):
    """Pixel-centre coordinates over [-ratio, ratio]; x varies along axis 1."""
    if sampling <= 1:
        raise ValueError('make_xy: sampling must be larger than 1')
    v = (np.arange(sampling, dtype=dtype) - (sampling - 1) / 2.0) / (sampling / 2.0) * ratio
    x = np.tile(v, (sampling, 1))
    return x, x.T.copy()


def make_mask(np_size, obsratio=0.0, diaratio=1.0, xc=0.0, yc=0.0, square=False, inverse=False):
    """uint8 mask: circular (r < dia, r >= dia*obs) or square (Chebyshev) annulus."""
    obsratio = 0.0 if obsratio is None else obsratio
    diaratio = 1.0 if diaratio is None else diaratio
    x, y = make_xy(np_size, 1.0)
    dx, dy = x - xc, y - yc
    if square:
        ax, ay = np.abs(dx), np.abs(dy)
        sel = (ax <= diaratio) & (ay <= diaratio) & ((ax >= diaratio * obsratio) | (ay >= diaratio * obsratio))
    else:
        r2 = dx ** 2 + dy ** 2
        sel = (r2 < diaratio ** 2) & (r2 >= (diaratio * obsratio) ** 2)
    m = sel.astype(np.uint8)
    return 1 - m if inverse else m
