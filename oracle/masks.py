"""Oracle: sampling grids and masks (test infrastructure only).

Restates specula/lib/make_xy.py:1-186 (cartesian branch only) and
specula/lib/make_mask.py:7-146 (no spiders).
"""
import numpy as np

ASEC2RAD = np.pi / (3600 * 180)
RAD2ASEC = 1.0 / ASEC2RAD


def make_xy(sampling, ratio, dtype=None):
    """Pixel-centre coordinates of a sampling x sampling grid spanning
    [-ratio, ratio]; x varies along axis 1, y along axis 0
    (make_xy.py:155-176, non-quarter, non-fft, not zero_sampled)."""
    if sampling <= 1:
        raise ValueError('sampling must be larger than 1')
    x0 = (sampling - 1) / 2.0
    x = (np.arange(sampling, dtype=dtype) - x0) / (sampling / 2.0) * ratio
    xx = np.tile(x, (sampling, 1))
    return xx, xx.T.copy()


def make_mask(n, obsratio=0.0, diaratio=1.0, xc=0.0, yc=0.0, square=False):
    """uint8 pupil / field-stop mask (make_mask.py:58-104)."""
    if diaratio is None:
        diaratio = 1.0
    if obsratio is None:
        obsratio = 0.0
    x, y = make_xy(n, 1.0)
    dx = x - xc
    dy = y - yc
    if square:
        inside = (np.abs(dx) <= diaratio) & (np.abs(dy) <= diaratio) & \
                 ((np.abs(dx) >= diaratio * obsratio) | (np.abs(dy) >= diaratio * obsratio))
    else:
        r2 = dx ** 2 + dy ** 2
        inside = (r2 < diaratio ** 2) & (r2 >= (diaratio * obsratio) ** 2)
    m = np.zeros((n, n), dtype=np.uint8)
    m[inside] = 1
    return m
