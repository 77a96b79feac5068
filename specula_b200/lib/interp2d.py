"""Sampling coordinates of the reference's Interp2D (specula/lib/interp2d.py:48-93)
for the SH oversampling path; the resampling itself is the sb_interp2d_field
kernel."""
import numpy as np


def interp_coords(input_shape, output_shape, rotInDeg=0, rowShiftInPixels=0, colShiftInPixels=0,
                  dtype=np.float32):
    """Clamped float32 row/column coordinates (flattened) of every output pixel."""
    yy, xx = (g.astype(dtype) for g in np.mgrid[0:output_shape[0], 0:output_shape[1]])
    yy *= (input_shape[0] - 1) / output_shape[0]
    xx *= (input_shape[1] - 1) / output_shape[1]
    if rotInDeg != 0:
        yc = input_shape[0] / 2 - 0.5
        xc = input_shape[1] / 2 - 0.5
        # the reference uses 3.1415 for pi here; kept for identical sampling
        ang = rotInDeg * 3.1415 / 180.0
        c, s = np.cos(ang), np.sin(ang)
        xr = (xx - xc) * c - (yy - yc) * s
        yr = (xx - xc) * s + (yy - yc) * c
        xx, yy = xr + xc, yr + yc
    if rowShiftInPixels != 0 or colShiftInPixels != 0:
        yy += rowShiftInPixels
        xx += colShiftInPixels
    yy = np.clip(yy, 0, input_shape[0] - 1).astype(dtype)
    xx = np.clip(xx, 0, input_shape[1] - 1).astype(dtype)
    return yy.ravel(), xx.ravel()


def interp_coords_xy(input_shape, yy, xx, rotInDeg=0, dtype=np.float32):
    """Clamped, flattened sample coordinates from caller-given float64 grids
    (Interp2D with xx / yy set, interp2d.py:56-90): rounded to ``dtype``,
    rotated about the input centre when ``rotInDeg`` is non-zero (in float64
    once the float32 grid meets the float64 cosines, as in the reference),
    clamped to the input and stored as ``dtype``."""
    yy = np.array(yy, dtype=dtype)
    xx = np.array(xx, dtype=dtype)
    if rotInDeg != 0:
        yc = input_shape[0] / 2 - 0.5
        xc = input_shape[1] / 2 - 0.5
        # the reference uses 3.1415 for pi here; kept for identical sampling
        c, s = np.cos(rotInDeg * 3.1415 / 180.0), np.sin(rotInDeg * 3.1415 / 180.0)
        xr = (xx - xc) * c - (yy - yc) * s
        yr = (xx - xc) * s + (yy - yc) * c
        xx, yy = xr + xc, yr + yc
    yy = np.clip(yy, 0, input_shape[0] - 1).astype(dtype)
    xx = np.clip(xx, 0, input_shape[1] - 1).astype(dtype)
    return yy.ravel(), xx.ravel()
