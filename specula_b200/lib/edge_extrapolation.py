"""Edge-pixel extrapolation tables for the SH oversampling path.

Builds the same integer tables as
specula/lib/extrapolate_edge_pixel_mat_define.py:5-143: for each pixel just
outside the pupil (1-pixel ring, then the 2-pixel ring), the first in-pupil
neighbour found along +col, -col, +row, -row (the reference's y-before-x
precedence) and, when the next pixel in that direction is inside too, that
second pixel for a linear extrapolation.  Edge limits keep the reference's
strict ``< size-1`` / ``> 0`` tests.

``per_pixel_tables`` turns them into the flat per-pixel form consumed by the
sb_edge_extrapolate kernel.
"""
import numpy as np


def extrapolation_tables(mask, do_ext_2_pix=True):
    mask = np.asarray(mask)
    nr, nc = mask.shape
    inside = mask > 0
    flat_index = np.arange(nr * nc, dtype=np.int64).reshape(nr, nc)
    src1 = np.full((nr, nc), -1, dtype=np.int64)
    src2 = np.full((nr, nc), -1, dtype=np.int64)
    # the rings use the raw amplitude values, as the reference does
    f = mask.astype(float)

    def ring(d):
        return (np.roll(f, d, 0) + np.roll(f, -d, 0) + np.roll(f, d, 1) + np.roll(f, -d, 1)) * (1.0 - f)

    r1 = ring(1)
    r2 = ring(2)
    passes = [(1, np.argwhere(r1 > 0))]
    if do_ext_2_pix:
        passes.append((2, np.argwhere((r2 > 0) & (r1 == 0))))
    dirs = ((0, 1), (0, -1), (1, 0), (-1, 0))
    for d, pix in passes:
        guard = src1 if d == 1 else src2
        for r, c in pix:
            fallback = -1
            for dr, dc in dirs:
                if guard[r, c] != -1:
                    break
                ra, ca = r + dr * d, c + dc * d
                rb, cb = r + dr * (d + 1), c + dc * (d + 1)
                if dr == 0:
                    ok_a = ca < nc - 1 if dc > 0 else ca > 0
                    ok_b = cb < nc - 1 if dc > 0 else cb > 0
                else:
                    ok_a = ra < nr - 1 if dr > 0 else ra > 0
                    ok_b = rb < nr - 1 if dr > 0 else rb > 0
                if not ok_a or not inside[ra, ca]:
                    continue
                if ok_b and inside[rb, cb]:
                    src2[r, c] = flat_index[rb, cb]
                    src1[r, c] = flat_index[ra, ca]
                else:
                    fallback = flat_index[ra, ca]
            if src1[r, c] == -1 and fallback >= 0:
                src1[r, c] = fallback
    return src1.astype(np.int32), src2.astype(np.int32)


def per_pixel_tables(src1, src2):
    """Flat int32 tables for sb_edge_extrapolate: s1[p] < 0 keeps the pixel,
    s2[p] < 0 copies s1[p], else 2*phase[s1] - phase[s2]."""
    s1 = np.asarray(src1, dtype=np.int32).ravel().copy()
    s2 = np.asarray(src2, dtype=np.int32).ravel().copy()
    s2[s1 < 0] = -1
    return s1, s2
