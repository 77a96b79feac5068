"""Shared test cases: the SH geometries the golden fixtures were made with
(same list as tests/golden/make_golden.py)."""
import numpy as np

RAD2ASEC = 180 * 3600 / np.pi


def lam_over_d_arcsec(lam_nm, d_m):
    return lam_nm * 1e-9 / d_m * RAD2ASEC


SH_CASES = [
    ('c1_plain16', 160, 0.05, 750.0, 8 * 0.875 * lam_over_d_arcsec(750, 0.4), 0.875 * lam_over_d_arcsec(750, 0.4), 20, 8, 1.0),
    ('c1_interp', 160, 0.05, 750.0, 8 * lam_over_d_arcsec(750, 0.4), lam_over_d_arcsec(750, 0.4), 20, 8, 0.0),
    ('flux120', 120, 0.05, 500.0, 3.0, 0.5, 20, 6, 0.0),
    ('test64', 64, 0.015625, 600.0, 4.0, 0.5, 8, 8, 0.0),
    ('n16_fft32', 128, 0.05, 750.0, 6 * 0.5 * lam_over_d_arcsec(750, 0.4), 0.5 * lam_over_d_arcsec(750, 0.4), 16, 6, 1.0),
    ('n16_fft16', 128, 0.05, 750.0, 6 * lam_over_d_arcsec(750, 0.4), lam_over_d_arcsec(750, 0.4), 16, 6, 1.0),
]
SH_S0 = 7.0


def rel_max_err(a, b):
    """max |a - b| / max |b| (the intensity / slope tolerance metric; complex
    arrays compare as complex numbers)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    a = np.asarray(a, dtype=np.complex128 if cplx else np.float64)
    b = np.asarray(b, dtype=np.complex128 if cplx else np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
