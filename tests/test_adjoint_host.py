"""Host-side pieces of the adjoint interaction matrix (no GPU): the index
tables handed to sb_sh_slopes_jacobian / sb_intmat_contract, and the adjoint
equations the kernel implements, restated in float64 numpy on the same
device tables and checked against central differences of the float64
oracle forward (SH then CoG)."""
import math

import numpy as np
import pytest

from oracle import sh as osh, slopec as osl
from oracle.masks import make_mask
from tests.cases import SH_CASES, rel_max_err


def test_lenslet_index_from_subap_table():
    from specula_b200.lib.sh_adjoint import lenslet_index
    n, npx = 5, 4
    idxs, _ = osl.detect_subaps(np.ones((n * npx, n * npx)), n, 0.5)
    lens = lenslet_index(idxs, n, npx)
    ncols = n * npx
    for s, L in enumerate(lens):
        li, lj = divmod(int(L), n)
        box = [(li * npx + r) * ncols + lj * npx + c for r in range(npx) for c in range(npx)]
        assert sorted(idxs[s].tolist()) == box


def test_lenslet_index_rejects_misaligned_boxes():
    from specula_b200.lib.sh_adjoint import lenslet_index
    idxs = np.array([[1, 2, 9, 10]])
    with pytest.raises(ValueError):
        lenslet_index(idxs, 4, 2)


def test_pixel_to_column_with_crop():
    from specula_b200.lib.sh_adjoint import pixel_to_column
    dm_shape = (6, 7)
    mask = np.zeros(dm_shape, bool)
    mask[1:5, 2:6] = True
    mask[0, 0] = True                      # outside the cropped field
    idx = np.flatnonzero(mask.ravel())
    out = pixel_to_column(idx, dm_shape, 4, top=1, left=2)
    assert out.shape == (16,)
    assert np.all(out >= 0)
    for col, flat in enumerate(idx):
        r, c = divmod(int(flat), dm_shape[1])
        if (r, c) == (0, 0):
            assert col not in out
        else:
            assert out[(r - 1) * 4 + (c - 2)] == col


def _smooth(pix, rng, rms, kmax=5):
    y, x = np.mgrid[0:pix, 0:pix] / pix
    f = np.zeros((pix, pix))
    for kx in range(-kmax, kmax + 1):
        for ky in range(0, kmax + 1):
            if kx or ky:
                f += rng.standard_normal() / (kx * kx + ky * ky) ** (11 / 12) * \
                    np.cos(2 * np.pi * (kx * x + ky * y) + rng.uniform(0, 2 * np.pi))
    return f * (rms / f.std())


@pytest.mark.parametrize('name', ['c1_plain16', 'n16_fft16'])
def test_adjoint_equations_match_oracle_finite_differences(name):
    """g = (w - s mw)/tot -> R^T g R -> 2 (h M) F -> W^H Gf conj(W) ->
    -k Im(conj(dE) E), on the pruned-DFT / field-stop / rebin tables that
    the SH plan uploads, against float64 central differences."""
    from specula_b200.lib import sh_geometry as shg
    from specula_b200.lib.sh_adjoint import lenslet_index
    case = [c for c in SH_CASES if c[0] == name][0]
    _, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    g = shg.solve(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    P, CS, NPX = g.ovs_np_sub, g.cutsize, g.subap_npx
    W = shg.twiddle_table(P, g.fft_size, g.cutpixels).astype(np.complex128)
    T = shg.tilt_table(P, g.fft_size).astype(np.complex128)
    M = shg.field_stop_cut(g).astype(np.float64).reshape(CS, CS)
    R = shg.rebin_table(CS, NPX).astype(np.float64).reshape(NPX, CS)
    k = 2 * math.pi / lam
    A = make_mask(pix, 0.14, 1.0).astype(np.float64)
    geom = osh.sh_geometry(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    flat = osh.SHOracle(geom, lam, precision=1).forward(A.astype(np.float32), np.zeros((pix, pix), np.float32),
                                                        5.0, pitch)
    idxs, _ = osl.detect_subaps(flat, n, 0.5)
    lens = lenslet_index(idxs, n, npx)
    o64 = osh.SHOracle(geom, lam, precision=0)

    def s64(ph):
        return osl.sh_slopes(o64.forward(A, ph, 5.0, pitch), idxs, precision=0)[0]

    nm_per_rad = lam / (2 * math.pi)
    ph0 = _smooth(pix, np.random.default_rng(7), 0.6) * nm_per_rad * A
    v = np.linspace(-1, 1, NPX)
    xw, yw = np.meshgrid(v, v)
    nv = len(lens)
    J = np.zeros((2, nv, P * P))
    for s, L in enumerate(lens):
        li, lj = divmod(int(L), n)
        blk = np.s_[li * P:(li + 1) * P, lj * P:(lj + 1) * P]
        E = A[blk] * np.exp(1j * k * ph0[blk]) * T
        F = W @ E @ W.T
        D = R @ (np.abs(F) ** 2 * M) @ R.T
        tot = D.sum()
        for ax, w in enumerate((xw, yw)):
            gD = (w - (D * w).sum() / tot) / tot
            Gf = 2 * (R.T @ gD @ R) * M * F
            dE = W.conj().T @ Gf @ W.conj()
            J[ax, s] = (-k * np.imag(np.conj(dE) * E)).ravel()
    eps = 1e-3
    d = _smooth(pix, np.random.default_rng(100), 1.0) * nm_per_rad
    ad = np.zeros(2 * nv)
    for s, L in enumerate(lens):
        li, lj = divmod(int(L), n)
        blk = d[li * P:(li + 1) * P, lj * P:(lj + 1) * P].ravel()
        ad[s], ad[nv + s] = J[0, s] @ blk, J[1, s] @ blk
    fd = (s64(ph0 + eps * d) - s64(ph0 - eps * d)) / (2 * eps)
    assert rel_max_err(ad, fd) <= 1e-6
