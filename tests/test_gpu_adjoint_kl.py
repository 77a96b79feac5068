"""The differentiable-SH workload at its stated size: 40x40 sub-apertures on
a 320 px / 8 m pupil, FFT 16 (6x6 detector pixels of lambda/d), noise-free,
500 KL modes of unit RMS.

* The adjoint interaction matrix with the KL basis against the float64
  oracle push-pull (im_rec_calibrator.py:58-63) at a small amplitude, on
  sampled modes: per-mode max|d|/max|ref| <= 1e-4.
* The slope Jacobian against float64 central differences (step 1e-3 rad RMS)
  along 32 seeded Kolmogorov phase probes of 1 rad RMS (von Karman screens
  of lib/calc_phasescreen.py, L0 25 m, seeds 0..31), at the flat calibration
  point and at four turbulent operating points: max|d|/max|ref| <= 1e-4.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import atmo as oatm, sh as osh, slopec as osl, control as octl  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-4
N_PROBES = 32
FD_STEP = 1e-3          # rad RMS


@pytest.fixture(scope='module')
def kl_system(cuda):
    from specula_b200.calibration import ShCalibrationSystem
    cal = ShCalibrationSystem(modes='kl')
    sh = cal.sh
    g = sh.geometry
    pix = cal.pupil.shape[0]
    geom = osh.sh_geometry(sh._wavelengthInNm, sh._subap_wanted_fov_arcsec, sh._sensor_pxscale_arcsec, g.n_lenses,
                           g.subap_npx, pix, cal.simul_params.pixel_pitch, fov_ovs_coeff=1.0)
    o64 = osh.SHOracle(geom, sh._wavelengthInNm, precision=0)
    A = cal.pupil.astype(np.float64)

    def slopes64(phase_nm):
        img = o64.forward(A, phase_nm, 1.0, cal.simul_params.pixel_pitch)
        return osl.sh_slopes(img, cal.subapdata.idxs, precision=0)[0]

    return cal, slopes64


def kolmogorov_probe(cal, seed, rms_rad=1.0):
    """Seeded von Karman screen cropped to the pupil, de-meaned and scaled to
    ``rms_rad`` over it, in nm."""
    pix = cal.pupil.shape[0]
    scr = oatm.calc_phasescreen(25.0, pix, cal.simul_params.pixel_pitch, seed=seed)[:pix, :pix]
    m = cal.pupil > 0
    scr = (scr - scr[m].mean()) * m
    scr *= rms_rad / np.sqrt(np.mean(scr[m] ** 2))
    return scr * cal.sh._wavelengthInNm / (2 * math.pi)


def dir_derivative(cal, jac, delta):
    """sum_px J[j][px] delta[px] (float64, host) from the Jacobian blocks."""
    adj = cal.adjoint
    J = jac.cpu().numpy().astype(np.float64)
    p, n, nv = adj.np_sub, adj.n_lenses, adj.n_valid
    out = np.zeros(2 * nv)
    for s, L in enumerate(adj._lenslet.cpu().numpy()):
        li, lj = divmod(int(L), n)
        blk = delta[li * p:(li + 1) * p, lj * p:(lj + 1) * p].ravel()
        out[s] = J[0, s] @ blk
        out[nv + s] = J[1, s] @ blk
    return out


def test_kl_basis_has_unit_rms_modes(kl_system):
    cal, _ = kl_system
    f = cal.dm._ifunc.influence_function.double()
    assert f.shape == (500, int((cal.pupil > 0).sum()))
    rms = torch.sqrt((f ** 2).mean(dim=1)).cpu().numpy()
    assert np.all(np.abs(rms - 1.0) < 1e-5)
    assert float(f.mean(dim=1).abs().max()) < 1e-5


def test_kl_adjoint_intmat_matches_fp64_pushpull(kl_system):
    cal, slopes64 = kl_system
    im = cal.adjoint_intmat().cpu().numpy()
    assert im.shape == (500, 2 * cal.n_valid)
    IF = cal.dm._ifunc.influence_function.cpu().numpy().astype(np.float64)
    amp = 1e-2                                   # nm RMS: O(a^2) truncation far below the tolerance

    def s64(k, a):
        cmd = np.zeros(IF.shape[0])
        cmd[k] = a
        return slopes64(octl.dm_phase(IF, cal.pupil, cmd, sign=cal.dm.sign, precision=0))

    for k in (0, 1, 2, 9, 50, 120, 250, 400, 499):
        ref = (s64(k, amp) - s64(k, -amp)) / amp
        assert rel_max_err(im[k], ref) <= ADJ_TOL, k


def test_kl_adjoint_full_intmat_matches_fp64_pushpull(kl_system):
    """Every row of the 500 x 2 n_valid matrix against the float64 oracle's
    push-pull at 1e-2 nm RMS (im_rec_calibrator.py:58-63: row k is
    s(+a)/a + s(-a)/(-a)), 1000 oracle forwards.  Mode k's phase is
    sign * a * IF[k] on the pupil, which is what dm.py:72-86 gives for a
    one-hot command."""
    cal, slopes64 = kl_system
    im = cal.adjoint_intmat().cpu().numpy().astype(np.float64)
    IF = cal.dm._ifunc.influence_function.cpu().numpy().astype(np.float64)
    idx = np.where(cal.pupil > 0)
    amp = 1e-2

    def s64(k, a):
        ph = np.zeros(cal.pupil.shape)
        ph[idx] = cal.dm.sign * a * IF[k]
        return slopes64(ph)

    ref = octl.pushpull_intmat(s64, IF.shape[0], np.full(IF.shape[0], amp))
    assert ref.shape == im.shape
    per_mode = np.array([rel_max_err(im[k], ref[k]) for k in range(im.shape[0])])
    print(f'full adjoint IM vs float64 push-pull: whole matrix {rel_max_err(im, ref):.2e}, '
          f'per mode max {per_mode.max():.2e} (mode {int(per_mode.argmax())}), median {np.median(per_mode):.2e}')
    assert rel_max_err(im, ref) <= ADJ_TOL
    assert per_mode.max() <= ADJ_TOL, int(per_mode.argmax())


@pytest.mark.parametrize('operating_point', [None, 0, 1, 2, 3])
def test_jacobian_on_kolmogorov_probes(kl_system, operating_point):
    """Flat calibration point (None) along all 32 probes; probe k as the
    operating point along four other probes."""
    cal, slopes64 = kl_system
    if operating_point is None:
        phi0 = np.zeros(cal.pupil.shape)
        directions = range(N_PROBES)
    else:
        phi0 = kolmogorov_probe(cal, operating_point)
        directions = [(operating_point + 7 * j + 1) % N_PROBES for j in range(4)]
    jac = cal.adjoint.jacobian(cal.A, torch.as_tensor(phi0.astype(np.float32), device=cal.device))
    for d in directions:
        delta = kolmogorov_probe(cal, d)
        ad = dir_derivative(cal, jac, delta)
        fd = (slopes64(phi0 + FD_STEP * delta) - slopes64(phi0 - FD_STEP * delta)) / (2 * FD_STEP)
        assert rel_max_err(ad, fd) <= ADJ_TOL, (operating_point, d)
