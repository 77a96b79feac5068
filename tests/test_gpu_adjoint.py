"""GPU parity of the SH slopes adjoint and the adjoint interaction matrix
(sb_sh_slopes_jacobian, sb_sh_slopes_vjp, sb_intmat_contract) against the
float64 oracle: central finite differences of the oracle forward (SH then
CoG) and the oracle's push-pull matrix at a small amplitude.

Tolerances (written per test): directional derivatives and interaction
matrices max|d|/max|ref| <= 1e-4; internal consistency of the VJP with the
Jacobian <= 1e-5.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import sh as osh, slopec as osl, control as octl  # noqa: E402
from oracle.masks import make_mask  # noqa: E402
from tests.cases import SH_CASES, rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-4
VJP_TOL = 1e-5
S0 = 5.0
FLAT_CASES = [c for c in SH_CASES if c[8] == 1.0]    # one phase sample per lenslet pixel


def smooth_field(pix, rng, rms, kmax=5):
    """Seeded smooth random field (sum of low spatial frequencies), given RMS."""
    y, x = np.mgrid[0:pix, 0:pix] / pix
    f = np.zeros((pix, pix))
    for kx in range(-kmax, kmax + 1):
        for ky in range(0, kmax + 1):
            if kx == 0 and ky == 0:
                continue
            amp = rng.standard_normal() / (kx * kx + ky * ky) ** (11 / 12)
            f += amp * np.cos(2 * np.pi * (kx * x + ky * y) + rng.uniform(0, 2 * np.pi))
    return f * (rms / f.std())


def _setup(case):
    from specula_b200.processing_objects.sh import SH
    from specula_b200.processing_objects.sh_slopec import ShSlopec
    from specula_b200.data_objects.electric_field import ElectricField
    from specula_b200.data_objects.pixels import Pixels
    from specula_b200.data_objects.subap_data import SubapData
    from specula_b200.lib.sh_adjoint import ShSlopesAdjoint
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n, subap_npx=npx,
            fov_ovs_coeff=coeff, target_device_idx=0)
    ef = ElectricField(pix, pix, pitch, S0=S0, target_device_idx=0)
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    ef.A.copy_(torch.as_tensor(A))
    sh.inputs['in_ef'].set(ef)
    sh.setup()
    geom = osh.sh_geometry(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    flat = osh.SHOracle(geom, lam, ef_A_for_tables=A, precision=1).forward(A, np.zeros_like(A), S0, pitch)
    idxs, dmap = osl.detect_subaps(flat, n, 0.5)
    px = Pixels(n * npx, n * npx, target_device_idx=0)
    sl = ShSlopec(SubapData(idxs=idxs, display_map=dmap, nx=n, ny=n, target_device_idx=0), target_device_idx=0)
    sl.inputs['in_pixels'].set(px)
    sl.setup()
    adj = ShSlopesAdjoint(sh, sl)
    oracle64 = osh.SHOracle(geom, lam, ef_A_for_tables=A, precision=0)

    def slopes64(phase):
        img = oracle64.forward(A.astype(np.float64), phase, S0, pitch)
        return osl.sh_slopes(img, idxs, precision=0)[0]

    return dict(sh=sh, sl=sl, adj=adj, A=A, idxs=idxs, lam=lam, pix=pix, n=n, slopes64=slopes64)


def _dir_derivative(jac, idxs_lenslet, n, p, delta):
    """sum_px J[j][px] delta[px] on the host (float64) from the Jacobian blocks."""
    jac = jac.detach().cpu().numpy().astype(np.float64)
    out = np.zeros(2 * jac.shape[1])
    nv = jac.shape[1]
    for s, L in enumerate(idxs_lenslet):
        li, lj = divmod(int(L), n)
        blk = delta[li * p:(li + 1) * p, lj * p:(lj + 1) * p].ravel()
        out[s] = jac[0, s] @ blk
        out[nv + s] = jac[1, s] @ blk
    return out


@pytest.mark.parametrize('case', FLAT_CASES, ids=[c[0] for c in FLAT_CASES])
def test_jacobian_matches_fp64_finite_differences(case, cuda):
    c = _setup(case)
    adj, A, lam, pix = c['adj'], c['A'], c['lam'], c['pix']
    rng = np.random.default_rng(7)
    nm_per_rad = lam / (2 * math.pi)
    phase0 = (smooth_field(pix, rng, 0.6) * nm_per_rad * A).astype(np.float32)
    jac = adj.jacobian(torch.as_tensor(A), torch.as_tensor(phase0))
    lens = adj._lenslet.cpu().numpy()
    eps = 1e-3                                   # rad RMS of the probe step
    for probe in range(4):
        delta = smooth_field(pix, np.random.default_rng(100 + probe), 1.0) * nm_per_rad
        ad = _dir_derivative(jac, lens, c['n'], adj.np_sub, delta)
        p64 = phase0.astype(np.float64)
        fd = (c['slopes64'](p64 + eps * delta) - c['slopes64'](p64 - eps * delta)) / (2 * eps)
        assert rel_max_err(ad, fd) <= ADJ_TOL, probe


@pytest.mark.parametrize('case', FLAT_CASES[:2], ids=[c[0] for c in FLAT_CASES[:2]])
def test_vjp_equals_jacobian_transpose(case, cuda):
    c = _setup(case)
    adj, A, pix, n = c['adj'], c['A'], c['pix'], c['n']
    rng = np.random.default_rng(3)
    phase0 = (smooth_field(pix, rng, 80.0) * A).astype(np.float32)
    jac = adj.jacobian(torch.as_tensor(A), torch.as_tensor(phase0)).cpu().numpy().astype(np.float64)
    seed = rng.standard_normal(2 * adj.n_valid).astype(np.float32)
    got = adj.vjp(torch.as_tensor(A), torch.as_tensor(phase0), torch.as_tensor(seed)).cpu().numpy()
    ref = np.zeros((pix, pix))
    p, nv = adj.np_sub, adj.n_valid
    for s, L in enumerate(adj._lenslet.cpu().numpy()):
        li, lj = divmod(int(L), n)
        blk = seed[s] * jac[0, s] + seed[nv + s] * jac[1, s]
        ref[li * p:(li + 1) * p, lj * p:(lj + 1) * p] = blk.reshape(p, p)
    assert rel_max_err(got, ref) <= VJP_TOL


def _dm(c, n_modes, seed):
    from specula_b200.processing_objects.dm import DM
    from specula_b200.data_objects.ifunc import IFunc
    from specula_b200.data_objects.simul_params import SimulParams
    from specula_b200.base_value import BaseValue
    pix, A = c['pix'], c['A']
    mask = A > 0
    rng = np.random.default_rng(seed)
    IF = np.stack([smooth_field(pix, rng, 1.0, kmax=3 + k // 4)[mask] for k in range(n_modes)]).astype(np.float32)
    sp = SimulParams(pixel_pupil=pix, pixel_pitch=0.05, time_step=0.001)
    dm = DM(sp, 0, ifunc=IFunc(ifunc=IF, mask=mask.astype(np.float32), target_device_idx=0), target_device_idx=0)
    dm.inputs['in_command'].set(BaseValue(value=np.zeros(n_modes, np.float32), target_device_idx=0))
    dm.setup()
    return dm, IF, mask


@pytest.mark.parametrize('case', FLAT_CASES, ids=[c[0] for c in FLAT_CASES])
def test_adjoint_intmat_matches_fp64_pushpull(case, cuda):
    c = _setup(case)
    adj, A, pix = c['adj'], c['A'], c['pix']
    dm, IF, mask = _dm(c, 10, seed=5)
    flat = torch.zeros((pix, pix), dtype=torch.float32, device='cuda')
    im = adj.intmat(torch.as_tensor(A), flat, dm).cpu().numpy()
    # the reference's push-pull (im_rec_calibrator.py:58-63) in float64 at
    # a small amplitude (truncation O(a^2) far below the tolerance)
    amp = 1e-2

    def slopes_fn(k, a):
        cmd = np.zeros(IF.shape[0])
        cmd[k] = a
        return c['slopes64'](octl.dm_phase(IF.astype(np.float64), mask, cmd, sign=dm.sign, precision=0))

    ref = octl.pushpull_intmat(slopes_fn, IF.shape[0], [amp] * IF.shape[0])
    assert im.shape == ref.shape
    assert rel_max_err(im, ref) <= ADJ_TOL


INTERP_CASES = [c for c in SH_CASES if c[0] == 'c1_interp']    # the SH resamples its field (fov_ovs != 1)


@pytest.mark.parametrize('case', INTERP_CASES, ids=[c[0] for c in INTERP_CASES])
def test_adjoint_intmat_with_resampling_matches_fp64_pushpull(case, cuda):
    """The adjoint interaction matrix through the SH's edge extrapolation and
    interpolation (sh.py:353-357,447-460): the influence functions resampled
    by the same linear map, against the float64 oracle's push-pull."""
    c = _setup(case)
    adj, A, pix = c['adj'], c['A'], c['pix']
    assert adj.interp and adj.field != pix
    dm, IF, mask = _dm(c, 10, seed=5)
    flat = torch.zeros((pix, pix), dtype=torch.float32, device='cuda')
    im = adj.intmat(torch.as_tensor(A), flat, dm).cpu().numpy()
    amp = 1e-2

    def slopes_fn(k, a):
        cmd = np.zeros(IF.shape[0])
        cmd[k] = a
        return c['slopes64'](octl.dm_phase(IF.astype(np.float64), mask, cmd, sign=dm.sign, precision=0))

    ref = octl.pushpull_intmat(slopes_fn, IF.shape[0], [amp] * IF.shape[0])
    assert rel_max_err(im, ref) <= ADJ_TOL
    # the push-pull on the GPU chain, resampling included, agrees too
    pp, _ = adj.pushpull_intmat(torch.as_tensor(A), dm, 1.0, graph=False)
    assert rel_max_err(pp.cpu().numpy(), ref) <= 1e-3


@pytest.mark.parametrize('case', INTERP_CASES, ids=[c[0] for c in INTERP_CASES])
def test_jacobian_and_vjp_with_resampling_match_fp64_finite_differences(case, cuda):
    """The Jacobian (on the resampled samples) through the resampling matrix
    against central differences of the float64 oracle along random
    directions of the input phase (<= 1e-4), and the VJP on the input grid
    consistent with it (<= 1e-5)."""
    c = _setup(case)
    adj, A, lam, pix = c['adj'], c['A'], c['lam'], c['pix']
    rng = np.random.default_rng(11)
    nm_per_rad = lam / (2 * math.pi)
    phase0 = (smooth_field(pix, rng, 0.6) * nm_per_rad * A).astype(np.float32)
    jac = adj.jacobian(torch.as_tensor(A), torch.as_tensor(phase0))
    M = adj.resample_matrix()
    lens = adj._lenslet.cpu().numpy()
    seed = rng.standard_normal(2 * adj.n_valid).astype(np.float32)
    grad = adj.vjp(torch.as_tensor(A), torch.as_tensor(phase0), torch.as_tensor(seed)).cpu().numpy()
    eps = 1e-3
    for probe in range(3):
        delta = smooth_field(pix, np.random.default_rng(200 + probe), 1.0) * nm_per_rad
        d_res = torch.sparse.mm(M, torch.as_tensor(delta.reshape(-1, 1), device='cuda')).cpu().numpy()
        ad = _dir_derivative(jac, lens, c['n'], adj.np_sub, d_res.reshape(adj.field, adj.field))
        p64 = phase0.astype(np.float64)
        fd = (c['slopes64'](p64 + eps * delta) - c['slopes64'](p64 - eps * delta)) / (2 * eps)
        assert rel_max_err(ad, fd) <= ADJ_TOL, probe
        lhs = float((grad.astype(np.float64) * delta).sum())
        rhs = float(seed.astype(np.float64) @ ad)
        assert abs(lhs - rhs) <= VJP_TOL * float(np.abs(seed).astype(np.float64) @ np.abs(ad)), probe


def test_intmat_contract_matches_host_contraction(cuda):
    c = _setup(FLAT_CASES[0])
    adj, A, pix, n = c['adj'], c['A'], c['pix'], c['n']
    dm, IF, mask = _dm(c, 24, seed=9)
    rng = np.random.default_rng(1)
    phase0 = (smooth_field(pix, rng, 60.0) * A).astype(np.float32)
    jac = adj.jacobian(torch.as_tensor(A), torch.as_tensor(phase0))
    im = adj.intmat(torch.as_tensor(A), torch.as_tensor(phase0), dm, jac=jac).cpu().numpy()
    J = jac.cpu().numpy().astype(np.float64)
    col = np.full(pix * pix, -1)
    col[np.flatnonzero(mask.ravel())] = np.arange(IF.shape[1])
    p, nv = adj.np_sub, adj.n_valid
    ref = np.zeros((IF.shape[0], 2 * nv))
    for s, L in enumerate(adj._lenslet.cpu().numpy()):
        li, lj = divmod(int(L), n)
        cc = col.reshape(pix, pix)[li * p:(li + 1) * p, lj * p:(lj + 1) * p].ravel()
        f = np.where(cc[None, :] >= 0, IF[:, np.maximum(cc, 0)], 0.0)
        ref[:, s] = f @ J[0, s]
        ref[:, nv + s] = f @ J[1, s]
    ref *= 2 * dm.sign
    assert rel_max_err(im, ref) <= VJP_TOL


def test_gpu_pushpull_matches_fp64_pushpull(cuda):
    c = _setup(FLAT_CASES[0])
    adj, A, pix = c['adj'], c['A'], c['pix']
    dm, IF, mask = _dm(c, 6, seed=4)
    amp = 10.0
    im, replay = adj.pushpull_intmat(torch.as_tensor(A), dm, amp)
    im2 = replay()                                   # second replay of the captured graph

    def slopes_fn(k, a):
        cmd = np.zeros(IF.shape[0])
        cmd[k] = a
        return c['slopes64'](octl.dm_phase(IF.astype(np.float64), mask, cmd, sign=dm.sign, precision=0))

    ref = octl.pushpull_intmat(slopes_fn, IF.shape[0], [amp] * IF.shape[0])
    # float32 push-pull: the difference of two slope vectors loses digits
    assert rel_max_err(im.cpu().numpy(), ref) <= 1e-3
    assert torch.equal(im, im2)


def test_calibration_system_adjoint_matches_fp64_pushpull_full_size(cuda):
    """The 40x40 / 320 px / FFT 16 / 500-Zernike calibration system: the
    adjoint matrix against the float64 oracle push-pull at a small amplitude
    on every mode (per-mode max|d|/max|ref| <= 1e-4), and against the
    float32 GPU push-pull at 10 nm (which carries its own O(a^2) truncation
    and float32 cancellation)."""
    from specula_b200.calibration import ShCalibrationSystem
    cal = ShCalibrationSystem()
    im = cal.adjoint_intmat().cpu().numpy()
    assert im.shape == (500, 2 * cal.n_valid)
    sh = cal.sh
    g = sh.geometry
    pix = cal.pupil.shape[0]
    geom = osh.sh_geometry(sh._wavelengthInNm, sh._subap_wanted_fov_arcsec, sh._sensor_pxscale_arcsec, g.n_lenses,
                           g.subap_npx, pix, cal.simul_params.pixel_pitch, fov_ovs_coeff=1.0)
    o64 = osh.SHOracle(geom, sh._wavelengthInNm, precision=0)
    A = cal.pupil.astype(np.float64)
    IF = cal.dm._ifunc.influence_function.cpu().numpy().astype(np.float64)
    idxs = cal.subapdata.idxs
    amp = 1e-2

    def s64(k, a):
        cmd = np.zeros(IF.shape[0])
        cmd[k] = a
        ph = octl.dm_phase(IF, cal.pupil, cmd, sign=cal.dm.sign, precision=0)
        return osl.sh_slopes(o64.forward(A, ph, 1.0, cal.simul_params.pixel_pitch), idxs, precision=0)[0]

    # every one of the 500 x 2 n_valid entries: the whole matrix, mode by mode
    mask = cal.pupil > 0
    worst = (0.0, -1)
    for k in range(IF.shape[0]):
        def s64k(a):
            ph = np.zeros(cal.pupil.shape)
            ph[mask] = cal.dm.sign * a * IF[k]
            return osl.sh_slopes(o64.forward(A, ph, 1.0, cal.simul_params.pixel_pitch), idxs, precision=0)[0]
        ref = (s64k(amp) - s64k(-amp)) / amp
        e = rel_max_err(im[k], ref)
        worst = max(worst, (e, k))
        assert e <= ADJ_TOL, k
    print(f'adjoint vs float64 push-pull, all {IF.shape[0]} modes: worst {worst[0]:.2e} (mode {worst[1]})')
    # the GPU push-pull at 10 nm against the float64 push-pull at 10 nm (same
    # O(a^2) truncation, which reaches several percent on high-order modes)
    pp = cal.pushpull_intmat(10.0).cpu().numpy()
    for k in (0, 20, 499):
        ref = (s64(k, 10.0) - s64(k, -10.0)) / 10.0
        assert rel_max_err(pp[k], ref) <= 1e-3, k


def test_im_rec_calibrator_loop_matches_chain_pushpull(cuda):
    """The reference's calibration loop, object by object: FuncGenerator
    ('PUSHPULL') -> DM -> AtmoPropagation -> SH -> CCD (noise off) ->
    ShSlopec -> ImRecCalibrator, against the graph-captured push-pull of
    ShSlopesAdjoint on the same chain and the adjoint matrix."""
    from specula_b200.loop_control import LoopControl
    from specula_b200.processing_objects.func_generator import FuncGenerator
    from specula_b200.processing_objects.dm import DM
    from specula_b200.processing_objects.atmo_propagation import AtmoPropagation
    from specula_b200.processing_objects.sh import SH
    from specula_b200.processing_objects.ccd import CCD
    from specula_b200.processing_objects.sh_slopec import ShSlopec
    from specula_b200.processing_objects.im_rec_calibrator import ImRecCalibrator
    from specula_b200.data_objects.ifunc import IFunc
    from specula_b200.data_objects.pupilstop import Pupilstop
    from specula_b200.data_objects.simul_params import SimulParams
    from specula_b200.data_objects.source import Source
    from specula_b200.data_objects.subap_data import SubapData
    from specula_b200.lib.sh_adjoint import ShSlopesAdjoint
    from specula_b200.scao import valid_subaps
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = FLAT_CASES[0]
    sp = SimulParams(pixel_pupil=pix, pixel_pitch=pitch, time_step=0.001)
    pupil = make_mask(pix, 0.14, 1.0)
    n_modes, amp = 6, 10.0
    rng = np.random.default_rng(21)
    IF = np.stack([smooth_field(pix, rng, 1.0, kmax=4)[pupil > 0] for _ in range(n_modes)]).astype(np.float32)
    func = FuncGenerator('PUSHPULL', nmodes=n_modes, vect_amplitude=[amp] * n_modes, target_device_idx=0)
    dm = DM(sp, 0, ifunc=IFunc(ifunc=IF, mask=pupil, target_device_idx=0), target_device_idx=0)
    dm.inputs['in_command'].set(func.outputs['output'])
    pup = Pupilstop(sp, obs_diam=0.14, target_device_idx=0)
    prop = AtmoPropagation(sp, {'src': Source([0, 0], 8, lam, phot_density_value=50.0)}, target_device_idx=0)
    prop.inputs['common_layer_list'].set([pup, dm.layer])
    sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n, subap_npx=npx,
            fov_ovs_coeff=coeff, target_device_idx=0)
    sh.inputs['in_ef'].set(prop.outputs['out_src_ef'])
    ccd = CCD(sp, size=[n * npx, n * npx], dt=0.001, bandw=300, quantum_eff=0.8, target_device_idx=0)
    ccd.inputs['in_i'].set(sh.outputs['out_i'])
    idxs, dmap = valid_subaps(pupil, n, npx)
    sl = ShSlopec(SubapData(idxs=idxs, display_map=dmap, nx=n, ny=n, target_device_idx=0), target_device_idx=0)
    sl.inputs['in_pixels'].set(ccd.outputs['out_pixels'])
    cal = ImRecCalibrator(nmodes=n_modes, rec_tag='rec', target_device_idx=0)
    cal.inputs['in_slopes'].set(sl.outputs['out_slopes'])
    cal.inputs['in_commands'].set(func.outputs['output'])
    loop = LoopControl()
    for k, obj in enumerate([func, dm, prop, sh, ccd, sl, cal]):
        loop.add(obj, k)
    loop.start(2 * n_modes * 0.001, 0.001)
    for _ in range(2 * n_modes):
        loop.iter()
    loop.finish()
    im_loop = cal.intmat.intmat.cpu().numpy()
    assert cal.rec.recmat.shape == (n_modes, 2 * len(idxs))
    adj = ShSlopesAdjoint(sh, sl)
    A = torch.as_tensor(pupil.astype(np.float32), device='cuda')
    im_pp, _ = adj.pushpull_intmat(A, dm, amp)
    assert rel_max_err(im_loop, im_pp.cpu().numpy()) <= 1e-3
    im_adj = adj.intmat(A, torch.zeros_like(A), dm).cpu().numpy()
    assert rel_max_err(im_loop, im_adj) <= 1e-2       # push-pull carries its O(a^2) truncation at 10 nm


def test_autograd_function_gradient_matches_jacobian(cuda):
    from specula_b200.lib.sh_adjoint import sh_slopes
    c = _setup(FLAT_CASES[1])
    adj, A, pix = c['adj'], c['A'], c['pix']
    rng = np.random.default_rng(12)
    phase0 = torch.as_tensor((smooth_field(pix, rng, 50.0) * A).astype(np.float32), device='cuda')
    At = torch.as_tensor(A, device='cuda')
    w = torch.as_tensor(rng.standard_normal(2 * adj.n_valid).astype(np.float32), device='cuda')
    ph = phase0.clone().requires_grad_(True)
    s = sh_slopes(adj, At, ph)
    (s * w).sum().backward()
    ref = adj.vjp(At, phase0, w)
    assert torch.allclose(ph.grad, ref, rtol=0, atol=1e-6 * float(ref.abs().max()))
    # and the forward equals the processing objects' slopes
    sl_fwd, _ = adj.slopes(At, phase0)
    assert torch.equal(s.detach(), sl_fwd)


def test_tma_contraction_equals_gather_contraction(cuda):
    """sb_intmat_contract_rows (influence functions streamed by TMA) gives
    the matrix of sb_intmat_contract (gathers) bit for bit, on the
    500-Zernike calibration system with the CoG cut-off applied."""
    from specula_b200 import _lib
    from specula_b200.calibration import ShCalibrationSystem
    cal = ShCalibrationSystem()
    adj, dm = cal.adjoint, cal.dm
    assert adj._segments(cal._pix2col, dm._IF, dm._ld) is not None
    im_tma = cal.adjoint_intmat()
    A = cal.A
    jac = adj._jacobian(A, cal._flat, None)
    tot = adj._tot
    im_gather = torch.empty_like(im_tma)
    _lib.call('sb_intmat_contract', jac.data_ptr(), tot.data_ptr(), adj.n_valid, adj.np_sub, adj.n_lenses,
              adj.field, adj._slot.data_ptr(), cal._pix2col.data_ptr(), dm._IF.data_ptr(), dm._IF.shape[0], dm._ld,
              float(2.0 * dm.sign), im_gather.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    _lib.call('sb_device_status')
    assert torch.equal(im_tma, im_gather)
    assert float(im_tma.abs().max()) > 0


def test_tma_contraction_reports_a_short_segment(cuda):
    """A row segment that misses columns under a valid sub-aperture is not
    read past its end: those entries are skipped and sb_device_status reports
    SB_EINVAL (the box itself stays aligned and inside the matrix)."""
    from specula_b200 import _lib
    from specula_b200.calibration import ShCalibrationSystem
    cal = ShCalibrationSystem()
    adj, dm = cal.adjoint, cal.dm
    seg, seg_max = adj._segments(cal._pix2col, dm._IF, dm._ld)
    bad = seg.clone()
    li = int(torch.nonzero(bad[:, 1] > 64)[0])
    bad[li, 1] = 32                                  # 32 columns where the row needs more
    jac = adj._jacobian(cal.A, cal._flat, None)
    im = torch.zeros((dm._IF.shape[0], 2 * adj.n_valid), device=cal.A.device)
    _lib.call('sb_intmat_contract_rows', jac.data_ptr(), adj._tot.data_ptr(), adj.n_valid, adj.np_sub, adj.n_lenses,
              adj.field, adj._slot.data_ptr(), cal._pix2col.data_ptr(), bad.data_ptr(), seg_max, dm._IF.data_ptr(),
              dm._IF.shape[0], dm._ld, float(2.0 * dm.sign), im.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    lib = _lib.load()
    assert lib.sb_device_status() == -1
    assert b'segment' in lib.sb_last_error()
    assert lib.sb_device_status() == 0               # the flag is cleared once read
