"""ShSlopec options on the GPU (sh_slopec.py:48-60 set as attributes, read by
calc_slopes_nofor at every trigger) against the reference's own outputs in
tests/golden/slopec_opt_fp32.npz (make_golden.py --slopec-options): pedestal
threshold, window matrix, multiplication factor, quad-cell weights, a
windowed mask and the per-sub-aperture relative threshold; the Gaussian
weighted mask against the oracle; the time switch of weightedPixRad; the
batched launch; and the fused chain standing aside when an option is on."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import slopec as osl  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402
from tests.test_oracle_golden import SLOPEC_OPT_CASES, slopec_option_kwargs  # noqa: E402

pytestmark = pytest.mark.gpu

ATTRS = {
    'pedestal': dict(thr_pedestal=True),
    'window': dict(winMatWindowed='win'),
    'mult': dict(mult_factor=2.5),
    'quadcell': dict(quadcell_mode=True),
    'windowing': dict(weightedPixRad=2.0, windowing=True),
    'ratio_for0.3': dict(thr_ratio_value=0.3),
    'ratio_for0.6': dict(thr_ratio_value=0.6, winMatWindowed='win'),
}


@pytest.fixture(scope='module')
def opt():
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'slopec_opt_fp32.npz')) as z:
        return {k: z[k] for k in z.files}


def _slopec(golden, thr_value=-1, attrs=None, win=None):
    from specula_b200.processing_objects.sh_slopec import ShSlopec
    from specula_b200.data_objects.subap_data import SubapData
    from specula_b200.data_objects.pixels import Pixels
    ref = golden['ref_fits']
    sd = SubapData(idxs=ref['subaps/idxs'], display_map=ref['subaps/display_map'], nx=8, ny=8, target_device_idx=0)
    sc = ShSlopec(sd, thr_value=thr_value, target_device_idx=0)
    for k, v in (attrs or {}).items():
        setattr(sc, k, win if v == 'win' else v)
    sc.set_xy_weights()
    pix = Pixels(64, 64, target_device_idx=0)
    sc.inputs['in_pixels'].set(pix)
    sc.setup()
    return sc, pix


def _step(sc, pix, frame, t):
    pix.pixels.copy_(torch.as_tensor(frame))
    pix.generation_time = t
    sc.check_ready(t)
    sc.trigger()
    sc.post_trigger()
    return sc.slopes.slopes.cpu().numpy()


@pytest.mark.parametrize('case', list(ATTRS))
def test_option_matches_reference(golden, cuda, opt, case):
    sc, pix = _slopec(golden, SLOPEC_OPT_CASES[case].get('thr_value', -1), ATTRS[case], opt['slopec_opt/window'])
    for t in range(2):
        got = _step(sc, pix, opt['slopec_opt/frame%d' % t], t + 1)
        assert rel_max_err(got, opt['slopec_opt/%s/slopes%d' % (case, t)]) <= 1e-5, (case, t)
    assert sc.options_plain() == (case in ('quadcell', 'windowing'))


def test_gaussian_mask_matches_oracle(golden, cuda, opt):
    """Weighted CoG with the Gaussian mask (FWHM 1 on the [-1, 1] grid)."""
    sc, pix = _slopec(golden, attrs=dict(weightedPixRad=1.0))
    idxs = golden['ref_fits']['subaps/idxs']
    w = osl.xy_weights(8, weighted_pix_rad=1.0)
    for t in range(2):
        got = _step(sc, pix, opt['slopec_opt/frame%d' % t], t + 1)
        ref, _ = osl.sh_slopes(opt['slopec_opt/frame%d' % t], idxs, weights=w)
        assert rel_max_err(got, ref) <= 1e-5


def test_options_change_between_triggers(golden, cuda, opt):
    """The attributes are read at each trigger, as calc_slopes_nofor reads
    them; thr_value with thr_ratio_value raises (sh_slopec.py:326-327)."""
    sc, pix = _slopec(golden, thr_value=10.0)
    idxs = golden['ref_fits']['subaps/idxs']
    f = opt['slopec_opt/frame0']
    a = _step(sc, pix, f, 1)
    assert rel_max_err(a, osl.sh_slopes(f, idxs, thr_value=10.0)[0]) <= 1e-5
    sc.winMatWindowed = opt['slopec_opt/window']
    sc.mult_factor = -1.5
    b = _step(sc, pix, f, 2)
    ref = osl.sh_slopes(f, idxs, thr_value=10.0, win_mat=opt['slopec_opt/window'], mult_factor=-1.5)[0]
    assert rel_max_err(b, ref) <= 1e-5
    sc.thr_ratio_value = 0.2
    with pytest.raises(ValueError, match='thr_ratio_value'):
        _step(sc, pix, f, 3)


def test_weighted_radius_switches_in_time(golden, cuda, opt):
    """vecWeiPixRadT rows (weightedPixRad, start time): the window of the last
    row whose time has passed (sh_slopec.py:136-143)."""
    sc, pix = _slopec(golden, attrs=dict(windowing=True))
    sc.vecWeiPixRadT = np.array([[2.0, 0.0015], [3.0, 0.0035]])
    idxs = golden['ref_fits']['subaps/idxs']
    f = opt['slopec_opt/frame1']
    for t_ms, rad in ((1, 0.0), (2, 2.0), (3, 2.0), (4, 3.0)):
        got = _step(sc, pix, f, t_ms * 1000000)
        w = osl.xy_weights(8, weighted_pix_rad=rad, windowing=True)
        assert rel_max_err(got, osl.sh_slopes(f, idxs, weights=w)[0]) <= 1e-5, t_ms


def test_batched_options_match_single(golden, cuda, opt):
    """sb_slopec_batched with a window and the relative threshold: each
    realisation equals the single-frame launch."""
    import ctypes
    from specula_b200 import _lib
    sc, pix = _slopec(golden, attrs=dict(thr_ratio_value=0.4, winMatWindowed='win', mult_factor=3.0),
                      win=opt['slopec_opt/window'])
    frames = [opt['slopec_opt/frame0'], opt['slopec_opt/frame1'], opt['slopec_opt/frame0'][::-1].copy()]
    single = [_step(sc, pix, f, i + 1) for i, f in enumerate(frames)]
    n = sc._plan.n_subaps
    P = torch.as_tensor(np.stack(frames), device='cuda').contiguous()
    S = torch.zeros(3, 2 * n + 3, device='cuda')
    F = torch.zeros(3, n + 1, device='cuda')
    nb = 3 * _lib.load().sb_slopec_scratch_bytes(ctypes.byref(sc._plan))
    scratch = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.call('sb_slopec_batched', ctypes.byref(sc._plan), P.data_ptr(), 64 * 64, S.data_ptr(), S.stride(0),
              F.data_ptr(), F.stride(0), 3, scratch.data_ptr(), nb, None)
    torch.cuda.synchronize()
    for b in range(3):
        assert np.array_equal(S[b, :2 * n].cpu().numpy(), single[b])


def test_fused_chain_stands_aside_for_options(cuda):
    """The loop's fused SH / detector / slope launch implements thr_value
    only: with a slope option on, the capture keeps the separate launches
    and the step equals the sequential one."""
    from specula_b200.scao import ScaoConfig, ScaoLoop
    loop = ScaoLoop(ScaoConfig(n_modes=8, photon_noise=False, readout_noise=0.0), device_idx=0)
    loop.start()
    loop.step_eager()
    assert loop._can_fuse_chain()
    loop.slopec.thr_pedestal = True
    loop.slopec.thr_value = 1e-3
    assert not loop._can_fuse_chain()
    loop.capture()
    assert not loop.fused_chain
    loop.replay()
    torch.cuda.synchronize()
    s_graph = loop.slopec.slopes.slopes.clone()
    assert torch.isfinite(s_graph).all()
