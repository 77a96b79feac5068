"""sb_sh_ccd_slopec (SH forward, then normalisation + detector + CoG in one
launch) against the separate calls it replaces (sb_sh_forward or
sb_sh_forward_split_bf16, sb_ccd_step, sb_slopec): the same bits in the
normalised intensity, the integrated frame, the pixels, the slopes, the flux
and the detector frame state, over consecutive frames, with photon and
read-out noise, and with sub-apertures dark enough for the CoG flux cut-off."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu


def _loop(cfg, dft='fp32'):
    from specula_b200.scao import ScaoLoop
    cfg.sh_dft = dft
    loop = ScaoLoop(cfg, device_idx=0)
    loop.start()
    loop.step_eager()
    loop._setup_chain()
    torch.cuda.synchronize()
    return loop


def _state(loop):
    return {'intensity': loop.sh._out_i.i.clone(), 'integrated': loop.ccd._integrated_i.i.clone(),
            'pixels': loop.ccd._pixels.pixels.clone(), 'slopes': loop.slopec.slopes.slopes.clone(),
            'flux': loop.slopec._flux.clone(), 'ccd_state': loop.ccd._state.clone()}


def _restore(loop, st):
    loop.ccd._integrated_i.i.copy_(st['integrated'])
    loop.ccd._pixels.pixels.copy_(st['pixels'])
    loop.ccd._state.copy_(st['ccd_state'])


def _compare(loop, frames, darken=None):
    ef = loop.sh._in_ef
    if darken is not None:
        ef.A.mul_(darken)
    rng = np.random.default_rng(5)
    for f in range(frames):
        ef.phaseInNm.add_(torch.as_tensor(rng.standard_normal(ef.phaseInNm.shape).astype(np.float32) * 30.0,
                                          device=ef.A.device) * ef.A)
        before = _state(loop)
        loop.sh.trigger_code()
        loop.ccd.trigger_code()
        loop.slopec.trigger_code()
        ref = _state(loop)
        _restore(loop, before)
        loop._sh_ccd_slopec()
        got = _state(loop)
        torch.cuda.synchronize()
        for k in ref:
            assert torch.equal(ref[k], got[k]), (f, k)
    from specula_b200 import _lib
    _lib.call('sb_device_status')
    return ref


@pytest.mark.parametrize('dft', ['fp32', 'split_bf16'])
def test_fused_chain_elt_equals_separate_calls(dft, cuda):
    from specula_b200.scao import elt_config
    loop = _loop(elt_config(n_modes=8), dft)
    ref = _compare(loop, 3)
    assert int(ref['ccd_state'][0]) >= 4                     # frames advanced by both paths alike
    assert float(ref['slopes'].abs().max()) > 0


def test_fused_chain_config1_with_cutoff(cuda):
    """20x20 sub-apertures of 8x8 pixels, noise-free detector (read-out noise
    alone would lift a dark sub-aperture's clamped CoG denominator far above
    the cut-off); a few lit lenslets darkened to 1e-4 of their flux so the
    1e-3 * mean cut-off zeroes their slopes."""
    from specula_b200.scao import ScaoConfig
    loop = _loop(ScaoConfig(n_modes=8, photon_noise=False, readout_noise=0.0))
    L = loop.cfg.pixel_pupil
    n = loop.cfg.n_lenses
    dark = torch.ones((L, L), device=loop.device)
    ps = L // n
    lmap = loop.lenslet_subap_map()
    valid = np.flatnonzero(lmap >= 0)
    chosen = valid[[0, len(valid) // 3, len(valid) - 1]]         # three valid lenslets
    for k in chosen:
        i, j = divmod(int(k), n)
        dark[i * ps:(i + 1) * ps, j * ps:(j + 1) * ps] = 1e-2     # amplitude 1e-2: flux 1e-4
    ref = _compare(loop, 2, darken=dark)
    s = ref['slopes'].cpu().numpy()
    nv = s.size // 2
    for k in chosen:
        sub = lmap[k]
        assert s[sub] == 0 and s[nv + sub] == 0, k
