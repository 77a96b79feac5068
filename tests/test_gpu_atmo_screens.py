"""AtmoEvolution's screen sources on the GPU: the reference's FITS cache in
``data_dir`` (written on the first construction, read on the second, same
strips) and a user-defined FITS screen (transposed when wider than tall,
de-meaned, in nm), followed by a step through sb_atmo_evolve_inputs against
the same step on strips held in memory."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _sp(pix=64, pitch=0.01):
    from specula_b200.data_objects.simul_params import SimulParams
    return SimulParams(pixel_pupil=pix, pixel_pitch=pitch, time_step=0.001)


def _step(atmo, n_layers, steps=3):
    from specula_b200.base_value import BaseValue
    vals = [BaseValue(value=v, target_device_idx=0) for v in (0.8, [7.0] * n_layers, [33.0] * n_layers)]
    for k, v in zip(('seeing', 'wind_speed', 'wind_direction'), vals):
        atmo.inputs[k].set(v)
    atmo.setup()
    out = []
    for t in range(steps):
        tt = t * 1000000
        for v in vals:
            v.generation_time = tt
        atmo.check_ready(tt)
        atmo.trigger()
        atmo.post_trigger()
        out.append([layer.phaseInNm.clone() for layer in atmo.layer_list])
    return out


def test_data_dir_cache_round_trip(cuda, tmp_path):
    from specula_b200.processing_objects.atmo_evolution import AtmoEvolution
    from specula_b200.lib.phasescreen_manager import phasescreen_names
    kw = dict(L0=25, heights=[0, 1000, 5000], Cn2=[0.5, 0.3, 0.2], pixel_phasescreens=256, seed=3,
              target_device_idx=0)
    d = str(tmp_path / 'ps')
    a = AtmoEvolution(_sp(), data_dir=d, **kw)
    assert sorted(os.listdir(d)) == [phasescreen_names(3, 256, 0.01, 25.0, 1)[0]]
    b = AtmoEvolution(_sp(), data_dir=d, **kw)           # read back from the file
    for x, y in zip(a.phasescreens, b.phasescreens):
        assert torch.equal(x, y)
    mem = AtmoEvolution(_sp(), data_dir='', **kw)        # float64 synthesis, no file
    for x, y in zip(a.phasescreens, mem.phasescreens):
        assert rel_max_err(x.cpu().numpy(), y.cpu().numpy()) <= 1e-5
    la, lb = _step(a, 3), _step(b, 3)
    for sa, sb in zip(la, lb):
        for x, y in zip(sa, sb):
            assert torch.equal(x, y)


def test_user_defined_screen(cuda, tmp_path):
    from specula_b200.processing_objects.atmo_evolution import AtmoEvolution
    from specula_b200.lib import fits_io
    rng = np.random.default_rng(9)
    scr = rng.standard_normal((66, 300)).astype(np.float32)     # wider than tall: transposed on load
    p = str(tmp_path / 'user.fits')
    fits_io.writeto(p, scr)
    atmo = AtmoEvolution(_sp(), L0=25, heights=[0], Cn2=[1.0], data_dir='', user_defined_phasescreen=p,
                         pixel_phasescreens=256, target_device_idx=0)
    want = scr.T - np.mean(scr.T)
    want = want * np.float32(500.0 / (2 * np.pi))
    got = atmo.phasescreens[0].cpu().numpy()
    assert got.shape == (300, 66)
    assert rel_max_err(got, want) <= 1e-6
    mem = AtmoEvolution(_sp(), L0=25, heights=[0], Cn2=[1.0], data_dir='', pixel_phasescreens=256,
                        target_device_idx=0)
    mem.phasescreens = [atmo.phasescreens[0].clone()]
    mem.phasescreens_sizes = [66]
    for sa, sb in zip(_step(atmo, 1), _step(mem, 1)):
        assert torch.equal(sa[0], sb[0])
    with pytest.raises(ValueError):
        AtmoEvolution(_sp(), L0=25, heights=[0, 1000], Cn2=[0.5, 0.5], data_dir='', user_defined_phasescreen=p,
                      pixel_phasescreens=256, target_device_idx=0)
