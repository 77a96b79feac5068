"""CCD with b x b binning (sb_ccd_step_binned through the CCD object) against
the CPU oracle's restatement of ccd.py:264-280 (block sums of the
full-resolution frame scaled by b^2 * sum(frame) / sum(blocks), then QE and
background): noise-free frames of two loop steps within 1e-6; with photon
noise the frames are whole ADU steps and their mean follows the noise-free
frame.  (The reference's own binning path cannot run: its integrated frame
gets the binned shape from a tuple repetition in ccd.py:113.)"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle.ccd import CCDOracle  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _ccd(b, **kw):
    from specula_b200.processing_objects.ccd import CCD
    from specula_b200.data_objects.intensity import Intensity
    from specula_b200.data_objects.simul_params import SimulParams
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    c = CCD(sp, size=[48, 48], dt=0.002, bandw=300, quantum_eff=0.8, binning=b, background_noise=True,
            background_level=0.25, target_device_idx=0, **kw)
    ii = Intensity(48, 48, target_device_idx=0)
    c.inputs['in_i'].set(ii)
    c.setup()
    return c, ii


@pytest.mark.parametrize('b', [2, 3])
def test_binned_frames_match_oracle(cuda, b):
    rng = np.random.default_rng(17 + b)
    c, ii = _ccd(b)
    orc = CCDOracle((48, 48), 0.002, 0.001, 300, binning=b, background_noise=True, background_level=0.25,
                    quantum_eff=0.8)
    for t in range(6):
        inten = (rng.random((48, 48)) * 0.2).astype(np.float32)
        ii.i.copy_(torch.as_tensor(inten))
        ii.generation_time = t * 1000000
        c.check_ready(t * 1000000)
        c.trigger()
        c.post_trigger()
        ref = orc.step(inten)
        if ref is not None:
            got = c.outputs['out_pixels'].pixels.cpu().numpy()
            assert got.shape == (48 // b, 48 // b)
            assert rel_max_err(got, ref) <= 1e-6, (b, t)


def test_binned_photon_noise(cuda):
    rng = np.random.default_rng(5)
    inten = (rng.random((48, 48)) * 0.2).astype(np.float32)
    clean, ci = _ccd(2)
    noisy, ni = _ccd(2, photon_noise=True)
    frames = []
    for t in range(40):
        for obj, ii in ((clean, ci), (noisy, ni)):
            ii.i.copy_(torch.as_tensor(inten))
            ii.generation_time = t * 1000000
            obj.check_ready(t * 1000000)
            obj.trigger()
            obj.post_trigger()
        if t % 2 == 1:
            frames.append(noisy.outputs['out_pixels'].pixels.cpu().numpy())
    ref = clean.outputs['out_pixels'].pixels.cpu().numpy().astype(np.float64)
    f = np.array(frames, dtype=np.float64)
    assert np.all(np.abs(f * 8 - np.round(f * 8)) < 1e-6)          # ADU steps of 1/gain
    mean = f.mean(axis=0)
    sigma = np.sqrt(ref / len(frames))
    assert np.mean(np.abs(mean - ref) / sigma) < 1.2               # Poisson mean within its error
