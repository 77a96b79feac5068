"""Detector-structure options of the CCD object on the device (ccd.py:218-262):
EMCCD excess noise and clock-induced charge by their statistics (the draws
come from the device's own counter-based streams), and the deterministic
options against the oracle's restatement: charge-transfer matrices, pixel
gains, a per-pixel QE map with and without its normalisation."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle.ccd import CCDOracle  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

SIDE = 256


def _ccd(side=SIDE, set_attrs=None, **kw):
    from specula_b200.processing_objects.ccd import CCD
    from specula_b200.data_objects.intensity import Intensity
    from specula_b200.data_objects.simul_params import SimulParams
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    c = CCD(sp, size=[side, side], dt=0.001, bandw=1000, target_device_idx=0, **kw)
    for k, v in (set_attrs or {}).items():
        setattr(c, k, v)
    ii = Intensity(side, side, target_device_idx=0)
    c.inputs['in_i'].set(ii)
    c.setup()
    return c, ii


def _frames(c, ii, inten, n):
    out = []
    for t in range(n):
        ii.i.copy_(torch.as_tensor(inten))
        ii.generation_time = t * 1000000
        c.check_ready(t * 1000000)
        c.trigger()
        c.post_trigger()
        out.append(c.outputs['out_pixels'].pixels.cpu().numpy().astype(np.float64))
    from specula_b200 import _lib
    _lib.call('sb_device_status')
    return np.array(out)


@pytest.mark.parametrize('delta', [1.0, 0.5])
def test_emccd_excess_noise_statistics(cuda, delta):
    """Photon noise and EMCCD multiplication (gain 400, ADU gain 1/20 as the
    reference sets them): mean lambda, variance lambda (1 + 1/delta), i.e. the
    excess factor 2 for delta = 1."""
    lam = 20.0
    c, ii = _ccd(photon_noise=True, excess_noise=True, excess_delta=delta)
    assert c._emccd_gain == 400 and abs(c._ADU_gain - 0.05) < 1e-12
    f = _frames(c, ii, np.full((SIDE, SIDE), lam, np.float32), 3)        # rate 1: lambda electrons per frame
    v = f.reshape(-1)
    n = v.size
    assert abs(v.mean() - lam) <= 4 * np.sqrt(lam * (1 + 1 / delta) / n) + 0.01
    ratio = v.var() / lam
    assert abs(ratio - (1 + 1 / delta)) <= 0.05 * (1 + 1 / delta), ratio
    assert (f[0] == f[1]).mean() < 0.05           # each frame draws anew (equal values only by chance)


def test_cic_statistics(cuda):
    """Clock-induced charge: without photon noise every pixel reads lambda or
    lambda + 1 with P(+1) = cic_level; with photon noise on a dark frame the
    mean is cic_level."""
    p = 0.1
    c, ii = _ccd(cic_noise=True, cic_level=p)
    f = _frames(c, ii, np.full((SIDE, SIDE), 3.0, np.float32), 2)
    assert set(np.unique(f)) <= {3.0, 4.0}
    frac = (f == 4.0).mean()
    assert abs(frac - p) <= 4 * np.sqrt(p * (1 - p) / f.size)
    c, ii = _ccd(cic_noise=True, cic_level=p, photon_noise=True)
    f = _frames(c, ii, np.zeros((SIDE, SIDE), np.float32), 2)
    assert abs(f.mean() - p) <= 4 * np.sqrt(2 * p / f.size)


def test_cte_matches_oracle(cuda):
    """Charge-transfer matrices (near-identity smearing along rows and
    columns), background, QE: noise-free frames within 1e-5 of the oracle."""
    side = 96
    rng = np.random.default_rng(3)
    m = np.zeros((side, side, 2), np.float32)
    for k in range(2):
        m[:, :, k] = np.eye(side) * 0.98 + np.eye(side, k=1) * 0.015 + rng.random((side, side)) * 1e-4
    kw = dict(cte_noise=True, cte_mat=m, background_noise=True, background_level=0.5, quantum_eff=0.9)
    c, ii = _ccd(side, **kw)
    orc = CCDOracle((side, side), 0.001, 0.001, 1000, background_noise=True, background_level=0.5,
                    quantum_eff=0.9, cte_mat=m)
    inten = (rng.random((side, side)) * 0.05).astype(np.float32)
    got = _frames(c, ii, inten, 1)[0]
    ref = orc.step(inten)
    assert rel_max_err(got, ref) <= 1e-5
    assert rel_max_err(got, (inten * 0.9 + 0.5)) > 1e-3          # the matrices did act


@pytest.mark.parametrize('normalise', [False, True])
def test_pixel_gains_and_qe_map_match_oracle(cuda, normalise):
    """Pixel gains (set by quadrant) and a per-pixel QE map, with read-out
    noise: the read-out draws differ from the oracle's, so the frames are
    compared noise-free and the read-out noise is checked by its variance."""
    side = 64
    rng = np.random.default_rng(9)
    qe = (0.7 + 0.3 * rng.random((side, side))).astype(np.float32)
    attrs = dict(_notUniformQe=True, _notUniformQeMatrix=qe, _normNotUniformQe=normalise)
    from specula_b200.processing_objects.ccd import CCD  # noqa: F401
    c, ii = _ccd(side, set_attrs=attrs)
    c.setQuadrantGains([1.0, 1.1, 0.9, 1.2])
    c.setup()
    gains = c._pixelGains
    orc = CCDOracle((side, side), 0.001, 0.001, 1000, pixel_gains=gains, qe_map=qe, qe_map_normalise=normalise)
    inten = (rng.random((side, side)) * 0.05).astype(np.float32)
    got = _frames(c, ii, inten, 1)[0]
    ref = orc.step(inten)
    assert rel_max_err(got, ref) <= 1e-6
    # read-out noise scaled by the gains (and the map when normalising)
    c2, ii2 = _ccd(side, set_attrs=attrs, readout_noise=True, readout_level=2.0)
    c2.setQuadrantGains([1.0, 1.1, 0.9, 1.2])
    c2.setup()
    f = _frames(c2, ii2, np.zeros((side, side), np.float32), 8)
    scale = gains / (qe if normalise else 1.0)
    z = (f / scale[None]).reshape(-1)
    assert abs(z.std() - 2.0) <= 0.05 * 2.0


def test_pixel_gains_on_an_integer_frame_are_rejected(cuda):
    with pytest.raises(ValueError, match='integer'):
        _ccd(64, photon_noise=True, pixelGains=np.ones((64, 64), np.float32))


@pytest.mark.parametrize('start_steps, frame_steps', [(3, 2), (4, 1), (5, 3)])
def test_start_time_gates_integration_and_frames(cuda, start_steps, frame_steps):
    """start_time (ccd.py:199-207): nothing integrates before it, and a frame
    closes at step t when (t + 1 - D - S) % D == 0 (S the start and D the
    frame length in steps).  Each frame then equals that of a detector
    started at step 0 and fed the same intensities from step S on."""
    from specula_b200.processing_objects.ccd import CCD
    from specula_b200.data_objects.intensity import Intensity
    from specula_b200.data_objects.simul_params import SimulParams
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    side, n = 32, 14
    rng = np.random.default_rng(start_steps)
    inten = [rng.uniform(0.0, 50.0, (side, side)).astype(np.float32) for _ in range(n)]

    def run(start, feed_from):
        c = CCD(sp, size=[side, side], dt=0.001 * frame_steps, bandw=1000, target_device_idx=0,
                start_time=0.001 * start)
        ii = Intensity(side, side, target_device_idx=0)
        c.inputs['in_i'].set(ii)
        c.setup()
        frames, stamps = [], []
        for t in range(n - feed_from):
            ii.i.copy_(torch.as_tensor(inten[t + feed_from]))
            ii.generation_time = t * 1000000
            c.check_ready(t * 1000000)
            c.trigger()
            c.post_trigger()
            frames.append(c.outputs['out_pixels'].pixels.cpu().numpy().copy())
            stamps.append(c.outputs['out_pixels'].generation_time)
        return frames, stamps

    frames, stamps = run(start_steps, 0)
    ref_frames, _ = run(0, start_steps)
    S, D = start_steps, frame_steps
    closes = [t for t in range(n) if t >= S and (t + 1 - D - S) % D == 0]
    assert closes, 'no frame in the test window'
    for t in range(n):
        done = [c for c in closes if c <= t]
        assert stamps[t] == (done[-1] * 1000000 if done else stamps[0]), t
        if not done:
            assert float(np.abs(frames[t]).max()) == 0.0, t
    for c in closes:
        assert np.array_equal(frames[c], ref_frames[c - S]), c
        assert float(frames[c].max()) > 0
    from specula_b200 import _lib
    _lib.call('sb_device_status')


def test_start_time_off_the_step_grid_is_rejected():
    from specula_b200.processing_objects.ccd import CCD
    from specula_b200.data_objects.simul_params import SimulParams
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    with pytest.raises(NotImplementedError, match='multiple of the time step'):
        CCD(sp, size=[16, 16], dt=0.002, bandw=1000, start_time=0.0015)
    with pytest.raises(NotImplementedError, match="'auto'"):
        CCD(sp, size=[16, 16], dt=0.002, bandw=1000, readout_level='auto', darkcurrent_level=1, background_level=1)
