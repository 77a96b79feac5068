"""GPU parity of the PSF object (sb_strehl, and sb_psf_tc: the two DFT
products on the tensor cores with split-BF16 operands) against the reference
PSF object's outputs (golden fixtures) and the float64 oracle, up to the ELT
field (640 px, nd 8: a 5120 x 5120 PSF).

Tolerances: PSF images max|d|/max|ref| <= 1e-5; Strehl ratios relative
1e-5 against the reference's float32 run and 1e-6 against float64.
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import psf as opsf  # noqa: E402
from oracle.masks import make_mask  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

PSF_TOL = 1e-5
SR_TOL = 1e-5
SR_TOL_FP64 = 1e-6


def _psf(A, lam, nd, start_time):
    from specula_b200.processing_objects.psf import PSF
    from specula_b200.data_objects.electric_field import ElectricField
    pix = A.shape[0]
    ef = ElectricField(pix, pix, 0.05, S0=1.0, target_device_idx=0)
    ef.A.copy_(torch.as_tensor(A))
    p = PSF(wavelengthInNm=lam, nd=nd, start_time=start_time, target_device_idx=0)
    p.inputs['in_ef'].set(ef)
    p.setup()
    return p, ef


def _step(p, ef, phase, t):
    ef.phaseInNm.copy_(torch.as_tensor(phase))
    ef.generation_time = t
    p.check_ready(t)
    p.trigger()
    p.post_trigger()


@pytest.mark.parametrize('pix,nd,lam,t0', [(32, 2, 1650.0, 0.002), (25, 3, 750.0, 0.0)])
def test_psf_matches_reference(golden, cuda, pix, nd, lam, t0):
    g = golden['psf_fp32']
    key = 'psf_%d_%d' % (pix, nd)
    p, ef = _psf(g[key + '/A'], lam, nd, t0)
    for step in range(4):
        _step(p, ef, g[key + '/phase%d' % step], step * 1000000)
        assert rel_max_err(p.psf.value.cpu().numpy(), g[key + '/psf%d' % step]) <= PSF_TOL, step
        sr_ref = float(g[key + '/sr%d' % step])
        assert abs(float(p.sr.value) - sr_ref) <= SR_TOL * abs(sr_ref), step
    assert rel_max_err(p.int_psf.value.cpu().numpy(), g[key + '/int_psf']) <= PSF_TOL
    ref_int = float(g[key + '/int_sr'])
    assert abs(float(p.int_sr.value) - ref_int) <= SR_TOL * abs(ref_int)


def test_psf_and_strehl_against_fp64_at_160px_nd8(cuda):
    pix, nd, lam = 160, 8, 1650.0
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    rng = np.random.default_rng(3)
    p, ef = _psf(A, lam, nd, 0.0)
    o64 = opsf.PSFOracle(A.shape, lam, nd=nd, precision=0)
    for step in range(2):
        ph = (rng.standard_normal((pix, pix)) * 150.0).astype(np.float32) * A
        _step(p, ef, ph, step * 1000000)
        ref, sr64 = o64.step(A, ph, step * 1e-3)
        assert p.psf.value.shape == (1280, 1280)
        assert rel_max_err(p.psf.value.cpu().numpy(), ref) <= PSF_TOL, step
        assert abs(float(p.sr.value) - sr64) <= SR_TOL_FP64 * sr64, step


def test_psf_tensor_cores_at_elt_size_against_fp64(cuda):
    """640 px pupil, nd 8 (5120 x 5120 PSF, the size where the tensor cores
    carry 450 GFLOP of split-BF16 products): PSF within 1e-5 of the float64
    oracle, Strehl within 1e-6, two steps integrated; no device timeout."""
    from specula_b200 import _lib
    pix, nd, lam = 640, 8, 1650.0
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    rng = np.random.default_rng(11)
    p, ef = _psf(A, lam, nd, 0.0)
    o64 = opsf.PSFOracle(A.shape, lam, nd=nd, precision=0)
    acc = None
    for step in range(2):
        ph = (rng.standard_normal((pix, pix)) * 120.0).astype(np.float32) * A
        _step(p, ef, ph, step * 1000000)
        ref, sr64 = o64.step(A, ph, step * 1e-3)
        got = p.psf.value.cpu().numpy()
        assert got.shape == (5120, 5120)
        e = rel_max_err(got, ref)
        print(f'640 px nd 8 step {step}: PSF {e:.2e} of the peak, SR {float(p.sr.value):.6f} vs {sr64:.6f}')
        assert e <= PSF_TOL, step
        assert abs(float(p.sr.value) - sr64) <= SR_TOL_FP64 * sr64, step
        acc = ref.astype(np.float64) if acc is None else acc + ref
    assert rel_max_err(p.int_psf.value.cpu().numpy(), acc) <= PSF_TOL
    _lib.call('sb_device_status')
