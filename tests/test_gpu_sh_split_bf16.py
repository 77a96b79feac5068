"""Split-BF16 tensor-core SH (sb_sh_forward_split_bf16) against float64.

The bar for both forms: slopes within 1e-4 (max |d| / max |ref|) and
normalised intensities within 1e-5 of the peak, against an FP64 run of the
reference (measured: split-BF16 about 5e-6 / 1.4e-5, FP32 about 3e-7 /
4e-7; the split operands carry about 2^-16 relative error, twice per DFT
stage).  Inputs: the reference's golden fields of the supported geometries,
and seeded turbulent phases at the 80x80 ELT size (FFT 16 and 32) against
the float64 oracle; the FP32 form at the ELT size is also held against the
float32 oracle.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import sh as osh, slopec as osl  # noqa: E402
from oracle.masks import make_mask  # noqa: E402
from tests.cases import SH_CASES, SH_S0, rel_max_err, lam_over_d_arcsec  # noqa: E402

pytestmark = pytest.mark.gpu

INTENSITY_TOL = 1e-5
SLOPE_TOL = 1e-4

SUPPORTED = ['c1_plain16', 'n16_fft32', 'n16_fft16']


def _sh(case, A, phase, dft, S0=SH_S0):
    from specula_b200.processing_objects.sh import SH
    from specula_b200.data_objects.electric_field import ElectricField
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n, subap_npx=npx,
            fov_ovs_coeff=coeff, target_device_idx=0, dft=dft)
    ef = ElectricField(pix, pix, pitch, S0=S0, target_device_idx=0)
    ef.A.copy_(torch.as_tensor(A))
    ef.phaseInNm.copy_(torch.as_tensor(phase))
    ef.generation_time = 1
    sh.inputs['in_ef'].set(ef)
    sh.setup()
    out = None
    for t in range(2):                 # the second step replays the captured graph
        ef.generation_time = 1 + t
        sh.check_ready(1 + t)
        sh.trigger()
        sh.post_trigger()
        out = sh.outputs['out_i'].i.cpu().numpy()
    return out, sh


def _slopes(frame, n, thr=0.5, flat=None):
    idxs, _ = osl.detect_subaps(flat if flat is not None else frame, n, thr)
    return osl.sh_slopes(frame.astype(np.float64), idxs, precision=0)[0]


@pytest.mark.parametrize('name', SUPPORTED)
def test_split_bf16_matches_reference_fp64(name, golden, cuda):
    case = [c for c in SH_CASES if c[0] == name][0]
    A = golden['sh_fp32'][name + '/A']
    ph = golden['sh_fp32'][name + '/phase']
    out, sh = _sh(case, A, ph, 'split_bf16')
    assert sh.geometry.ovs_np_sub == 8
    ref64 = golden['sh_fp64'][name + '/intensity']
    e_i = rel_max_err(out, ref64)
    n = case[6]
    flat, _ = _sh(case, A, np.zeros_like(ph), 'fp32')
    e_s = rel_max_err(_slopes(out, n, flat=flat), _slopes(ref64, n, flat=flat))
    print(f'{name}: split-BF16 vs reference FP64: intensity {e_i:.2e}, slopes {e_s:.2e}')
    assert e_i <= INTENSITY_TOL
    assert e_s <= SLOPE_TOL
    # photon normalisation is applied after the DFTs, so the total is exact to FP32 rounding
    assert abs(out.sum() / (SH_S0 * case[2] ** 2 * A.sum()) - 1) < 1e-5


def _elt_case(fft=16):
    lamd = lam_over_d_arcsec(750.0, 39.0 / 80)
    pxs = lamd if fft == 16 else 0.5 * lamd
    return ('elt80', 640, 39.0 / 640, 750.0, 6 * pxs, pxs, 80, 6, 1.0)


def _turbulent_phase(pix, seed, rms_rad, lam):
    rng = np.random.default_rng(seed)
    f = np.fft.fftfreq(pix)
    fx, fy = np.meshgrid(f, f)
    psd = (fx ** 2 + fy ** 2 + (1.0 / pix) ** 2) ** (-11.0 / 12.0)
    scr = np.real(np.fft.ifft2(psd * (rng.standard_normal((pix, pix)) + 1j * rng.standard_normal((pix, pix)))))
    scr *= rms_rad / scr.std()
    return (scr * lam / (2 * math.pi)).astype(np.float32)


@pytest.mark.parametrize('fft', [16, 32])
def test_split_bf16_elt_matches_fp64_oracle(fft, cuda):
    """80x80 sub-apertures on 640 px (FFT 16 with cut 4, and FFT 32 with cut 20), a
    seeded turbulent phase of 2 rad RMS: split-BF16 frame and CoG slopes against the
    float64 oracle."""
    case = _elt_case(fft)
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    ph = _turbulent_phase(pix, 11 + fft, 2.0, lam) * A
    out, sh = _sh(case, A, ph, 'split_bf16')
    out32, _ = _sh(case, A, ph, 'fp32')
    g = osh.sh_geometry(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    ref = osh.SHOracle(g, lam, precision=0).forward(A.astype(np.float64), ph.astype(np.float64), SH_S0, pitch)
    flat, _ = _sh(case, A, np.zeros_like(ph), 'fp32')
    s_ref = _slopes(ref, n, flat=flat)
    e_i, e_s = rel_max_err(out, ref), rel_max_err(_slopes(out, n, flat=flat), s_ref)
    e_i32, e_s32 = rel_max_err(out32, ref), rel_max_err(_slopes(out32, n, flat=flat), s_ref)
    ref32 = osh.SHOracle(g, lam, precision=1).forward(A, ph, SH_S0, pitch)
    e_i32o = rel_max_err(out32, ref32)
    e_s32o = rel_max_err(_slopes(out32, n, flat=flat), _slopes(ref32, n, flat=flat))
    print(f'elt80 fft{fft} (cut {sh.geometry.cutsize}): split-BF16 intensity {e_i:.2e} slopes {e_s:.2e}; '
          f'FP32 intensity {e_i32:.2e} slopes {e_s32:.2e} (vs FP32 oracle {e_i32o:.2e} / {e_s32o:.2e})')
    assert e_i <= INTENSITY_TOL
    assert e_s <= SLOPE_TOL
    # the plain FP32 form, the bench's headline SH, at the ELT size
    assert e_i32 <= INTENSITY_TOL
    assert e_s32 <= SLOPE_TOL
    assert e_i32o <= INTENSITY_TOL
    assert e_s32o <= SLOPE_TOL


def test_split_bf16_batched_equals_single(cuda):
    """The batched launch gives every realisation the frame of a single launch, bit for bit."""
    from specula_b200 import _lib
    case = _elt_case(16)
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    _, sh = _sh(case, A, np.zeros_like(A), 'split_bf16')
    B = 3
    dev = torch.device('cuda', 0)
    At = torch.as_tensor(A, device=dev)
    ph = torch.stack([torch.as_tensor(_turbulent_phase(pix, 40 + b, 1.5, lam), device=dev) * At for b in range(B)])
    side = n * npx
    out_b = torch.empty((B, side, side), device=dev)
    nbytes = _lib.load().sb_sh_scratch_bytes(sh._plan)
    scratch = torch.zeros(nbytes * B, dtype=torch.uint8, device=dev)
    from specula_b200.processing_objects.sh import C_plan
    plan = C_plan(sh._plan)
    scale = SH_S0 * pitch ** 2
    _lib.call('sb_sh_forward_split_bf16_batched', plan, At.data_ptr(), 0, ph.data_ptr(), pix * pix, At.data_ptr(), 0,
              pix * pix, scale, out_b.data_ptr(), side * side, B, scratch.data_ptr(), scratch.numel(), 0)
    for b in range(B):
        one = torch.empty((side, side), device=dev)
        _lib.call('sb_sh_forward_split_bf16', plan, At.data_ptr(), ph[b].data_ptr(), At.data_ptr(), pix * pix, scale,
                  one.data_ptr(), scratch.data_ptr(), nbytes, 0)
        torch.cuda.synchronize()
        assert torch.equal(one, out_b[b])
    _lib.call('sb_device_status')


def test_split_bf16_rejects_unsupported_geometry(cuda):
    case = [c for c in SH_CASES if c[0] == 'flux120'][0]     # 6 phase px per sub-aperture
    A = np.ones((case[1], case[1]), np.float32)
    with pytest.raises(ValueError, match='split-BF16'):
        _sh(case, A, np.zeros_like(A), 'split_bf16')
