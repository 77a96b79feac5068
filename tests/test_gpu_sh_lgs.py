"""Laser-guide-star SH on the GPU (sb_sh_forward_lgs through the SH object
with a LaserLaunchTelescope) against the reference's own frames
(tests/golden/lgs_fp32.npz, both kernel kinds) and against the float64
oracle; a new sodium profile between steps reaches the captured graph.

Tolerances: intensities max|d|/max <= 1e-5 against the reference FP32 and
float64; kernel maps <= 1e-6."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import sh as osh  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402
from tests.test_lgs_kernels import LGS, _case  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _sh(name, lgs, profile=None):
    from specula_b200.processing_objects.sh import SH
    from specula_b200.data_objects.electric_field import ElectricField
    from specula_b200.data_objects.laser_launch_telescope import LaserLaunchTelescope
    from specula_b200.base_value import BaseValue
    from tests.cases import lam_over_d_arcsec
    pxf, tel, sod, btt, spot = [c[1:] for c in LGS if c[0] == name][0]
    lam, pix, pitch, n, npx = 589.0, 160, 0.05, 20, 6
    pxs = pxf * lam_over_d_arcsec(lam, pix * pitch / n)
    llt = LaserLaunchTelescope(spot_size=spot, tel_position=tel, beacon_focus=90e3, beacon_tt=btt)
    sh = SH(wavelengthInNm=lam, subap_wanted_fov=npx * pxs, sensor_pxscale=pxs, subap_on_diameter=n, subap_npx=npx,
            fov_ovs_coeff=1.0, laser_launch_tel=llt, target_device_idx=0)
    ef = ElectricField(pix, pix, pitch, S0=7.0, target_device_idx=0)
    ef.A.copy_(torch.as_tensor(lgs[name + '/A']))
    ef.phaseInNm.copy_(torch.as_tensor(lgs[name + '/phase']))
    ef.generation_time = 1
    sh.inputs['in_ef'].set(ef)
    vals = None
    if sod:
        vals = (BaseValue(value=torch.as_tensor(lgs[name + '/sodium_altitude'], device='cuda'), target_device_idx=0),
                BaseValue(value=torch.as_tensor(lgs[name + '/sodium_intensity'], device='cuda'), target_device_idx=0))
        for v in vals:
            v.generation_time = 1
        sh.inputs['sodium_altitude'].set(vals[0])
        sh.inputs['sodium_intensity'].set(vals[1])
    sh.setup()
    return sh, ef, vals


def _step(sh, ef, t, vals=None):
    ef.generation_time = t
    if vals is not None:
        for v in vals:
            v.generation_time = t
    sh.check_ready(t)
    sh.trigger()
    sh.post_trigger()
    return sh.outputs['out_i'].i.cpu().numpy()


@pytest.mark.parametrize('name', [c[0] for c in LGS])
def test_lgs_sh_matches_reference_and_fp64(cuda, lgs, name):
    sh, ef, vals = _sh(name, lgs)
    out = [_step(sh, ef, t, vals) for t in (1, 2)]        # eager set-up step, then the captured graph
    ref = lgs[name + '/intensity']
    g, args, tt, (lam, pitch, n, *_) = _case(name, lgs)
    spec = osh.lgs_kernel_spectra(osh.lgs_map_sh(*args, theta=tt), n)
    ref64 = osh.SHOracle(g, lam, precision=0).forward(lgs[name + '/A'].astype(np.float64),
                                                      lgs[name + '/phase'].astype(np.float64), 7.0, pitch,
                                                      kernels_fft=spec)
    for o in out:
        e32, e64 = rel_max_err(o, ref), rel_max_err(o, ref64)
        print(f'{name}: vs reference FP32 {e32:.2e}, vs float64 {e64:.2e}')
        assert e32 <= TOL and e64 <= TOL
    idx = lgs[name + '/kernel_index']
    assert rel_max_err(sh._kernelobj.real_kernels.cpu().numpy()[idx], lgs[name + '/real_kernels']) <= 1e-6
    from specula_b200 import _lib
    _lib.call('sb_device_status')


def test_new_sodium_profile_reaches_the_graph(cuda, lgs):
    name = 'lgs_elong'
    sh, ef, vals = _sh(name, lgs)
    _step(sh, ef, 1, vals)
    _step(sh, ef, 2, vals)
    z = lgs[name + '/sodium_altitude']
    prof = np.exp(-0.5 * ((z - 88e3) / 2e3) ** 2)
    prof /= prof.sum()
    vals[1].value.copy_(torch.as_tensor(prof, device='cuda'))
    got = _step(sh, ef, 3, vals)
    g, args, tt, (lam, pitch, n, ps, spot, tel, sod, btt) = _case(name, lgs)
    args = args[:5] + (prof,) + args[6:]
    spec = osh.lgs_kernel_spectra(osh.lgs_map_sh(*args, theta=tt), n)
    ref64 = osh.SHOracle(g, lam, precision=0).forward(lgs[name + '/A'].astype(np.float64),
                                                      lgs[name + '/phase'].astype(np.float64), 7.0, pitch,
                                                      kernels_fft=spec)
    assert rel_max_err(got, ref64) <= TOL
    assert rel_max_err(got, lgs[name + '/intensity']) > 1e-3     # the profile change is visible


def test_lgs_rejects_split_bf16(cuda):
    from specula_b200.processing_objects.sh import SH
    from specula_b200.data_objects.laser_launch_telescope import LaserLaunchTelescope
    with pytest.raises(ValueError):
        SH(wavelengthInNm=589.0, subap_wanted_fov=2.0, sensor_pxscale=0.3, subap_on_diameter=20, subap_npx=6,
           laser_launch_tel=LaserLaunchTelescope(spot_size=1.0), target_device_idx=0, dft='split_bf16')
