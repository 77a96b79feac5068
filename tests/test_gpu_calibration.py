"""The reference's SH calibration sequence (test/test_sh_calibration.py with
params_scao_sh_test{,_subap,_sn,_rec}.yml: 8x8 SH on a 64 px, 1 m pupil,
0.5"/px, 4" field, 600 nm, 40 Zernike modes with 0.1 obstruction, push-pull
at 50 nm, noise-free CCD) run object by object on the GPU, against the
reference's committed result files (scao_subaps_n8_th0.5_ref.fits,
scao_sn_n8_th0.5_ref.fits, scao_rec_n8_th0.5_ref.fits) with the reference
test's own tolerances: sub-aperture table exact, slope nulls to 5 decimals,
reconstructor to 3 decimals.
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu


def _common():
    from specula_b200.data_objects.simul_params import SimulParams
    from specula_b200.data_objects.pupilstop import Pupilstop
    from specula_b200.data_objects.source import Source
    from specula_b200.processing_objects.atmo_propagation import AtmoPropagation
    from specula_b200.processing_objects.sh import SH
    from specula_b200.processing_objects.ccd import CCD
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.015625, time_step=0.001)
    pup = Pupilstop(sp, target_device_idx=0)
    prop = AtmoPropagation(sp, {'on_axis_source': Source([0.0, 0.0], 5, 600, phot_density_value=1e6)},
                           target_device_idx=0)
    sh = SH(wavelengthInNm=600, subap_wanted_fov=4.0, sensor_pxscale=0.5, subap_npx=8, subap_on_diameter=8,
            target_device_idx=0)
    sh.inputs['in_ef'].set(prop.outputs['out_on_axis_source_ef'])
    ccd = CCD(sp, size=[64, 64], dt=0.001, bandw=300, photon_noise=False, readout_noise=False, readout_level=1.0,
              quantum_eff=0.3, target_device_idx=0)
    ccd.inputs['in_i'].set(sh.outputs['out_i'])
    return sp, pup, prop, sh, ccd


def _run(objs, steps):
    from specula_b200.loop_control import LoopControl
    loop = LoopControl()
    for k, o in enumerate(objs):
        loop.add(o, k)
    loop.start(steps * 0.001, 0.001)
    for _ in range(steps):
        loop.iter()
    loop.finish()


def test_subap_calibration_matches_reference_file(golden, cuda):
    from specula_b200.processing_objects.sh_subap_calibrator import ShSubapCalibrator
    sp, pup, prop, sh, ccd = _common()
    prop.inputs['common_layer_list'].set([pup])
    cal = ShSubapCalibrator(subap_on_diameter=8, energy_th=0.5, output_tag='scao_subaps_n8_th0.5',
                            target_device_idx=0)
    cal.inputs['in_i'].set(sh.outputs['out_i'])
    _run([prop, sh, cal], 1)
    ref = golden['ref_fits']
    assert np.array_equal(cal.subaps.idxs, ref['subaps/idxs'])
    assert np.array_equal(cal.subaps.display_map, ref['subaps/display_map'])


def _slopec(ccd, golden):
    from specula_b200.processing_objects.sh_slopec import ShSlopec
    from specula_b200.data_objects.subap_data import SubapData
    ref = golden['ref_fits']
    sd = SubapData(idxs=ref['subaps/idxs'], display_map=ref['subaps/display_map'], nx=8, ny=8, target_device_idx=0)
    sl = ShSlopec(sd, target_device_idx=0)
    sl.inputs['in_pixels'].set(ccd.outputs['out_pixels'])
    return sl


def test_slope_null_calibration_matches_reference_file(golden, cuda):
    from specula_b200.processing_objects.sn_calibrator import SnCalibrator
    sp, pup, prop, sh, ccd = _common()
    prop.inputs['common_layer_list'].set([pup])
    sl = _slopec(ccd, golden)
    cal = SnCalibrator(output_tag='scao_sn_n8_th0.5', target_device_idx=0)
    cal.inputs['in_slopes'].set(sl.outputs['out_slopes'])
    _run([prop, sh, ccd, sl, cal], 1)
    got = cal.slopes.slopes.cpu().numpy()
    np.testing.assert_array_almost_equal(got, golden['ref_fits']['sn/slopes'], decimal=5)


def test_pushpull_reconstructor_matches_reference_file(golden, cuda):
    from specula_b200.processing_objects.func_generator import FuncGenerator
    from specula_b200.processing_objects.dm import DM
    from specula_b200.processing_objects.im_rec_calibrator import ImRecCalibrator
    sp, pup, prop, sh, ccd = _common()
    pp = FuncGenerator('PUSHPULL', nmodes=40, vect_amplitude=[50] * 40, target_device_idx=0)
    dm = DM(sp, 0, type_str='zernike', nmodes=40, npixels=64, obsratio=0.1, sign=1, target_device_idx=0)
    dm.inputs['in_command'].set(pp.outputs['output'])
    prop.inputs['common_layer_list'].set([pup, dm.layer])
    sl = _slopec(ccd, golden)
    cal = ImRecCalibrator(nmodes=40, rec_tag='scao_rec_n8_th0.5', target_device_idx=0)
    cal.inputs['in_slopes'].set(sl.outputs['out_slopes'])
    cal.inputs['in_commands'].set(pp.outputs['output'])
    _run([pp, dm, prop, sh, ccd, sl, cal], 80)
    rec = cal.rec.recmat.cpu().numpy()
    ref = golden['ref_fits']['rec/recmat_T']
    assert rec.shape == ref.shape
    np.testing.assert_array_almost_equal(rec, ref, decimal=3)
