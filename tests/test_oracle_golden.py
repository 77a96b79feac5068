"""The oracle is pinned against the reference: golden vectors produced by
running SPECULA itself (tests/golden/make_golden.py) and the reference's own
committed FITS fixtures (test/data/*.fits, converted to ref_fits.npz)."""
import os

import numpy as np
import pytest

import oracle
from oracle import sh as osh, slopec as osl, ccd as occd, control as octl, atmo as oatm
from oracle.masks import make_mask
from tests.cases import SH_CASES, SH_S0, rel_max_err


def _oracle_sh(case, precision, golden):
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    g = osh.sh_geometry(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    A = golden['sh_fp32'][name + '/A']
    ph = golden['sh_fp32'][name + '/phase']
    o = osh.SHOracle(g, lam, ef_A_for_tables=A, precision=precision)
    dt = np.float32 if precision == 1 else np.float64
    return o.forward(A.astype(dt), ph.astype(dt), SH_S0, pitch), g


@pytest.mark.parametrize('case', SH_CASES, ids=[c[0] for c in SH_CASES])
def test_sh_fp32_matches_reference(case, golden):
    out, g = _oracle_sh(case, 1, golden)
    ref = golden['sh_fp32'][case[0] + '/intensity']
    assert out.dtype == np.float32 and out.shape == ref.shape
    # bit-exact on the machine that generated the fixtures; 1e-6 allows a
    # different CPU's FFT vectorisation
    assert rel_max_err(out, ref) <= 1e-6


@pytest.mark.parametrize('case', SH_CASES, ids=[c[0] for c in SH_CASES])
def test_sh_fp64_matches_reference(case, golden):
    out, _ = _oracle_sh(case, 0, golden)
    ref = golden['sh_fp64'][case[0] + '/intensity']
    assert rel_max_err(out, ref) <= 1e-12


@pytest.mark.parametrize('case', SH_CASES, ids=[c[0] for c in SH_CASES])
def test_sh_geometry_matches_reference(case, golden):
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    g = osh.sh_geometry(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    ref = golden['geometry'][name]
    for k in ('np_sub', 'ovs_np_sub', 'fft_size', 'cutpixels', 'cutsize'):
        assert getattr(g, k) == ref[k], k
    assert g.fov_ovs == ref['fov_ovs']
    m = make_mask(g.fft_size, diaratio=g.fp_diaratio, square=True)
    assert int(m.sum()) == ref['fp_mask_sum']
    assert np.array_equal(m, golden['sh_fp32'][name + '/fp_mask'])


def test_slopec_matches_reference(golden):
    c = golden['chain_fp32']
    idxs, dmap = osl.detect_subaps(c['slopec/image'], 12, 0.5)
    assert np.array_equal(idxs, c['slopec/idxs'])
    assert np.array_equal(dmap, c['slopec/display_map'])
    s, flux = osl.sh_slopes(c['slopec/image'], idxs)
    assert rel_max_err(s, c['slopec/slopes']) <= 1e-6
    assert rel_max_err(flux, c['slopec/flux']) <= 1e-6


@pytest.mark.parametrize('tag,kw', [('clean', {}),
                                    ('noisy', dict(photon_noise=True, readout_noise=True, readout_level=3.0)),
                                    ('ron_only', dict(readout_noise=True, readout_level=2.0)),
                                    ('dt3', dict(dt_s=0.003))])
def test_ccd_matches_reference(golden, tag, kw):
    c = golden['chain_fp32']
    kk = dict(dt_s=0.001)
    kk.update(kw)
    o = occd.CCDOracle((48, 48), loop_dt_s=0.001, bandw=300, quantum_eff=0.5, **kk)
    ref = c['ccd/' + tag]
    last = None
    for t in range(4):
        f = o.step(c['ccd/intensity'])
        last = f if f is not None else last
        if last is not None:
            # the reference keeps its last frame between read-outs
            np.testing.assert_allclose(np.asarray(last, dtype=np.float64), ref[t], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize('tag,start,kw', [('clean_s3_d2', 3, dict(dt_s=0.002)),
                                          ('clean_s4_d3', 4, dict(dt_s=0.003)),
                                          ('noisy_s3_d2', 3, dict(dt_s=0.002, photon_noise=True,
                                                                  readout_noise=True, readout_level=3.0))])
def test_ccd_start_time_matches_reference(tag, start, kw):
    """The oracle's start_time gate and read-out rule (ccd.py:199-207)
    against the reference CCD run with start_time > 0
    (tests/golden/ccd_start_fp32.npz): the frame held at every step and the
    steps at which frames close."""
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'ccd_start_fp32.npz')) as z:
        g = {k: z[k] for k in z.files}
    o = occd.CCDOracle((24, 24), loop_dt_s=0.001, bandw=300, quantum_eff=0.5, **kw)
    frames, stamps = g[tag + '/frames'], g[tag + '/stamps']
    held, when = np.zeros((24, 24)), -1
    for t in range(len(frames)):
        f = o.step_at(g['intensity'][t], t, start)
        if f is not None:
            held, when = np.asarray(f, dtype=np.float64), t * 1000000
        assert stamps[t] == when, t
        np.testing.assert_allclose(held, frames[t], rtol=1e-6, atol=1e-6)
    assert when > 0


def test_integrator_matches_reference(golden):
    c = golden['chain_fp32']
    o = octl.IntegratorOracle(c['iir/gains'], delay=2)
    for t in range(len(c['iir/in'])):
        assert np.array_equal(o.step(c['iir/in'][t]), c['iir/out'][t])


def test_modalrec_and_dm_match_reference(golden):
    c = golden['chain_fp32']
    assert rel_max_err(octl.modalrec(c['rec/R'], c['rec/s']), c['rec/modes']) <= 1e-6
    ph = octl.dm_phase(c['dm/ifunc'], c['dm/mask'], c['dm/cmd'])
    assert rel_max_err(ph, c['dm/phase']) <= 1e-6


def test_atmo_matches_reference(golden):
    c = golden['chain_fp32']
    strips = [s for s in c['atmo/strips']]
    ev = oatm.AtmoEvolutionOracle(strips, 64, 0.01, precision=1)
    pup = c['dm/mask']
    for t in range(4):
        layers = ev.step(t * 1000000, 0.8, c['atmo/wind_speed'], c['atmo/wind_direction'])
        for k in range(3):
            assert rel_max_err(layers[k], c['atmo/layers'][t][k]) <= 1e-6
        A, P = oatm.propagate_on_axis([np.ones((64, 64), np.float32)] * 3 + [pup.astype(np.float32)],
                                      layers + [np.zeros((64, 64), np.float32)], 64)
        assert np.array_equal(A, c['atmo/ef_A'][t])
        assert rel_max_err(P, c['atmo/ef_phase'][t]) <= 1e-6


def test_phasescreen_strips_match_reference(golden):
    c = golden['chain_fp32']
    sq = [oatm.calc_phasescreen(np.array([25])[0], 256, 0.01, seed=1, precision=1)]
    strips = oatm.prepare_strips(sq, 3, 64, [0.5, 0.3, 0.2], precision=1)
    for a, b in zip(strips, c['atmo/strips']):
        assert rel_max_err(a, b) <= 1e-5


def test_extrapolation_tables_match_reference_fits(golden):
    r = golden['ref_fits']
    for flag, two in (('False', False), ('True', True)):
        s1, s2, idx1, idx2 = osh.extrapol_tables(r['extrapol/mask'], do_ext_2_pix=two)
        assert np.array_equal(s1, r['extrapol/mat1_' + flag].astype(np.int32))
        assert np.array_equal(s2, r['extrapol/mat2_' + flag].astype(np.int32))
        out = osh.extrapolate_edge(r['extrapol/phase'], s1, s2, idx1, idx2)
        ref = r['extrapol/extrapolated1' if not two else 'extrapol/extrapolated2']
        np.testing.assert_array_almost_equal(out, ref)


def _calibration_image():
    """Flat-wavefront SH image of the reference's SCAO SH test configuration
    (test/params_scao_sh_test.yml: 64 px, 8x8 lenslets, 8 px, 4", 0.5"/px,
    600 nm, CCD with QE 0.3, bandwidth 300 nm, noise off)."""
    pup = make_mask(64, 0.0, 1.0).astype(np.float32)
    g = osh.sh_geometry(600.0, 4.0, 0.5, 8, 8, 64, 0.015625)
    o = osh.SHOracle(g, 600.0, ef_A_for_tables=pup, precision=1)
    inten = o.forward(pup, np.zeros_like(pup), 1e4, 0.015625)
    ccd = occd.CCDOracle((64, 64), 0.001, 0.001, 300, quantum_eff=0.3)
    return ccd.step(inten)


def test_subaps_match_reference_calibration_fits(golden):
    r = golden['ref_fits']
    frame = _calibration_image()
    idxs, dmap = osl.detect_subaps(frame, 8, 0.5)
    assert np.array_equal(idxs, r['subaps/idxs'])
    assert np.array_equal(dmap, r['subaps/display_map'])


def test_slope_nulls_match_reference_calibration_fits(golden):
    r = golden['ref_fits']
    frame = _calibration_image()
    s, _ = osl.sh_slopes(frame, r['subaps/idxs'])
    np.testing.assert_array_almost_equal(s, r['sn/slopes'], decimal=5)


@pytest.mark.parametrize('pix,nd,lam,t0', [(32, 2, 1650.0, 0.002), (25, 3, 750.0, 0.0)])
def test_psf_oracle_matches_reference(golden, pix, nd, lam, t0):
    """oracle.psf against the reference PSF object over 4 steps: per-step PSF
    and Strehl, integrated PSF and Strehl after start_time."""
    from oracle.psf import PSFOracle
    g = golden['psf_fp32']
    key = 'psf_%d_%d' % (pix, nd)
    A = g[key + '/A']
    o = PSFOracle(A.shape, lam, nd=nd, start_time=t0)
    for step in range(4):
        psf, sr = o.step(A, g[key + '/phase%d' % step], step * 1e-3)
        np.testing.assert_allclose(psf, g[key + '/psf%d' % step], rtol=1e-5, atol=1e-7 * float(psf.max()))
        assert abs(sr - float(g[key + '/sr%d' % step])) <= 1e-5 * abs(float(g[key + '/sr%d' % step]))
    np.testing.assert_allclose(o.int_psf, g[key + '/int_psf'], rtol=1e-5, atol=1e-7 * float(o.int_psf.max()))
    assert abs(o.int_sr - float(g[key + '/int_sr'])) <= 1e-5 * abs(float(g[key + '/int_sr']))


SLOPEC_OPT_CASES = {
    'pedestal': dict(thr_value=30.0, thr_pedestal=True),
    'window': dict(thr_value=10.0, win=True),
    'mult': dict(mult_factor=2.5),
    'quadcell': dict(weights=dict(quadcell_mode=True)),
    'windowing': dict(weights=dict(weighted_pix_rad=2.0, windowing=True)),
    'ratio_for0.3': dict(thr_ratio_value=0.3),
    'ratio_for0.6': dict(thr_ratio_value=0.6, win=True),
}


def slopec_option_kwargs(case, opt):
    """Oracle keyword arguments of one slope-option case of slopec_opt_fp32.npz."""
    c = dict(SLOPEC_OPT_CASES[case])
    kw = {k: c[k] for k in ('thr_value', 'thr_pedestal', 'mult_factor', 'thr_ratio_value') if k in c}
    if c.get('win'):
        kw['win_mat'] = opt['slopec_opt/window']
    if 'weights' in c:
        kw['weights'] = osl.xy_weights(8, **c['weights'])
    return kw


@pytest.fixture(scope='module')
def slopec_opt():
    import os
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'slopec_opt_fp32.npz')) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize('case', list(SLOPEC_OPT_CASES))
def test_slopec_options_match_reference(golden, slopec_opt, case):
    """Pedestal threshold, window matrix, multiplication factor, quad-cell
    weights, a windowed mask (calc_slopes_nofor) and the relative threshold
    (calc_slopes_for) on the reference's 8x8 sub-aperture table."""
    idxs = golden['ref_fits']['subaps/idxs']
    kw = slopec_option_kwargs(case, slopec_opt)
    for t in range(2):
        s, _ = osl.sh_slopes(slopec_opt['slopec_opt/frame%d' % t], idxs, **kw)
        assert rel_max_err(s, slopec_opt['slopec_opt/%s/slopes%d' % (case, t)]) <= 2e-6, (case, t)
    if 'weights' in SLOPEC_OPT_CASES[case]:
        xw, _, mw = kw['weights']
        assert np.array_equal(xw, slopec_opt['slopec_opt/%s/xweights' % case])
        assert np.array_equal(mw, slopec_opt['slopec_opt/%s/mask' % case])


def test_slopec_option_cases_the_reference_raises_on(slopec_opt):
    """The relative threshold and the Gaussian weighted mask raise in the
    reference's calc_slopes_nofor / computeXYweights (an index into a scalar,
    a three-argument call of a two-argument method); the oracle computes the
    per-sub-aperture form and the Gaussian of psf_gaussian instead (parity for
    the Gaussian mask is by construction only)."""
    assert str(slopec_opt['slopec_opt/ratio/raises']) == 'IndexError'
    assert str(slopec_opt['slopec_opt/gaussian/raises']) == 'TypeError'
    x, y, m = osl.xy_weights(8, weighted_pix_rad=1.0)
    v = np.linspace(-1, 1, 8)
    g = np.exp(-4 * np.log(2) * (v[None, :] ** 2 + v[:, None] ** 2))
    assert np.allclose(m, g / g.max(), rtol=1e-6)
    assert m.max() == 1.0 and np.allclose(x, np.meshgrid(v, v)[0] * m)


def _interp_fits_case():
    import os
    from specula_b200.lib.make_mask import make_xy
    from specula_b200.lib.interp2d import interp_coords_xy
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'interp_fits.npz')) as z:
        phase, ref = z['interp/input_phase'], z['interp/ref_phase']
    # the sampling of the reference's test_interp2d.py:25-33
    xx, yy = make_xy(480, 479.84003 / 2.0)
    yy, xx = interp_coords_xy(phase.shape, yy + 240.5 + 0.0, xx + 240.5 + 0.0930127)
    return phase, ref, yy, xx


def test_interp2d_matches_reference_fits():
    """The reference's Interp2D fixture (test_interp2d.py:19-43, 482^2 ->
    480^2 with a sub-pixel shift) at the reference test's tolerance (rtol
    4e-2, its one known outlier pixel excepted)."""
    phase, ref, yy, xx = _interp_fits_case()
    got = osh.interp2d(phase, yy, xx, ref.shape)
    got[394, 365] = ref[394, 365]
    np.testing.assert_allclose(got, ref, rtol=4e-2)
