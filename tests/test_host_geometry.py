"""Host-side logic of the product (no GPU): geometry solve, the device
tables of the pruned-DFT SH kernel, edge-extrapolation tables and
interpolation coordinates, each checked against the reference's goldens or
the oracle."""
import math

import numpy as np
import pytest

from oracle import sh as osh
from specula_b200.lib import sh_geometry as shg
from specula_b200.lib.edge_extrapolation import extrapolation_tables, per_pixel_tables
from specula_b200.lib.interp2d import interp_coords
from specula_b200.lib.make_mask import make_mask
from tests.cases import SH_CASES, SH_S0, rel_max_err


def test_geometry_matches_reference_for_every_config(golden):
    for name, ref in golden['geometry'].items():
        g = shg.solve(ref['lam'], ref['fov'], ref['pxscale'], ref['n'], ref['npx'], ref['pix'], ref['pitch'],
                      fov_ovs_coeff=ref['coeff'])
        assert (g.np_sub, g.ovs_np_sub, g.fft_size, g.cutpixels, g.cutsize) == \
            (ref['np_sub'], ref['ovs_np_sub'], ref['fft_size'], ref['cutpixels'], ref['cutsize']), name
        assert g.fov_ovs == ref['fov_ovs'], name
        m = make_mask(g.fft_size, diaratio=g.fp_diaratio, square=True)
        assert int(m.sum()) == ref['fp_mask_sum'], name


def test_literal_config1_geometry_is_uncut():
    """16x16 FFT onto an 8x8 detector (the literal config 1): cutpixels == 0,
    which the reference cannot slice; here it means 'no cut'."""
    lamd = 750e-9 / 0.4 * 180 * 3600 / math.pi
    g = shg.solve(750, 8 * lamd, lamd, 20, 8, 160, 0.05, fov_ovs_coeff=1.0)
    assert (g.fft_size, g.cutpixels, g.cutsize) == (16, 0, 16)


def test_geometry_rejects_indivisible_field():
    with pytest.raises(ValueError):
        shg.solve(750, 3.0, 0.5, 7, 6, 100, 0.05, fov_ovs_coeff=1.0)


def _emulate_kernel(A, phase, g, lam, S0, pitch):
    """NumPy emulation of sh_forward_kernel + sh_normalize_kernel with the
    product's device tables (no interpolation geometries)."""
    p, n, cs, npx = g.ovs_np_sub, g.n_lenses, g.cutsize, g.subap_npx
    W = shg.twiddle_table(p, g.fft_size, g.cutpixels).astype(np.complex128)
    T = shg.tilt_table(p, g.fft_size).astype(np.complex128)
    M = shg.field_stop_cut(g).astype(np.float64)
    R = shg.rebin_table(cs, npx).astype(np.float64)
    k = float(np.float32(2 * math.pi / lam))
    out = np.zeros((n * npx, n * npx))
    for i in range(n):
        for j in range(n):
            a = A[i * p:(i + 1) * p, j * p:(j + 1) * p].astype(np.float64)
            ph = phase[i * p:(i + 1) * p, j * p:(j + 1) * p].astype(np.float64)
            E = a * np.exp(1j * ph * k) * T
            F = W @ E @ W.T
            I = np.abs(F) ** 2 * M
            out[i * npx:(i + 1) * npx, j * npx:(j + 1) * npx] = R @ I @ R.T
    return out * (S0 * pitch ** 2 * A.sum() / out.sum())


@pytest.mark.parametrize('case', [c for c in SH_CASES if c[8] == 1.0], ids=lambda c: c[0])
def test_pruned_dft_tables_reproduce_reference(case, golden):
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    g = shg.solve(lam, fov, pxs, n, npx, pix, pitch, fov_ovs_coeff=coeff)
    A = golden['sh_fp32'][name + '/A']
    ph = golden['sh_fp32'][name + '/phase']
    em = _emulate_kernel(A, ph, g, lam, SH_S0, pitch)
    ref64 = golden['sh_fp64'][name + '/intensity']
    assert rel_max_err(em, ref64) <= 1e-6


def test_rebin_table_is_lcm_area_rebin():
    for cs, npx in ((12, 6), (14, 8), (26, 6), (16, 8), (8, 8), (7, 3)):
        R = shg.rebin_table(cs, npx).astype(np.float64)
        img = np.random.default_rng(cs * 10 + npx).random((cs, cs))
        ref = osh.toccd(img, (npx, npx))
        got = R @ img @ R.T
        # R is stored in float32 (e.g. 1/7 rounded), hence the 1e-6 tolerance
        np.testing.assert_allclose(got / got.sum() * img.sum(), ref, rtol=1e-6, atol=1e-12)


def test_extrapolation_tables_match_reference_fits(golden):
    r = golden['ref_fits']
    for flag, two in (('False', False), ('True', True)):
        s1, s2 = extrapolation_tables(r['extrapol/mask'], do_ext_2_pix=two)
        assert np.array_equal(s1, r['extrapol/mat1_' + flag].astype(np.int32))
        assert np.array_equal(s2, r['extrapol/mat2_' + flag].astype(np.int32))
        t1, t2 = per_pixel_tables(s1, s2)
        ph = r['extrapol/phase'].ravel()          # float32, like the kernel
        two_ = np.float32(2)
        out = np.where(t1 < 0, ph, np.where(t2 < 0, ph[np.maximum(t1, 0)],
                                            two_ * ph[np.maximum(t1, 0)] - ph[np.maximum(t2, 0)]))
        ref = r['extrapol/extrapolated2' if two else 'extrapol/extrapolated1']
        np.testing.assert_array_almost_equal(out.reshape(ref.shape), ref)


def test_interp_coords_match_oracle():
    for shape_in, shape_out, rot, sh in (((64, 64), (128, 128), 0, (0, 0)), ((120, 120), (240, 240), 0, (0, 0)),
                                         ((40, 40), (80, 80), 3.0, (1, -2))):
        a = interp_coords(shape_in, shape_out, rot, *sh)
        b = osh.interp2d_coords(shape_in, shape_out, rot, *sh)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_time_conversion_matches_reference():
    from specula_b200.base_time_obj import BaseTimeObj
    t = BaseTimeObj(target_device_idx=-1)
    for s, ns in ((0.001, 1000000), (1.0, 1000000000), (0.0015, 1500000), (2.5e-4, 250000), (0.1, 100000000)):
        assert t.seconds_to_t(s) == ns
        assert t.t_to_seconds(ns) == ns / 1e9


@pytest.mark.parametrize('dim,nz,obs', [(32, 10, 0.14), (48, 21, 0.0)])
def test_zernike_ifunc_matches_reference(golden, dim, nz, obs):
    """specula_b200.lib.zernike against the reference's compute_zern_ifunc
    output (bit-exact: same float64 evaluation, float32 QR)."""
    from specula_b200.lib.zernike import compute_zern_ifunc
    z, m = compute_zern_ifunc(dim, nz, obsratio=obs)
    ref = golden['zernike_fp32']
    assert np.array_equal(m, ref['zern_%d_%d/mask' % (dim, nz)])
    assert np.array_equal(z, ref['zern_%d_%d/ifunc' % (dim, nz)])
