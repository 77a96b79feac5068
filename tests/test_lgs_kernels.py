"""Laser-guide-star kernels on CPU (no GPU).

The oracle's sodium-beacon maps and LGS SH frames are pinned to the
reference's own outputs (tests/golden/lgs_fp32.npz, written by
make_golden.py --lgs from the reference SH with a laser launch telescope),
and to the reference's committed golden map (test/data/lgs_map_sh_ref.fits)
with that test's own tolerance (rtol = atol = 1e-5 after normalising).
The library's device-side map, spectra and kernel objects (run here on CPU
tensors) are checked against the oracle and the fixtures.
"""
import numpy as np
import pytest
import torch

from oracle import sh as osh
from tests.cases import lam_over_d_arcsec, rel_max_err

RAD2ASEC = 180 * 3600 / np.pi
LGS = [  # name, pxscale / (lambda/d), launcher, sodium profile, beacon tip-tilt, spot
    ('lgs_gauss', 1.0, [], False, [0.0, 0.0], 1.0),
    ('lgs_elong', 0.5, [4.0, -2.5, 0.0], True, [0.1, -0.05], 0.8),
]


def _case(name, lgs):
    pxf, tel, sod, btt, spot = [c[1:] for c in LGS if c[0] == name][0]
    lam, pix, pitch, n, npx = 589.0, 160, 0.05, 20, 6
    pxs = pxf * lam_over_d_arcsec(lam, pix * pitch / n)
    g = osh.sh_geometry(lam, npx * pxs, pxs, n, npx, pix, pitch, fov_ovs_coeff=1.0)
    ps = lam / 1e9 / (pitch * g.fft_size) * RAD2ASEC
    tt = np.array([0.5, 0.5]) * ps + np.array(btt)
    if sod:
        z, prof = lgs[name + '/sodium_altitude'], lgs[name + '/sodium_intensity']
        args = (n, pitch * pix, tel, 90e3, z - 90e3, prof, spot, ps, g.fft_size)
    else:
        args = (n, pitch * pix, 0.0, 90e3, [0.0], [1.0], spot, ps, g.fft_size)
    return g, args, tt, (lam, pitch, n, ps, spot, tel, sod, btt)


@pytest.mark.parametrize('name', [c[0] for c in LGS])
def test_oracle_matches_reference_lgs_sh(lgs, name):
    g, args, tt, (lam, pitch, n, *_) = _case(name, lgs)
    maps = osh.lgs_map_sh(*args, theta=tt)
    idx = lgs[name + '/kernel_index']
    assert rel_max_err(maps[idx], lgs[name + '/real_kernels']) <= 1e-6
    spec = osh.lgs_kernel_spectra(maps, n).astype(np.complex64)
    out = osh.SHOracle(g, lam, precision=1).forward(lgs[name + '/A'], lgs[name + '/phase'], 7.0, pitch,
                                                    kernels_fft=spec)
    assert rel_max_err(out, lgs[name + '/intensity']) <= 1e-6


def test_oracle_map_matches_reference_fits(lgs):
    """test/test_convolution_kernel.py:test_lgs_map_sh, same parameters and tolerance."""
    z = np.linspace(80e3, 100e3, 20)
    sigma = 10e3 / (2 * np.sqrt(2 * np.log(2)))
    prof = np.exp(-0.5 * ((z - 90e3) / sigma) ** 2)
    prof /= prof.sum()
    m = osh.lgs_map_sh(10, 8.0, [5, 5, 0], 90e3, z - 90e3, prof, 1.0, 0.1, 64)
    total = sum(m[i * 10 + j].sum() for i in range(10) for j in range(10))
    ref_total = float(lgs['lgs_map_sh_ref/sum'])
    for (j, i), blk in zip(lgs['lgs_map_sh_ref/blocks_ji'], lgs['lgs_map_sh_ref/blocks']):
        np.testing.assert_allclose(m[i * 10 + j] / total, blk / ref_total, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize('name', [c[0] for c in LGS])
def test_library_maps_and_kernel_objects_on_cpu(lgs, name, tmp_path):
    from specula_b200.lib.lgs import lgs_map_sh
    from specula_b200.data_objects.convolution_kernel import ConvolutionKernel, GaussianConvolutionKernel
    g, args, tt, (lam, pitch, n, ps, spot, tel, sod, btt) = _case(name, lgs)
    maps = lgs_map_sh(*args, theta=tt, device='cpu')
    idx = lgs[name + '/kernel_index']
    assert rel_max_err(maps.numpy()[idx], lgs[name + '/real_kernels']) <= 1e-6
    if sod:
        k = ConvolutionKernel(dimx=n, dimy=n, pxscale=ps, pupil_size_m=pitch * 160, dimension=g.fft_size,
                              launcher_pos=tel, launcher_size=spot, zfocus=90e3, theta=btt, target_device_idx=-1)
        k.prepare_for_sh(sodium_altitude=lgs[name + '/sodium_altitude'],
                         sodium_intensity=lgs[name + '/sodium_intensity'])
    else:
        k = GaussianConvolutionKernel(dimx=n, dimy=n, pxscale=ps, dimension=g.fft_size, spot_size=spot,
                                      pupil_size_m=pitch * 160, target_device_idx=-1)
        k.prepare_for_sh()
    ref_spec = osh.lgs_kernel_spectra(osh.lgs_map_sh(*args, theta=tt), n)
    assert rel_max_err(k.kernels.numpy(), ref_spec) <= 1e-6
    addr = k.kernels.data_ptr()
    fn = k._kernel_fn
    k.prepare_for_sh()                                  # unchanged parameters: nothing recomputed
    assert k._kernel_fn == fn and k.kernels.data_ptr() == addr
    path = str(tmp_path / 'kern.fits')
    k.save(path)
    r = type(k).restore(path, target_device_idx=-1, return_fft=True)
    assert torch.equal(r.real_kernels, k.real_kernels)
    assert rel_max_err(r.kernels.numpy(), k.kernels.numpy()) <= 1e-7
