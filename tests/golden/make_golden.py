"""Generate the golden fixtures under tests/golden/ by running the reference.

Run where a SPECULA source tree is available, naming its root in the
SPECULA_REF environment variable (there is no default location):

    SPECULA_REF=<path to the SPECULA checkout> python tests/golden/make_golden.py

The reference is imported on CPU (``specula.init(-1, precision)``) with the
harness-only stand-ins in tests/golden/_refstubs for astropy.io.fits and
matplotlib (both absent from the image).  Inputs are seeded; every array the
tests compare against is an output of the reference's own code.  The
reference's committed FITS fixtures (test/data/*.fits) are converted to
``ref_fits.npz`` with the small reader in fits_min.py.

Nothing in the test suite, smoke() or bench.py reads the reference at run
time; they only read the .npz/.json files written here.
"""
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get('SPECULA_REF')
if not REF:
    sys.exit('make_golden.py: set SPECULA_REF to the root of a SPECULA source tree')
sys.path.insert(0, os.path.join(HERE, '_refstubs'))
sys.path.insert(0, REF)
sys.path.insert(0, HERE)

import fits_min  # noqa: E402

RAD2ASEC = 180 * 3600 / np.pi


def lam_over_d_arcsec(lam_nm, d_m):
    return lam_nm * 1e-9 / d_m * RAD2ASEC


# (name, pixel_pupil, pitch, lambda_nm, fov_arcsec, pxscale_arcsec, n_lenses, subap_npx, fov_ovs_coeff)
SH_CASES = [
    ('c1_plain16', 160, 0.05, 750.0, 8 * 0.875 * lam_over_d_arcsec(750, 0.4), 0.875 * lam_over_d_arcsec(750, 0.4), 20, 8, 1.0),
    ('c1_interp', 160, 0.05, 750.0, 8 * lam_over_d_arcsec(750, 0.4), lam_over_d_arcsec(750, 0.4), 20, 8, 0.0),
    ('flux120', 120, 0.05, 500.0, 3.0, 0.5, 20, 6, 0.0),
    ('test64', 64, 0.015625, 600.0, 4.0, 0.5, 8, 8, 0.0),
    ('n16_fft32', 128, 0.05, 750.0, 6 * 0.5 * lam_over_d_arcsec(750, 0.4), 0.5 * lam_over_d_arcsec(750, 0.4), 16, 6, 1.0),
    ('n16_fft16', 128, 0.05, 750.0, 6 * lam_over_d_arcsec(750, 0.4), lam_over_d_arcsec(750, 0.4), 16, 6, 1.0),
]

# geometry-only cases (setup is cheap even at ELT size)
GEOM_CASES = SH_CASES + [
    ('c2_fft16', 640, 39.0 / 640, 750.0, 6 * lam_over_d_arcsec(750, 39.0 / 80), lam_over_d_arcsec(750, 39.0 / 80), 80, 6, 1.0),
    ('c2_fft32', 640, 39.0 / 640, 750.0, 6 * 0.5 * lam_over_d_arcsec(750, 39.0 / 80), 0.5 * lam_over_d_arcsec(750, 39.0 / 80), 80, 6, 1.0),
    ('c4_40x40', 320, 0.1, 750.0, 6 * lam_over_d_arcsec(750, 0.8), lam_over_d_arcsec(750, 0.8), 40, 6, 1.0),
    ('c3_74x74', 592, 39.0 / 592, 750.0, 6 * lam_over_d_arcsec(750, 39.0 / 74), lam_over_d_arcsec(750, 39.0 / 74), 74, 6, 1.0),
    ('c3_589nm', 320, 0.1, 589.0, 6 * lam_over_d_arcsec(589, 0.8), lam_over_d_arcsec(589, 0.8), 40, 6, 1.0),
]


def sh_input(pix, seed, amp_nm=60.0):
    """Seeded test field: annular pupil (obs 0.14) and Gaussian random phase."""
    from specula.lib.make_mask import make_mask
    mask = make_mask(pix, 0.14, 1.0, xp=np).astype(np.float32)
    rng = np.random.default_rng(seed)
    phase = (rng.standard_normal((pix, pix)) * amp_nm).astype(np.float32) * mask
    return mask, phase


def make_sh_cases(precision):
    import specula
    from specula.processing_objects.sh import SH
    from specula.data_objects.electric_field import ElectricField
    out = {}
    geoms = {}
    for (name, pix, pitch, lam, fov, pxs, n, npx, coeff) in GEOM_CASES:
        sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n,
                subap_npx=npx, fov_ovs_coeff=coeff, target_device_idx=-1, precision=precision)
        sh._noprints = True
        ef = ElectricField(pix, pix, pitch, S0=1.0, target_device_idx=-1, precision=precision)
        ef.generation_time = 1
        sh.inputs['in_ef'].set(ef)
        sh.set_in_ef(ef)
        sh.calc_trigger_geometry(ef)
        geoms[name] = dict(pix=pix, pitch=pitch, lam=lam, fov=fov, pxscale=pxs, n=n, npx=npx, coeff=coeff,
                           np_sub=int(sh._np_sub), ovs_np_sub=int(sh._ovs_np_sub), fov_ovs=float(sh._fov_ovs),
                           fft_size=int(sh._fft_size), cutpixels=int(sh._cutpixels), cutsize=int(sh._cutsize),
                           fp_mask_sum=int(np.sum(sh._fp_mask)))
    for ci, (name, pix, pitch, lam, fov, pxs, n, npx, coeff) in enumerate(SH_CASES):
        mask, phase = sh_input(pix, seed=100 + ci)
        sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n,
                subap_npx=npx, fov_ovs_coeff=coeff, target_device_idx=-1, precision=precision)
        sh._noprints = True
        ef = ElectricField(pix, pix, pitch, S0=7.0, target_device_idx=-1, precision=precision)
        ef.A[:] = mask
        ef.phaseInNm[:] = phase
        ef.generation_time = 1
        sh.inputs['in_ef'].set(ef)
        sh.setup()
        sh.check_ready(1)
        sh.trigger()
        sh.post_trigger()
        out[name + '/A'] = mask
        out[name + '/phase'] = phase
        out[name + '/intensity'] = np.array(sh.outputs['out_i'].i)
        out[name + '/fp_mask'] = np.array(sh._fp_mask)
    return out, geoms


def make_chain_cases():
    import specula  # noqa: F401
    from specula.processing_objects.sh_slopec import ShSlopec
    from specula.processing_objects.ccd import CCD
    from specula.processing_objects.integrator import Integrator
    from specula.processing_objects.dm import DM
    from specula.processing_objects.modalrec import Modalrec
    from specula.processing_objects.atmo_evolution import AtmoEvolution
    from specula.processing_objects.atmo_propagation import AtmoPropagation
    from specula.processing_objects.sh_subap_calibrator import ShSubapCalibrator
    from specula.data_objects.subap_data import SubapData
    from specula.data_objects.pixels import Pixels
    from specula.data_objects.intensity import Intensity
    from specula.data_objects.ifunc import IFunc
    from specula.data_objects.recmat import Recmat
    from specula.data_objects.slopes import Slopes
    from specula.data_objects.source import Source
    from specula.data_objects.pupilstop import Pupilstop
    from specula.data_objects.simul_params import SimulParams
    from specula.base_value import BaseValue
    out = {}
    rng = np.random.default_rng(7)

    # sub-aperture detection + slopes on a 12x12-lenslet, 6 px detector image
    img = (rng.random((72, 72)) * 50).astype(np.float32)
    img[:6, :6] = 0.0                                # a dark corner sub-aperture
    cal = ShSubapCalibrator(subap_on_diameter=12, energy_th=0.5, data_dir='/tmp', output_tag='x', target_device_idx=-1)
    sd = cal._detect_subaps(img, 0.5)
    out['slopec/image'] = img
    out['slopec/idxs'] = np.array(sd.idxs)
    out['slopec/display_map'] = np.array(sd.display_map)
    sl = ShSlopec(sd, target_device_idx=-1)
    px = Pixels(72, 72, target_device_idx=-1)
    px.pixels = img
    px.generation_time = 1
    sl.inputs['in_pixels'].set(px)
    sl.setup()
    sl.check_ready(1)
    sl.trigger()
    sl.post_trigger()
    out['slopec/slopes'] = np.array(sl.outputs['out_slopes'].slopes)
    out['slopec/flux'] = np.array(sl.flux_per_subaperture_vector.value)

    # CCD: noise-free and noisy (reference RNG) frames
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    inten = (rng.random((48, 48)) * 0.2).astype(np.float32)
    out['ccd/intensity'] = inten
    for tag, kw in (('clean', dict()),
                    ('noisy', dict(photon_noise=True, readout_noise=True, readout_level=3.0)),
                    ('ron_only', dict(readout_noise=True, readout_level=2.0)),
                    ('dt3', dict(dt=0.003))):
        kk = dict(dt=0.001)
        kk.update(kw)
        c = CCD(sp, size=[48, 48], bandw=300, quantum_eff=0.5, target_device_idx=-1, **kk)
        ii = Intensity(48, 48, target_device_idx=-1)
        ii.i[:] = inten
        c.inputs['in_i'].set(ii)
        c.setup()
        frames = []
        for t in range(4):
            tt = t * 1000000
            ii.generation_time = tt
            c.check_ready(tt)
            c.trigger()
            c.post_trigger()
            frames.append(np.array(c.outputs['out_pixels'].pixels, dtype=np.float64))
        out['ccd/' + tag] = np.array(frames)

    # Modalrec + integrator + DM
    nm, ns = 7, 40
    R = rng.standard_normal((nm, ns)).astype(np.float32)
    s = Slopes(slopes=rng.standard_normal(ns).astype(np.float32), target_device_idx=-1)
    s.generation_time = 1
    mr = Modalrec(recmat=Recmat(R, target_device_idx=-1), target_device_idx=-1)
    mr.inputs['in_slopes'].set(s)
    mr.setup()
    mr.check_ready(1)
    mr.trigger()
    mr.post_trigger()
    out['rec/R'] = R
    out['rec/s'] = s.slopes
    out['rec/modes'] = np.array(mr.modes.value)
    gains = rng.random(nm).astype(np.float32)
    integ = Integrator(sp, int_gain=list(gains), delay=2, target_device_idx=-1)
    dc = BaseValue(value=np.zeros(nm, np.float32))
    integ.inputs['delta_comm'].set(dc)
    integ.setup()
    ins, outs = [], []
    for t in range(6):
        dc.value = rng.standard_normal(nm).astype(np.float32)
        dc.generation_time = t
        integ.check_ready(t)
        integ.trigger()
        integ.post_trigger()
        ins.append(dc.value.copy())
        outs.append(np.array(integ.out_comm.value))
    out['iir/gains'] = gains
    out['iir/in'] = np.array(ins)
    out['iir/out'] = np.array(outs)
    pup = Pupilstop(sp, obs_diam=0.14, target_device_idx=-1)
    nv = int(np.sum(pup.A))
    IF = rng.standard_normal((nm, nv)).astype(np.float32)
    dm = DM(sp, 0, ifunc=IFunc(ifunc=IF, mask=pup.A, target_device_idx=-1), target_device_idx=-1)
    cm = BaseValue(value=rng.standard_normal(nm).astype(np.float32))
    cm.generation_time = 1
    dm.inputs['in_command'].set(cm)
    dm.setup()
    dm.check_ready(1)
    dm.trigger()
    dm.post_trigger()
    out['dm/mask'] = np.array(pup.A)
    out['dm/ifunc'] = IF
    out['dm/cmd'] = cm.value
    out['dm/phase'] = np.array(dm.layer.phaseInNm)

    # AtmoEvolution (3 layers, fractional-degree winds) + on-axis AtmoPropagation
    ws = [10.0, 25.0, 7.0]
    wd = [0.0, 123.4, 271.77]
    atmo = AtmoEvolution(sp, L0=25, heights=[0, 1000, 5000], Cn2=[0.5, 0.3, 0.2], data_dir='/tmp/golden_screens',
                         pixel_phasescreens=256, seed=1, target_device_idx=-1)
    see = BaseValue(value=0.8)
    wsv = BaseValue(value=np.array(ws))
    wdv = BaseValue(value=np.array(wd))
    atmo.inputs['seeing'].set(see)
    atmo.inputs['wind_speed'].set(wsv)
    atmo.inputs['wind_direction'].set(wdv)
    src = Source([0, 0], 8, 750)
    prop = AtmoPropagation(sp, {'on_axis_source': src}, target_device_idx=-1)
    prop.inputs['atmo_layer_list'].set(atmo.layer_list)
    prop.inputs['common_layer_list'].set([pup])
    atmo.setup()
    prop.setup()
    out['atmo/strips'] = np.array(atmo.phasescreens)
    layers, efA, efP = [], [], []
    for t in range(4):
        tt = t * 1000000
        for v in (see, wsv, wdv):
            v.generation_time = tt
        atmo.check_ready(tt)
        atmo.trigger()
        atmo.post_trigger()
        prop.check_ready(tt)
        prop.trigger()
        prop.post_trigger()
        layers.append(np.array([np.array(l.phaseInNm) for l in atmo.layer_list]))
        ef = prop.outputs['out_on_axis_source_ef']
        efA.append(np.array(ef.A))
        efP.append(np.array(ef.phaseInNm))
    out['atmo/layers'] = np.array(layers)
    out['atmo/ef_A'] = np.array(efA)
    out['atmo/ef_phase'] = np.array(efP)
    out['atmo/wind_speed'] = np.array(ws)
    out['atmo/wind_direction'] = np.array(wd)
    return out


def convert_ref_fits():
    d = os.path.join(REF, 'test', 'data')
    out = {}
    h = fits_min.read_hdus(os.path.join(d, 'scao_subaps_n8_th0.5_ref.fits'))
    out['subaps/idxs'] = h[1][1].T.astype(np.int64)        # SubapData.restore transposes
    out['subaps/display_map'] = h[2][1].astype(np.int64)
    out['subaps/np_sub'] = np.array(h[0][0]['NP_SUB'])
    h = fits_min.read_hdus(os.path.join(d, 'scao_sn_n8_th0.5_ref.fits'))
    out['sn/slopes'] = np.array(h[1][1], dtype=np.float64)
    h = fits_min.read_hdus(os.path.join(d, 'scao_rec_n8_th0.5_ref.fits'))
    out['rec/recmat_T'] = np.array(h[1][1], dtype=np.float64)
    out['extrapol/mask'] = fits_min.read_hdus(os.path.join(d, 'mask.fits'))[0][1]
    out['extrapol/phase'] = fits_min.read_hdus(os.path.join(d, 'phase.fits'))[0][1]
    out['extrapol/extrapolated1'] = fits_min.read_hdus(os.path.join(d, 'extrapolated1.fits'))[0][1]
    out['extrapol/extrapolated2'] = fits_min.read_hdus(os.path.join(d, 'extrapolated2.fits'))[0][1]
    for flag in ('False', 'True'):
        h = fits_min.read_hdus(os.path.join(d, 'extrapol_array_doExt2Pix%s.fits' % flag))
        out['extrapol/mat1_' + flag] = h[0][1]
        out['extrapol/mat2_' + flag] = h[1][1]
    return out


def convert_interp_fits():
    """The reference's Interp2D fixtures (test/data/input_phase.fits ->
    ref_phase.fits, checked by test_interp2d.py:19-43 at rtol 4e-2), with the
    sampling of that test: make_xy(480, 479.84003 / 2) shifted by the half
    layer (240.5, 240.5) and the position (0.0930127, 0)."""
    d = os.path.join(REF, 'test', 'data')
    return {'interp/input_phase': np.asarray(fits_min.read_hdus(os.path.join(d, 'input_phase.fits'))[0][1],
                                             dtype=np.float32),
            'interp/ref_phase': np.asarray(fits_min.read_hdus(os.path.join(d, 'ref_phase.fits'))[0][1],
                                           dtype=np.float32)}


def make_zernike_cases():
    """IFunc(type_str='zernike') tables (compute_zern_ifunc.py:6-29)."""
    from specula.lib.compute_zern_ifunc import compute_zern_ifunc
    out = {}
    for dim, nz, obs in ZERNIKE_CASES:
        z, m = compute_zern_ifunc(dim, nz, xp=np, dtype=np.float32, obsratio=obs)
        out['zern_%d_%d/ifunc' % (dim, nz)] = z
        out['zern_%d_%d/mask' % (dim, nz)] = m
    return out


ZERNIKE_CASES = [(32, 10, 0.14), (48, 21, 0.0)]

# PSF cases: (pupil px, nd, wavelength nm, start_time s, phase RMS nm)
PSF_CASES = [(32, 2, 1650.0, 0.002, 120.0), (25, 3, 750.0, 0.0, 60.0)]


def make_psf_cases():
    """The reference PSF object (psf.py:17-137) over 4 steps of seeded
    fields: per-step PSF and SR, integrated PSF and SR."""
    from specula.processing_objects.psf import PSF
    from specula.data_objects.electric_field import ElectricField
    out = {}
    for pix, nd, lam, t0, rms in PSF_CASES:
        rng = np.random.default_rng(pix + nd)
        key = 'psf_%d_%d' % (pix, nd)
        ef = ElectricField(pix, pix, 0.05, S0=1.0, target_device_idx=-1)
        A, _ = sh_input(pix, 1)
        ef.A[:] = A
        psf = PSF(wavelengthInNm=lam, nd=nd, start_time=t0, target_device_idx=-1)
        psf.inputs['in_ef'].set(ef)
        psf.setup()
        out[key + '/A'] = A
        for step in range(4):
            ph = (rng.standard_normal((pix, pix)) * rms).astype(np.float32) * A
            ef.phaseInNm[:] = ph
            t = step * 1000000
            ef.generation_time = t
            psf.check_ready(t)
            psf.trigger()
            psf.post_trigger()
            out[key + '/phase%d' % step] = ph
            out[key + '/psf%d' % step] = np.array(psf.psf.value, dtype=np.float32)
            out[key + '/sr%d' % step] = np.float64(psf.sr.value)
        out[key + '/int_psf'] = np.array(psf.int_psf.value, dtype=np.float32)
        out[key + '/int_sr'] = np.float64(psf.int_sr.value)
    return out


# LGS SH cases: (name, pix, pitch, lam, pxscale / (lambda/d), n, npx, spot arcsec, launcher position or [],
#                 sodium altitudes, beacon tip-tilt)
LGS_CASES = [
    ('lgs_gauss', 160, 0.05, 589.0, 1.0, 20, 6, 1.0, [], None, [0.0, 0.0]),
    ('lgs_elong', 160, 0.05, 589.0, 0.5, 20, 6, 0.8, [4.0, -2.5, 0.0], (85e3, 95e3, 7), [0.1, -0.05]),
]


def make_lgs_cases():
    """The reference SH with a laser launch telescope (sh.py:289-321, 382-394):
    Gaussian kernel (no launcher position) and elongated sodium-profile kernel."""
    import tempfile
    from specula.processing_objects.sh import SH
    from specula.data_objects.electric_field import ElectricField
    from specula.data_objects.laser_launch_telescope import LaserLaunchTelescope
    from specula.base_value import BaseValue
    out = {}
    cwd = os.getcwd()
    for ci, (name, pix, pitch, lam, pxf, n, npx, spot, tel, sod, btt) in enumerate(LGS_CASES):
        pxs = pxf * lam_over_d_arcsec(lam, pix * pitch / n)
        mask, phase = sh_input(pix, seed=300 + ci)
        llt = LaserLaunchTelescope(spot_size=spot, tel_position=tel, beacon_focus=90e3, beacon_tt=btt)
        sh = SH(wavelengthInNm=lam, subap_wanted_fov=npx * pxs, sensor_pxscale=pxs, subap_on_diameter=n,
                subap_npx=npx, fov_ovs_coeff=1.0, laser_launch_tel=llt, target_device_idx=-1, precision=1)
        sh._noprints = True
        ef = ElectricField(pix, pix, pitch, S0=7.0, target_device_idx=-1, precision=1)
        ef.A[:] = mask
        ef.phaseInNm[:] = phase
        ef.generation_time = 1
        sh.inputs['in_ef'].set(ef)
        if sod is not None:
            z = np.linspace(sod[0], sod[1], sod[2])
            prof = np.exp(-0.5 * ((z - 90e3) / 3e3) ** 2)
            prof /= prof.sum()
            alt = BaseValue(value=z, target_device_idx=-1)
            inten = BaseValue(value=prof, target_device_idx=-1)
            alt.generation_time = inten.generation_time = 1
            sh.inputs['sodium_altitude'].set(alt)
            sh.inputs['sodium_intensity'].set(inten)
            out[name + '/sodium_altitude'] = z
            out[name + '/sodium_intensity'] = prof
        with tempfile.TemporaryDirectory() as d:
            os.chdir(d)                # the kernel object caches by file name in the working directory
            try:
                sh.setup()
                sh.check_ready(1)
                sh.trigger()
                sh.post_trigger()
            finally:
                os.chdir(cwd)
        out[name + '/A'] = mask
        out[name + '/phase'] = phase
        out[name + '/pxscale'] = np.float64(pxs)
        out[name + '/intensity'] = np.array(sh.outputs['out_i'].i)
        # a spot-check subset of the kernel maps (the full cubes are MBs)
        out[name + '/kernel_index'] = LGS_KERNEL_INDEX
        out[name + '/real_kernels'] = np.array(sh._kernelobj.real_kernels, dtype=np.float32)[LGS_KERNEL_INDEX]
        out[name + '/fft_size'] = np.int64(sh._fft_size)
        out[name + '/cutpixels'] = np.int64(sh._cutpixels)
    # the reference's own golden LGS map (test/test_convolution_kernel.py:test_lgs_map_sh)
    h = fits_min.read_hdus(os.path.join(REF, 'test', 'data', 'lgs_map_sh_ref.fits'))
    ref = np.array(h[0][1], dtype=np.float64)
    out['lgs_map_sh_ref/sum'] = np.float64(ref.sum())
    out['lgs_map_sh_ref/blocks_ji'] = LGS_MAP_BLOCKS
    out['lgs_map_sh_ref/blocks'] = np.stack([ref[j * 64:(j + 1) * 64, i * 64:(i + 1) * 64]
                                             for j, i in LGS_MAP_BLOCKS]).astype(np.float32)
    return out


LGS_KERNEL_INDEX = np.array([0, 7, 19, 133, 210, 399])
LGS_MAP_BLOCKS = np.array([[0, 0], [2, 7], [5, 5], [9, 1], [9, 9]])


# zonal influence functions: (name, dim, n_act, circ_geom, mech coupling, slaving, obsratio)
ZONAL_CASES = [
    ('sq64', 64, 8, False, False, False, 0.0),
    ('circ128_slaved', 128, 8, True, False, True, 0.4),    # test/test_modal_basis.py:test_kl_basis_rms
    ('sq32_coupled', 32, 5, False, True, False, 0.0),
]
# KL bases: (zonal case, diameter, r0, L0, zern_modes, oversampling)
KL_CASES = [('sq64', 8.0, 0.2, 25.0, 0, 2), ('circ128_slaved', 8.0, 0.2, 25.0, 5, 1)]
KL_STORED_MODES = 12


def make_kl_cases():
    """Zonal influence functions (lib/compute_zonal_ifunc.py) and KL bases
    (lib/modal_base_generator.py:make_modal_base_from_ifs_fft) from the reference."""
    from specula.lib.compute_zonal_ifunc import compute_zonal_ifunc
    from specula.lib.modal_base_generator import make_modal_base_from_ifs_fft
    out = {}
    ifs = {}
    for name, dim, n_act, circ, coup, slav, obs in ZONAL_CASES:
        f, m, c = compute_zonal_ifunc(dim, n_act, xp=np, dtype=np.float32, circ_geom=circ, do_mech_coupling=coup,
                                      do_slaving=slav, obsratio=obs, return_coordinates=True)
        ifs[name] = (f, m)
        sel = np.linspace(0, f.shape[0] - 1, min(6, f.shape[0])).astype(int)   # a spot-check subset
        out['zonal/%s/n_act' % name] = np.int64(f.shape[0])
        out['zonal/%s/ifs_index' % name] = sel
        out['zonal/%s/ifs' % name] = np.asarray(f, dtype=np.float32)[sel]
        out['zonal/%s/mask' % name] = np.asarray(m, dtype=np.float32)
        out['zonal/%s/coords' % name] = np.asarray(c, dtype=np.float64)
    for name, diam, r0, L0, nz, ovs in KL_CASES:
        f, m = ifs[name]
        kl, m2c, sv = make_modal_base_from_ifs_fft(m, diam, f, r0, L0, zern_modes=nz, oversampling=ovs, xp=np,
                                                   dtype=np.float32)
        key = 'kl/%s' % name
        out[key + '/n_modes'] = np.int64(kl.shape[0])
        out[key + '/kl_basis'] = np.asarray(kl, dtype=np.float32)[:KL_STORED_MODES]
        out[key + '/m2c'] = np.asarray(m2c, dtype=np.float32)
        out[key + '/S1'] = np.asarray(sv['S1'], dtype=np.float64)
        out[key + '/S2'] = np.asarray(sv['S2'], dtype=np.float64)
    return out


def make_prop_cases():
    """AtmoPropagation with interpolated layers (atmo_propagation.py:104-209): an
    LGS at 90 km (cone effect), an off-axis NGS, layers with a shift, a rotation
    and a magnification, with the pupil stop and a ground layer cropped."""
    from specula.processing_objects.atmo_propagation import AtmoPropagation
    from specula.data_objects.layer import Layer
    from specula.data_objects.pupilstop import Pupilstop
    from specula.data_objects.source import Source
    from specula.data_objects.simul_params import SimulParams
    out = {}
    P, pitch, L = 64, 0.05, 160
    sp = SimulParams(pixel_pupil=P, pixel_pitch=pitch, time_step=0.001)
    rng = np.random.default_rng(77)
    specs = [  # height, shiftXY, rot, magnification, amplitude with zeros
        (0.0, (0.0, 0.0), 0.0, 1.0, False),
        (4000.0, (1.5, -2.0), 0.0, 1.0, False),
        (9000.0, (0.0, 0.0), 10.0, 1.0, False),
        (12000.0, (0.0, 0.0), 0.0, 1.3, True),
    ]
    layers = []
    for k, (h, sh, rot, mag, holes) in enumerate(specs):
        lay = Layer(L, L, pitch, h, shiftXYinPixel=sh, rotInDeg=rot, magnification=mag, target_device_idx=-1,
                    precision=1)
        ph = (rng.standard_normal((L, L)) * 50).astype(np.float32)
        A = np.ones((L, L), np.float32)
        if holes:
            A[rng.random((L, L)) < 0.1] = 0.0
        lay.phaseInNm[:] = ph
        lay.A[:] = A
        out['prop/layer%d/phase' % k] = ph
        out['prop/layer%d/A' % k] = A
        layers.append(lay)
    pup = Pupilstop(sp, mask_diam=1.0, obs_diam=0.14, target_device_idx=-1, precision=1)
    sources = {'lgs': Source([0.0, 0.0], 8.0, 589.0, height=90e3), 'ngs_off': Source([30.0, 45.0], 8.0, 750.0),
               'lgs_off': Source([20.0, -60.0], 8.0, 589.0, height=90e3)}
    prop = AtmoPropagation(sp, sources, target_device_idx=-1, precision=1)
    prop.inputs['atmo_layer_list'].set(layers)
    prop.inputs['common_layer_list'].set([pup])
    for lay in layers:
        lay.generation_time = 1
    pup.generation_time = 1
    prop.setup()
    prop.check_ready(1)
    prop.trigger()
    prop.post_trigger()
    for name in sources:
        ef = prop.outputs['out_%s_ef' % name]
        out['prop/%s/A' % name] = np.array(ef.A, dtype=np.float32)
        out['prop/%s/phase' % name] = np.array(ef.phaseInNm, dtype=np.float32)
    # the layer with holes had its phase at A == 0 set to the mean (in place)
    out['prop/layer3/phase_after'] = np.array(layers[3].phaseInNm, dtype=np.float32)
    out['prop/pupil_A'] = np.array(pup.A, dtype=np.float32)
    return out


# general IIR filters: (name, n filters, num taps, den taps, delay, orders shorter than the taps in row 0)
IIR_CASES = [('taps3x3_d2', 5, 3, 3, 2.0, False), ('taps4x2_d1.5', 4, 4, 2, 1.5, True),
             ('taps8x8_d0', 3, 8, 8, 0.0, False), ('taps1x1_d1', 2, 1, 1, 1.0, False)]


def make_iir_cases():
    """IirFilter (iir_filter.py:100-211) with general filters: the output of
    each of 6 steps of random inputs."""
    from specula.processing_objects.iir_filter import IirFilter
    from specula.data_objects.iir_filter_data import IirFilterData
    from specula.data_objects.simul_params import SimulParams
    from specula.base_value import BaseValue
    out = {}
    rng = np.random.default_rng(5)
    sp = SimulParams(pixel_pupil=8, pixel_pitch=0.1, time_step=0.001)
    for name, n, ni, no, delay, short in IIR_CASES:
        num = rng.standard_normal((n, ni)).astype(np.float32) * 0.5
        den = rng.standard_normal((n, no)).astype(np.float32) * 0.2
        den[:, -1] = 1.0 + np.abs(den[:, -1])
        ordnum = [ni] * n
        ordden = [no] * n
        if short and ni > 2:
            num[0, ni - 1:] = 0.0                 # a row of lower order: right-aligned by set_num
            ordnum[0] = ni - 1
        fd = IirFilterData(ordnum, ordden, num, den, target_device_idx=-1, precision=1)
        filt = IirFilter(sp, fd, delay=delay, target_device_idx=-1, precision=1)
        d = BaseValue(value=np.zeros(n, np.float32), target_device_idx=-1)
        filt.inputs['delta_comm'].set(d)
        filt.setup()
        key = 'iir/%s' % name
        out[key + '/num'], out[key + '/den'] = num, den
        out[key + '/ordnum'], out[key + '/ordden'] = np.array(ordnum), np.array(ordden)
        for t in range(6):
            x = rng.standard_normal(n).astype(np.float32)
            d.value = x.copy()
            d.generation_time = (t + 1) * 1000000
            filt.check_ready((t + 1) * 1000000)
            filt.trigger()
            filt.post_trigger()
            out[key + '/in%d' % t] = x
            out[key + '/out%d' % t] = np.array(filt.out_comm.value, dtype=np.float32)
    return out


def make_slopec_filter_cases(ref):
    """ShSlopec with slope filtering (slopec.py:92-101 through filtmat) on the
    reference's own sub-aperture table (8x8, 52 valid) and random frames."""
    from specula.processing_objects.sh_slopec import ShSlopec
    from specula.data_objects.subap_data import SubapData
    from specula.data_objects.pixels import Pixels
    out = {}
    rng = np.random.default_rng(33)
    idxs = ref['subaps/idxs']
    dmap = ref['subaps/display_map']
    sd = SubapData(idxs=idxs, display_map=dmap, nx=8, ny=8, target_device_idx=-1, precision=1)
    ns = 2 * idxs.shape[0]
    F = rng.standard_normal((2, ns, 6)).astype(np.float32) * 0.1
    sc = ShSlopec(sd, filtmat=F, target_device_idx=-1, precision=1)
    pix = Pixels(64, 64, target_device_idx=-1, precision=1)
    sc.inputs['in_pixels'].set(pix)
    sc.setup()
    out['slopec_filt/filtmat'] = F
    for t in range(2):
        frame = (rng.random((64, 64)) * 100).astype(np.float32)
        pix.pixels[:] = frame
        pix.generation_time = t + 1
        sc.check_ready(t + 1)
        sc.trigger()
        sc.post_trigger()
        out['slopec_filt/frame%d' % t] = frame
        out['slopec_filt/slopes%d' % t] = np.array(sc.slopes.slopes, dtype=np.float32)
    return out


def make_slopec_option_cases(ref):
    """ShSlopec options of calc_slopes_nofor set as attributes after
    construction, as the reference's own code sets them (sh_slopec.py:48-60):
    a pedestal threshold, a window matrix, a multiplication factor, quad-cell
    weights and a windowed mask (weightedPixRad with windowing), on the
    reference's 8x8 sub-aperture table and random frames.  The relative
    threshold (thr_ratio_value) and the Gaussian weighted mask stop with an
    exception in calc_slopes_nofor (sh_slopec.py:376 indexes a scalar, :121
    calls psf_gaussian with three arguments); their raising is recorded here.
    The relative threshold does run in the per-sub-aperture loop
    calc_slopes_for (:150-300, threshold at :231-232): 'ratio_for' holds its
    slopes, on frames where every sub-aperture is bright so that the two
    loops' denominators agree."""
    from specula.processing_objects.sh_slopec import ShSlopec
    from specula.data_objects.subap_data import SubapData
    from specula.data_objects.pixels import Pixels
    out = {}
    rng = np.random.default_rng(41)
    idxs = ref['subaps/idxs']
    dmap = ref['subaps/display_map']
    n, npx2 = idxs.shape
    np_sub = int(round(np.sqrt(npx2)))
    win = (0.5 + rng.random((np_sub, np_sub, n))).astype(np.float32)
    cases = {
        'pedestal': dict(thr_value=30.0, attrs=dict(thr_pedestal=True)),
        'window': dict(thr_value=10.0, attrs=dict(winMatWindowed=win)),
        'mult': dict(attrs=dict(mult_factor=2.5)),
        'quadcell': dict(attrs=dict(quadcell_mode=True), weights=True),
        'windowing': dict(attrs=dict(weightedPixRad=2.0, windowing=True), weights=True),
        'ratio': dict(attrs=dict(thr_ratio_value=0.002)),
        'gaussian': dict(attrs=dict(weightedPixRad=1.0), weights=True),
    }
    out['slopec_opt/window'] = win
    frames = [(rng.random((64, 64)) * 100).astype(np.float32) for _ in range(2)]
    for t, f in enumerate(frames):
        out['slopec_opt/frame%d' % t] = f
    for name, c in cases.items():
        sd = SubapData(idxs=idxs, display_map=dmap, nx=8, ny=8, target_device_idx=-1, precision=1)
        sc = ShSlopec(sd, thr_value=c.get('thr_value', -1), target_device_idx=-1, precision=1)
        for k, v in c['attrs'].items():
            setattr(sc, k, v)
        try:
            if c.get('weights'):
                sc.set_xy_weights()
            pix = Pixels(64, 64, target_device_idx=-1, precision=1)
            sc.inputs['in_pixels'].set(pix)
            sc.setup()
            for t, f in enumerate(frames):
                pix.pixels[:] = f
                pix.generation_time = t + 1
                sc.check_ready(t + 1)
                sc.trigger()
                sc.post_trigger()
                out['slopec_opt/%s/slopes%d' % (name, t)] = np.array(sc.slopes.slopes, dtype=np.float32)
            out['slopec_opt/%s/xweights' % name] = np.array(sc.xweights, dtype=np.float64)
            out['slopec_opt/%s/mask' % name] = np.array(sc.mask_weighted, dtype=np.float64)
        except Exception as e:            # the reference's failure, by exception type
            out['slopec_opt/%s/raises' % name] = np.array(type(e).__name__)
    for ratio in (0.3, 0.6):
        sd = SubapData(idxs=idxs, display_map=dmap, nx=8, ny=8, target_device_idx=-1, precision=1)
        sc = ShSlopec(sd, target_device_idx=-1, precision=1)
        sc.thr_ratio_value = ratio
        sc.winMatWindowed = win if ratio == 0.6 else None
        pix = Pixels(64, 64, target_device_idx=-1, precision=1)
        sc.inputs['in_pixels'].set(pix)
        sc.setup()
        for t, f in enumerate(frames):
            # the loop indexes its frame with the flat sub-aperture indices, as
            # it does the accumulated frame: hand it the flattened frame there
            sc.accumulated_pixels = types.SimpleNamespace(pixels=f.ravel().copy())
            sc.current_time = t + 1
            sc.calc_slopes_for(accumulated=True)
            out['slopec_opt/ratio_for%g/slopes%d' % (ratio, t)] = np.array(sc.accumulated_slopes.slopes,
                                                                          dtype=np.float32)
    return out


def make_polc_cases():
    """Modalrec with POLC (modalrec.py:126-156): pseudo-open-loop slopes
    s + IM c, modes R s - c, without and with a projection matrix, over three
    steps (the first without commands)."""
    from specula.processing_objects.modalrec import Modalrec
    from specula.data_objects.recmat import Recmat
    from specula.data_objects.intmat import Intmat
    from specula.data_objects.slopes import Slopes
    from specula.base_value import BaseValue
    out = {}
    rng = np.random.default_rng(91)
    ns, nm, npj = 40, 12, 9
    R = rng.standard_normal((nm, ns)).astype(np.float32)
    Pm = rng.standard_normal((npj, nm)).astype(np.float32)
    out['polc/R'], out['polc/P'] = R, Pm
    for case, proj in (('plain', None), ('proj', Pm)):
        ncmd = nm if proj is None else npj
        # slopes x commands, as the POLC product IM @ commands uses it
        IM = rng.standard_normal((ns, ncmd)).astype(np.float32)
        out['polc/%s/IM' % case] = IM
        rec = Modalrec(recmat=Recmat(R.copy(), target_device_idx=-1, precision=1),
                       projmat=None if proj is None else Recmat(proj.copy(), target_device_idx=-1, precision=1),
                       intmat=Intmat(IM.copy(), target_device_idx=-1, precision=1), polc=True,
                       target_device_idx=-1, precision=1)
        sl = Slopes(ns, target_device_idx=-1, precision=1)
        cmd = BaseValue(target_device_idx=-1)
        rec.inputs['in_slopes'].set(sl)
        rec.inputs['in_commands'].set(cmd)
        for t in range(3):
            s = rng.standard_normal(ns).astype(np.float32)
            sl.slopes[:] = s
            sl.generation_time = t + 1
            if t > 0:
                c = rng.standard_normal(ncmd).astype(np.float32)
                cmd.value = c.copy()
                cmd.generation_time = t + 1
                out['polc/%s/commands%d' % (case, t)] = c
            if t == 0:
                rec.setup()
            rec.check_ready(t + 1)
            rec.trigger()
            rec.post_trigger()
            out['polc/%s/slopes_in%d' % (case, t)] = s
            out['polc/%s/slopes_after%d' % (case, t)] = np.array(sl.slopes, dtype=np.float32)
            out['polc/%s/modes%d' % (case, t)] = np.array(rec.modes.value, dtype=np.float32)
            out['polc/%s/pol%d' % (case, t)] = np.array(rec.pseudo_ol_modes.value, dtype=np.float32)
    return out


PS_NAME_CASES = [
    # (L0 list, dimension, pixel_pitch, seeds, precision)
    ([25.0], 64, 0.05, [1, 2], 1),
    ([30.5], 100, 0.0609375, [7], 0),
    ([25.0, 40.0], 32, 0.125, [3, 4], 1),
]


def make_ccd_start_cases():
    """The reference CCD with start_time > 0 (ccd.py:199-207): seeded
    intensities per step, frame length 2 and 3 steps, noise-free and with
    photon + read-out noise (its own NumPy generators); per step the output
    frame and its generation time."""
    import specula  # noqa: F401
    from specula.processing_objects.ccd import CCD
    from specula.data_objects.intensity import Intensity
    from specula.data_objects.simul_params import SimulParams
    out = {}
    rng = np.random.default_rng(11)
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.01, time_step=0.001)
    n = 12
    inten = (rng.random((n, 24, 24)) * 0.3).astype(np.float32)
    out['intensity'] = inten
    for tag, kw in (('clean_s3_d2', dict(start_time=0.003, dt=0.002)),
                    ('clean_s4_d3', dict(start_time=0.004, dt=0.003)),
                    ('noisy_s3_d2', dict(start_time=0.003, dt=0.002, photon_noise=True, readout_noise=True,
                                         readout_level=3.0))):
        c = CCD(sp, size=[24, 24], bandw=300, quantum_eff=0.5, target_device_idx=-1, **kw)
        ii = Intensity(24, 24, target_device_idx=-1)
        c.inputs['in_i'].set(ii)
        c.setup()
        frames, stamps = [], []
        for t in range(n):
            ii.i[:] = inten[t]
            tt = t * 1000000
            ii.generation_time = tt
            c.check_ready(tt)
            c.trigger()
            c.post_trigger()
            frames.append(np.array(c.outputs['out_pixels'].pixels, dtype=np.float64))
            stamps.append(c.outputs['out_pixels'].generation_time)
        out[tag + '/frames'] = np.array(frames)
        out[tag + '/stamps'] = np.array(stamps, dtype=np.int64)
    return out


def make_phasescreen_names():
    """File names the reference's phasescreen cache writes
    (lib/phasescreen_manager.py), captured through the harness fits stand-in."""
    import tempfile
    from astropy.io import fits
    from specula.lib.phasescreen_manager import phasescreens_manager
    out = []
    for L0, dim, pitch, seeds, precision in PS_NAME_CASES:
        with tempfile.TemporaryDirectory() as d:
            fits._store.clear()
            phasescreens_manager(np.array(L0), dim, pitch, d, xp=np, precision=precision, seed=np.array(seeds))
            names = [os.path.basename(k) for k in fits._store]
        out.append({'L0': L0, 'dimension': dim, 'pixel_pitch': pitch, 'seeds': seeds, 'precision': precision,
                    'names': names})
    return out


def main():
    import subprocess
    # The reference binds its global precision at import time
    # (base_time_obj.py:1), so the float64 run needs its own process.
    subprocess.run([sys.executable, os.path.abspath(__file__), '--fp64'], check=True)
    import specula
    specula.init(-1, precision=1)
    ref = convert_ref_fits()
    np.savez_compressed(os.path.join(HERE, 'ref_fits.npz'), **ref)
    np.savez_compressed(os.path.join(HERE, 'interp_fits.npz'), **convert_interp_fits())
    sh32, geoms = make_sh_cases(precision=1)
    np.savez_compressed(os.path.join(HERE, 'sh_fp32.npz'), **sh32)
    with open(os.path.join(HERE, 'sh_geometry.json'), 'w') as f:
        json.dump(geoms, f, indent=1, sort_keys=True)
    chain = make_chain_cases()
    np.savez_compressed(os.path.join(HERE, 'chain_fp32.npz'), **chain)
    np.savez_compressed(os.path.join(HERE, 'zernike_fp32.npz'), **make_zernike_cases())
    np.savez_compressed(os.path.join(HERE, 'psf_fp32.npz'), **make_psf_cases())
    with open(os.path.join(HERE, 'phasescreen_names.json'), 'w') as f:
        json.dump(make_phasescreen_names(), f, indent=1)
    np.savez_compressed(os.path.join(HERE, 'lgs_fp32.npz'), **make_lgs_cases())
    np.savez_compressed(os.path.join(HERE, 'kl_fp32.npz'), **make_kl_cases())
    np.savez_compressed(os.path.join(HERE, 'prop_fp32.npz'), **make_prop_cases())
    np.savez_compressed(os.path.join(HERE, 'polc_fp32.npz'), **make_polc_cases())
    np.savez_compressed(os.path.join(HERE, 'iir_fp32.npz'), **make_iir_cases())
    np.savez_compressed(os.path.join(HERE, 'slopec_filt_fp32.npz'), **make_slopec_filter_cases(ref))
    np.savez_compressed(os.path.join(HERE, 'slopec_opt_fp32.npz'), **make_slopec_option_cases(ref))
    np.savez_compressed(os.path.join(HERE, 'ccd_start_fp32.npz'), **make_ccd_start_cases())
    print('wrote', sorted(os.listdir(HERE)))


def main_fp64():
    import specula
    specula.init(-1, precision=0)
    sh64, _ = make_sh_cases(precision=0)
    np.savez_compressed(os.path.join(HERE, 'sh_fp64.npz'),
                        **{k: v for k, v in sh64.items() if k.endswith('/intensity')})


if __name__ == '__main__':
    if '--fp64' in sys.argv:
        main_fp64()
    elif '--psf' in sys.argv:          # only the PSF / Strehl fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'psf_fp32.npz'), **make_psf_cases())
    elif '--slopec-filter' in sys.argv:  # only the slope-filtering fixtures
        import specula
        specula.init(-1, precision=1)
        with np.load(os.path.join(HERE, 'ref_fits.npz')) as z:
            ref = {k: z[k] for k in z.files}
        np.savez_compressed(os.path.join(HERE, 'slopec_filt_fp32.npz'), **make_slopec_filter_cases(ref))
    elif '--slopec-options' in sys.argv:  # only the slope-option fixtures
        import specula
        specula.init(-1, precision=1)
        with np.load(os.path.join(HERE, 'ref_fits.npz')) as z:
            ref = {k: z[k] for k in z.files}
        np.savez_compressed(os.path.join(HERE, 'slopec_opt_fp32.npz'), **make_slopec_option_cases(ref))
    elif '--interp-fits' in sys.argv:  # only the Interp2D FITS fixtures
        np.savez_compressed(os.path.join(HERE, 'interp_fits.npz'), **convert_interp_fits())
    elif '--iir' in sys.argv:          # only the general IIR filter fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'iir_fp32.npz'), **make_iir_cases())
    elif '--polc' in sys.argv:         # only the POLC reconstructor fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'polc_fp32.npz'), **make_polc_cases())
    elif '--prop' in sys.argv:         # only the interpolated-layer propagation fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'prop_fp32.npz'), **make_prop_cases())
    elif '--kl' in sys.argv:           # only the zonal influence functions and KL bases
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'kl_fp32.npz'), **make_kl_cases())
    elif '--lgs' in sys.argv:          # only the LGS SH fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'lgs_fp32.npz'), **make_lgs_cases())
    elif '--psnames' in sys.argv:      # only the phase-screen cache file names
        import specula
        specula.init(-1, precision=1)
        with open(os.path.join(HERE, 'phasescreen_names.json'), 'w') as f:
            json.dump(make_phasescreen_names(), f, indent=1)
    elif '--ccd-start' in sys.argv:    # only the CCD start_time fixtures
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'ccd_start_fp32.npz'), **make_ccd_start_cases())
    elif '--zernike' in sys.argv:      # only the Zernike influence-function tables
        import specula
        specula.init(-1, precision=1)
        np.savez_compressed(os.path.join(HERE, 'zernike_fp32.npz'), **make_zernike_cases())
    else:
        main()
