"""ctypes binding of libspecula_b200.so (the C ABI in include/specula_b200.h).

The library is built in-tree by ``specula_b200/csrc/build.py``.  There is no
CPU fallback: if the library is missing or cannot be loaded, every GPU entry
point raises ``RuntimeError`` naming the file it looked for.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libspecula_b200.so')

SB_OK = 0
STATUS_NAMES = {0: 'SB_OK', -1: 'SB_EINVAL', -2: 'SB_ESHAPE', -3: 'SB_ECUDA', -4: 'SB_ESCRATCH',
                -5: 'SB_ETIMEOUT', -6: 'SB_EUNSUPPORTED'}
SB_MAX_LAYERS = 16
SB_SH_STATIC_SCRATCH_BYTES = 64 * 1024

vp = C.c_void_p
fp = C.c_void_p   # device float*
ip = C.c_void_p   # device int32*


class ShPlan(C.Structure):
    _fields_ = [('n_lenses', C.c_int), ('np_sub', C.c_int), ('cutsize', C.c_int), ('subap_npx', C.c_int),
                ('field_ld', C.c_int), ('phase_to_rad', C.c_float),
                ('twiddle', fp), ('tilt', fp), ('fp_mask', fp), ('rebin', fp)]


class ShLgsTables(C.Structure):
    _fields_ = [('fft_size', C.c_int), ('w_full_t', vp), ('w_dft', vp), ('v_inv_t', vp), ('kernel_spectra', vp)]


class PropSampling(C.Structure):
    _fields_ = [('A', fp), ('phase', fp), ('ld', C.c_int), ('rows', C.c_int), ('cols', C.c_int), ('top', C.c_int),
                ('left', C.c_int), ('yy', fp), ('xx', fp)]


class CcdParams(C.Structure):
    _fields_ = [('n_pixels', C.c_int), ('frames_per_read', C.c_int), ('rate', C.c_float), ('qe', C.c_float),
                ('bg_plus_dark', C.c_float), ('photon_noise', C.c_int), ('readout_noise', C.c_int),
                ('readout_level', C.c_float), ('adu_gain', C.c_float), ('adu_bias', C.c_float),
                ('dark_level', C.c_float), ('dark_noise', C.c_int), ('photon_seed', C.c_uint64),
                ('readout_seed', C.c_uint64), ('state', vp),
                ('cic_noise', C.c_int), ('cic_level', C.c_float), ('excess_noise', C.c_int),
                ('excess_delta', C.c_float), ('emccd_gain', C.c_float), ('excess_seed', C.c_uint64),
                ('pixel_gains', fp), ('qe_map', fp), ('qe_map_normalise', C.c_int)]


class SlopecPlan(C.Structure):
    _fields_ = [('n_subaps', C.c_int), ('npx2', C.c_int), ('thr', C.c_float),
                ('idxs', ip), ('xw', fp), ('yw', fp), ('mw', fp),
                ('thr_pedestal', C.c_int), ('thr_ratio', C.c_float), ('window', fp), ('mult', C.c_float)]


class IirPlan(C.Structure):
    _fields_ = [('n', C.c_int), ('total', C.c_int), ('shift', C.c_int), ('k_out', C.c_int),
                ('rem', C.c_float), ('one_minus_rem', C.c_float),
                ('num', fp), ('den', fp), ('ist', fp), ('ost', fp), ('state', fp), ('out_next', fp),
                ('n_num', C.c_int), ('n_den', C.c_int)]


class AtmoLayer(C.Structure):
    _fields_ = [('screen', fp), ('screen_ld', C.c_int), ('screen_cols', C.c_int), ('delta', C.c_double),
                ('rot90', C.c_int), ('rotate', C.c_int),
                ('m00', C.c_double), ('m01', C.c_double), ('m10', C.c_double), ('m11', C.c_double),
                ('off0', C.c_double), ('off1', C.c_double), ('scale', C.c_float), ('out', fp)]


class AtmoInputs(C.Structure):
    _fields_ = [('seeing', vp), ('wind_speed', vp), ('wind_direction', vp), ('n_wind_speed', C.c_int),
                ('n_wind_direction', C.c_int), ('delta_time', C.c_double), ('pixel_pitch', C.c_double),
                ('pixel_pitch_f', C.c_float), ('airmass_pow', C.c_float), ('lambda_factor', C.c_float)]


class AtmoLayerInputs(C.Structure):
    _fields_ = [('seeing', vp), ('wind_speed', vp), ('wind_direction', vp), ('position', vp)]


class PropLayer(C.Structure):
    _fields_ = [('A', fp), ('phase', fp), ('ld', C.c_int), ('top', C.c_int), ('left', C.c_int)]


SB_MC_MAX_GROUPS = 8
SB_MC_LAUNCHES = 6


class McGroup(C.Structure):
    _fields_ = [('n_batch', C.c_int), ('n_atm', C.c_int), ('L', C.c_int),
                ('layers', C.POINTER(AtmoLayer)), ('inputs', C.POINTER(AtmoLayerInputs)), ('constants', AtmoInputs),
                ('atm', fp), ('atm_real_stride', C.c_longlong), ('stop_A', fp), ('stop_phase', fp), ('dm_A', fp),
                ('dm_phase', fp), ('dm_stride', C.c_longlong), ('field_A', fp), ('field_phase', fp),
                ('field_stride', C.c_longlong),
                ('sh', ShPlan), ('dft_mode', C.c_int), ('photon_scale', C.c_float),
                ('intensity', fp), ('integrated', fp), ('pixels', fp), ('frame_stride', C.c_longlong),
                ('ccd', CcdParams), ('photon_seeds', vp), ('readout_seeds', vp),
                ('slopec', SlopecPlan), ('lenslet_subap', ip), ('slopes', fp), ('slopes_stride', C.c_int),
                ('flux', fp), ('flux_stride', C.c_int),
                ('R', fp), ('n_modes', C.c_int), ('n_slopes', C.c_int), ('ldr', C.c_int), ('modes', fp),
                ('iir', IirPlan), ('commands', fp),
                ('ifunc', fp), ('n_valid', C.c_int), ('ld_if', C.c_int), ('mask_idx', ip), ('dm_sign', C.c_float),
                ('dm_phase_alt', fp), ('commands_next', fp)]


SB_MC_ATMO, SB_MC_SH, SB_MC_CHAIN, SB_MC_REC, SB_MC_DM = range(5)


# name -> (restype, argtypes); every function of include/specula_b200.h
SIGNATURES = {
    'sb_version': (C.c_int, []),
    'sb_mc_workspace_bytes': (C.c_size_t, [C.POINTER(McGroup), C.c_int]),
    'sb_mc_create': (C.c_int, [C.POINTER(McGroup), C.c_int, vp, C.c_size_t, C.POINTER(vp), vp]),
    'sb_mc_step': (C.c_int, [vp, vp]),
    'sb_mc_destroy': (None, [vp]),
    'sb_mc_stage': (C.c_int, [vp, C.c_int, C.c_int, vp]),
    'sb_sh_rows_parts': (C.c_int, [C.POINTER(ShPlan), C.c_int]),
    'sb_sh_forward_rows': (C.c_int, [C.POINTER(ShPlan), C.c_int, C.c_int, C.c_int, fp, fp, fp, C.c_int, fp, vp,
                                     C.c_size_t, vp]),
    'sb_ccd_slopec_rows': (C.c_int, [C.POINTER(ShPlan), fp, C.c_int, C.c_float, C.c_int, C.c_int, fp,
                                     C.POINTER(CcdParams), fp, fp, C.POINTER(SlopecPlan), ip, fp, fp, fp, vp]),
    'sb_slopec_cutoff': (C.c_int, [fp, fp, fp, C.c_int, fp, vp]),
    'sb_last_error': (C.c_char_p, []),
    'sb_sh_scratch_bytes': (C.c_size_t, [C.POINTER(ShPlan)]),
    'sb_sh_forward': (C.c_int, [C.POINTER(ShPlan), fp, fp, fp, C.c_int, C.c_float, fp, vp, C.c_size_t, vp]),
    'sb_sh_forward_static': (C.c_int, [C.POINTER(ShPlan), fp, fp, fp, C.c_int, C.c_float, fp, vp]),
    'sb_edge_extrapolate': (C.c_int, [fp, ip, ip, C.c_int, fp, vp]),
    'sb_interp2d_field': (C.c_int, [fp, fp, C.c_int, C.c_int, fp, fp, C.c_int, fp, fp, vp]),
    'sb_ccd_step': (C.c_int, [C.POINTER(CcdParams), fp, fp, fp, vp]),
    'sb_ccd_cte_scratch_bytes': (C.c_size_t, [C.c_int]),
    'sb_ccd_step_cte': (C.c_int, [C.POINTER(CcdParams), C.c_int, fp, fp, fp, fp, fp, vp, C.c_size_t, vp]),
    'sb_philox_raw': (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, vp, vp]),
    'sb_slopec_scratch_bytes': (C.c_size_t, [C.POINTER(SlopecPlan)]),
    'sb_slopec': (C.c_int, [C.POINTER(SlopecPlan), fp, fp, fp, vp, C.c_size_t, vp]),
    'sb_sh_ccd_slopec_scratch_bytes': (C.c_size_t, [C.POINTER(ShPlan), C.c_int]),
    'sb_sh_ccd_slopec': (C.c_int, [C.POINTER(ShPlan), C.c_int, fp, fp, fp, C.c_int, fp, fp, fp, fp, C.c_float, fp,
                                   C.POINTER(CcdParams), fp, fp, C.POINTER(SlopecPlan), ip, fp, fp, vp,
                                   C.c_size_t, vp]),
    'sb_modalrec': (C.c_int, [fp, C.c_int, C.c_int, C.c_int, fp, fp, vp]),
    'sb_integrator': (C.c_int, [C.POINTER(IirPlan), fp, fp, vp]),
    'sb_modalrec_integrator': (C.c_int, [fp, C.c_int, C.c_int, C.c_int, fp, fp, C.POINTER(IirPlan), fp, vp]),
    'sb_dm_project': (C.c_int, [fp, C.c_int, C.c_int, C.c_int, fp, C.c_int, C.c_float, ip, fp, vp]),
    'sb_device_status': (C.c_int, []),
    'sb_atmo_evolve_batched': (C.c_int, [C.POINTER(AtmoLayer), C.POINTER(AtmoLayerInputs), C.c_int, C.c_int,
                                         C.POINTER(AtmoInputs), vp, C.c_size_t, vp]),
    'sb_propagate_batched': (C.c_int, [fp, C.c_int, C.c_longlong, C.c_longlong, fp, fp, fp, fp, C.c_longlong, C.c_int,
                                       C.c_int, fp, fp, C.c_longlong, vp]),
    'sb_atmo_propagate_batched': (C.c_int, [C.POINTER(AtmoLayer), C.POINTER(AtmoLayerInputs), C.c_int, C.c_int,
                                            C.c_int, C.POINTER(AtmoInputs), vp, C.c_size_t, fp, fp, fp, fp,
                                            C.c_longlong, fp, fp, C.c_longlong, vp]),
    'sb_sh_forward_batched': (C.c_int, [C.POINTER(ShPlan), fp, C.c_longlong, fp, C.c_longlong, fp, C.c_longlong,
                                        C.c_int, C.c_float, fp, C.c_longlong, C.c_int, vp, C.c_size_t, vp]),
    'sb_sh_split_bf16_supported': (C.c_int, [C.POINTER(ShPlan)]),
    'sb_sh_forward_split_bf16': (C.c_int, [C.POINTER(ShPlan), fp, fp, fp, C.c_int, C.c_float, fp, vp, C.c_size_t, vp]),
    'sb_sh_forward_split_bf16_batched': (C.c_int, [C.POINTER(ShPlan), fp, C.c_longlong, fp, C.c_longlong, fp,
                                                   C.c_longlong, C.c_int, C.c_float, fp, C.c_longlong, C.c_int, vp,
                                                   C.c_size_t, vp]),
    'sb_sh_lgs_supported': (C.c_int, [C.POINTER(ShPlan), C.c_int]),
    'sb_sh_forward_lgs': (C.c_int, [C.POINTER(ShPlan), C.POINTER(ShLgsTables), fp, fp, fp, C.c_int, C.c_float, fp,
                                    vp, C.c_size_t, vp]),
    'sb_propagate': (C.c_int, [C.POINTER(PropSampling), C.c_int, C.c_int, fp, fp, vp]),
    'sb_tune_variants': (C.c_int, [C.c_int]),
    'sb_tune_variant_name': (C.c_char_p, [C.c_int, C.c_int]),
    'sb_tune_key': (C.c_ulonglong, [C.c_int, C.c_int, C.c_int]),
    'sb_tune_set': (C.c_int, [C.c_int, C.c_ulonglong, C.c_int]),
    'sb_tune_get': (C.c_int, [C.c_int, C.c_ulonglong]),
    'sb_ccd_binned_scratch_bytes': (C.c_size_t, [C.c_int, C.c_int, C.c_int]),
    'sb_ccd_step_binned': (C.c_int, [C.POINTER(CcdParams), C.c_int, C.c_int, C.c_int, fp, fp, fp, vp, C.c_size_t, vp]),
    'sb_ccd_step_batched': (C.c_int, [C.POINTER(CcdParams), vp, vp, C.c_int, fp, fp, fp, vp]),
    'sb_slopec_batched': (C.c_int, [C.POINTER(SlopecPlan), fp, C.c_longlong, fp, C.c_int, fp, C.c_int, C.c_int, vp,
                                    C.c_size_t, vp]),
    'sb_dm_project_batched': (C.c_int, [fp, C.c_int, C.c_int, C.c_int, fp, C.c_int, C.c_int, C.c_float, ip, fp,
                                        C.c_longlong, vp]),
    'sb_modalrec_batched': (C.c_int, [fp, C.c_int, C.c_int, C.c_int, fp, C.c_int, C.c_int, fp, C.c_int, vp]),
    'sb_atmo_evolve': (C.c_int, [C.POINTER(AtmoLayer), C.c_int, C.c_int, vp, vp]),
    'sb_atmo_work_bytes': (C.c_size_t, [C.c_int]),
    'sb_atmo_evolve_inputs': (C.c_int, [C.POINTER(AtmoLayer), C.c_int, C.c_int, vp, C.POINTER(AtmoInputs), vp,
                                        C.c_size_t, vp]),
    'sb_propagate_on_axis': (C.c_int, [C.POINTER(PropLayer), C.c_int, C.c_int, fp, fp, vp]),
    'sb_psf_scratch_bytes': (C.c_size_t, []),
    'sb_strehl': (C.c_int, [fp, fp, C.c_int, C.c_float, fp, vp, C.c_int, vp, C.c_size_t, vp]),
    'sb_psf_field': (C.c_int, [fp, fp, C.c_int, C.c_float, vp, vp]),
    'sb_psf_finish': (C.c_int, [vp, C.c_longlong, fp, fp, vp, C.c_size_t, vp]),
    'sb_psf_tc_dft_bytes': (C.c_size_t, [C.c_int, C.c_int]),
    'sb_psf_tc_prepare': (C.c_int, [C.c_int, C.c_int, vp, C.c_size_t, vp]),
    'sb_psf_tc_scratch_bytes': (C.c_size_t, [C.c_int, C.c_int]),
    'sb_psf_tc': (C.c_int, [fp, fp, C.c_int, C.c_int, C.c_float, vp, fp, fp, vp, C.c_size_t, vp]),
    'sb_sh_slopes_jacobian': (C.c_int, [C.POINTER(ShPlan), fp, fp, C.c_int, ip, fp, fp, fp, fp, fp, fp, vp]),
    'sb_sh_slopes_vjp': (C.c_int, [C.POINTER(ShPlan), fp, fp, C.c_int, ip, fp, fp, fp, fp, fp, fp, vp]),
    'sb_intmat_contract': (C.c_int, [fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, fp, C.c_int, C.c_int,
                                     C.c_float, fp, vp]),
    'sb_intmat_contract_rows': (C.c_int, [fp, fp, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, ip, C.c_int, fp,
                                          C.c_int, C.c_int, C.c_float, fp, vp]),
    'sb_intmat_lenslet_ifunc': (C.c_int, [fp, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_int, ip, fp,
                                          vp]),
    'sb_intmat_contract_lenslets': (C.c_int, [fp, fp, C.c_int, C.c_int, fp, C.c_int, C.c_float, fp, vp]),
}

_lib = None


# tunable kernel families (specula_b200.h)
SB_TUNE_DM_BATCHED = 0
SB_TUNE_SH_FP32 = 1
SB_TUNE_MODALREC_BATCHED = 2


def load():
    """Load the library (once) and bind every exported symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'specula_b200 CUDA library not found at {LIB_PATH}; '
                           'build it with `python specula_b200/csrc/build.py` (there is no CPU fallback)')
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def call(name, *args):
    """Call an entry point; raise RuntimeError with the library's message on failure."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != SB_OK:
        msg = lib.sb_last_error().decode(errors='replace')
        raise RuntimeError(f'{name} failed with {STATUS_NAMES.get(rc, rc)}: {msg}')
    return rc


def ptr(t):
    """Device address of a torch tensor (None -> NULL)."""
    return None if t is None else t.data_ptr()
