"""Shack-Hartmann modal calibration system on the B200: pupil, SH, ShSlopec
and a modal DM, wired for interaction-matrix measurement.

It is the calibration half of the reference's SCAO setup (the objects a
``params_scao_sh*_calib`` run builds: FuncGenerator('PUSHPULL') -> DM ->
AtmoPropagation -> SH -> CCD (noise off) -> ShSlopec -> ImRecCalibrator),
with two ways to get the interaction matrix:

* ``adjoint_intmat()``: one launch for every sub-aperture's slope Jacobian
  and one contraction with the influence functions
  (specula_b200.lib.sh_adjoint);
* ``pushpull_intmat(amplitude)``: the reference's push-pull sequence
  (+a_k, -a_k per mode, im_rec_calibrator.py:58-63) on the same CUDA chain,
  captured in one CUDA graph.

Default sizes: 8 m pupil on 320 px, 40x40 sub-apertures of 8x8 phase
samples, 6x6 detector pixels of lambda/d (FFT 16, cut 4), 750 nm, 500
Zernike modes (IFunc 'zernike'); ``modes='kl'`` uses the 500-mode KL basis
of the same pupil (``kl_ifunc``) instead.
"""

import numpy as np
import torch

from specula_b200 import RAD2ASEC
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.electric_field import ElectricField
from specula_b200.data_objects.ifunc import IFunc
from specula_b200.data_objects.pixels import Pixels
from specula_b200.data_objects.simul_params import SimulParams
from specula_b200.data_objects.subap_data import SubapData
from specula_b200.lib.make_mask import make_mask
from specula_b200.lib.sh_adjoint import ShSlopesAdjoint
from specula_b200.processing_objects.dm import DM
from specula_b200.processing_objects.sh import SH
from specula_b200.processing_objects.sh_slopec import ShSlopec


def kl_ifunc(pupil, diameter_m, n_modes=500, r0=0.15, L0=25.0, n_act=26, device_idx=0):
    """KL modes of a pupil as an (n_modes x n_pupil_pixels) float32 tensor on
    the device: thin-plate-spline zonal functions on a circular actuator
    layout (26 across: 547 actuators on 320 px), then the von Karman KL basis
    with piston removed (lib/modal_base_generator.py:make_modal_base_from_ifs_fft).
    Each mode has unit RMS over the pupil, so a command of a is a nm RMS."""
    from specula_b200.lib.modal_basis import make_modal_base_from_ifs_fft
    from specula_b200.lib.zonal_ifunc import compute_zonal_ifunc
    dev = torch.device('cuda', device_idx)
    f, mask = compute_zonal_ifunc(pupil.shape[0], n_act, circ_geom=True, mask=pupil, device=dev)
    kl, _, _ = make_modal_base_from_ifs_fft(mask, diameter_m, f, r0, L0, oversampling=2)
    if kl.shape[0] < n_modes:
        raise ValueError(f'{n_act} actuators across give {kl.shape[0]} KL modes, fewer than {n_modes}')
    return kl[:n_modes].contiguous()


class ShCalibrationSystem:
    def __init__(self, pixel_pupil=320, diameter_m=8.0, n_lenses=40, subap_npx=6, wavelength_nm=750.0,
                 n_modes=500, obsratio=0.14, ifunc=None, subap_threshold=0.5, sign=-1, modes='zernike',
                 device_idx=0):
        from specula_b200.scao import valid_subaps
        self.device = torch.device('cuda', device_idx)
        pitch = diameter_m / pixel_pupil
        self.simul_params = SimulParams(pixel_pupil=pixel_pupil, pixel_pitch=pitch, time_step=0.001)
        pupil = make_mask(pixel_pupil, obsratio, 1.0)
        self.pupil = pupil
        lamd = wavelength_nm * 1e-9 / (diameter_m / n_lenses) * RAD2ASEC
        self.ef = ElectricField(pixel_pupil, pixel_pupil, pitch, S0=1.0, target_device_idx=device_idx)
        self.ef.A.copy_(torch.as_tensor(pupil.astype(np.float32)))
        self.sh = SH(wavelengthInNm=wavelength_nm, subap_wanted_fov=subap_npx * lamd, sensor_pxscale=lamd,
                     subap_on_diameter=n_lenses, subap_npx=subap_npx, fov_ovs_coeff=1.0,
                     target_device_idx=device_idx)
        self.sh.inputs['in_ef'].set(self.ef)
        self.sh.setup()
        idxs, dmap = valid_subaps(pupil, n_lenses, subap_npx, subap_threshold)
        self.subapdata = SubapData(idxs=idxs, display_map=dmap, nx=n_lenses, ny=n_lenses,
                                   target_device_idx=device_idx)
        self.slopec = ShSlopec(self.subapdata, target_device_idx=device_idx)
        self.slopec.inputs['in_pixels'].set(Pixels(n_lenses * subap_npx, n_lenses * subap_npx,
                                                   target_device_idx=device_idx))
        self.slopec.setup()
        if ifunc is None and modes == 'kl':
            ifunc = IFunc(ifunc=kl_ifunc(pupil, diameter_m, n_modes, device_idx=device_idx), mask=pupil,
                          target_device_idx=device_idx)
        elif ifunc is None:
            ifunc = IFunc(type_str='zernike', mask=pupil, npixels=pixel_pupil, nmodes=n_modes,
                          target_device_idx=device_idx)
        elif not isinstance(ifunc, IFunc):
            ifunc = IFunc(ifunc=ifunc, mask=pupil, target_device_idx=device_idx)
        self.dm = DM(self.simul_params, 0, ifunc=ifunc, sign=sign, target_device_idx=device_idx)
        self.dm.inputs['in_command'].set(BaseValue(value=np.zeros(ifunc.size[0], np.float32),
                                                   target_device_idx=device_idx))
        self.dm.setup()
        self.adjoint = ShSlopesAdjoint(self.sh, self.slopec)
        self.n_modes = ifunc.size[0]
        self.n_valid = self.adjoint.n_valid
        self._pix2col = self.adjoint.pixel_to_column(self.dm)
        self._flat = torch.zeros((pixel_pupil, pixel_pupil), dtype=torch.float32, device=self.device)
        self._pushpull = None

    @property
    def A(self):
        return self.ef.A

    def adjoint_intmat(self, phase=None):
        """n_modes x 2 n_valid interaction matrix from the adjoint, linearised
        at ``phase`` (nm, default flat)."""
        ph = self._flat if phase is None else phase
        return self.adjoint.intmat(self.A, ph, self.dm, pix2col=self._pix2col)

    def pushpull_intmat(self, amplitude):
        """The reference's push-pull matrix at ``amplitude`` (scalar or one per
        mode, command units), captured once per amplitude and replayed."""
        key = tuple(np.atleast_1d(np.asarray(amplitude, dtype=np.float64)).tolist())
        if self._pushpull is None or self._pushpull[0] != key:
            im, replay = self.adjoint.pushpull_intmat(self.A, self.dm, amplitude, graph=True)
            self._pushpull = (key, replay)
            return im
        return self._pushpull[1]()

    @staticmethod
    def contract_bytes(n_modes, n_valid_pixels_in_subaps, n_valid, np2):
        """Algorithmic bytes of one sb_intmat_contract launch: every influence
        function sample under a valid sub-aperture read once, the Jacobian
        and index tables read, the matrix written."""
        return 4 * (n_modes * n_valid_pixels_in_subaps + 2 * n_valid * np2 + n_valid * np2 + n_valid +
                    n_modes * 2 * n_valid)

    def pixels_under_valid_subaps(self):
        """Mirror columns that fall inside a valid sub-aperture."""
        p = self.adjoint.np_sub
        n = self.adjoint.n_lenses
        col = self._pix2col.cpu().numpy().reshape(self.adjoint.field, self.adjoint.field)
        count = 0
        for L in self.adjoint._lenslet.cpu().numpy().tolist():
            li, lj = divmod(int(L), n)
            count += int((col[li * p:(li + 1) * p, lj * p:(lj + 1) * p] >= 0).sum())
        return count
