"""Pupil stop layer (mirrors specula/data_objects/pupilstop.py:8-60).

The reference keeps the mask as uint8; here it is stored in the object dtype
(0/1), which gives identical products in the propagation."""
import numpy as np

from specula_b200.data_objects.layer import Layer
from specula_b200.lib.make_mask import make_mask


class Pupilstop(Layer):
    def __init__(self, simul_params, input_mask=None, mask_diam: float = 1.0, obs_diam: float = None,
                 shiftXYinPixel: tuple = (0.0, 0.0), rotInDeg: float = 0.0, magnification: float = 1.0,
                 target_device_idx: int = None, precision: int = None):
        self.simul_params = simul_params
        self.pixel_pupil = simul_params.pixel_pupil
        self.pixel_pitch = simul_params.pixel_pitch
        super().__init__(self.pixel_pupil, self.pixel_pupil, self.pixel_pitch, height=0,
                         shiftXYinPixel=shiftXYinPixel, rotInDeg=rotInDeg, magnification=magnification,
                         target_device_idx=target_device_idx, precision=precision)
        self._input_mask = input_mask
        self._mask_diam = mask_diam
        self._obs_diam = obs_diam
        mask = np.asarray(input_mask) if input_mask is not None else make_mask(self.pixel_pupil, obs_diam, mask_diam)
        self.A = self._tensor(mask)
        self._generation_time = 0
