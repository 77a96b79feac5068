"""Atmospheric propagation on the B200 (mirrors
specula/processing_objects/atmo_propagation.py:15-250).

For an on-axis source (or ground layers) the reference crops every layer
around its centre and multiplies amplitudes / adds phases into the source's
field (:123-125); when every layer of every source is cropped, that is one
sb_propagate_on_axis call per source.  Off-axis sources, sources at a finite
height (LGS cone effect) and shifted, rotated or magnified layers are
resampled as the reference's Interp2D does (:127-209): the sample
coordinates are built on the host at setup, and one sb_propagate call per
source crops or bilinearly interpolates each layer.  Fresnel propagation
and mergeLayersContrib=False are not on this path.
"""
import numpy as np
import torch

from specula_b200 import ASEC2RAD, _lib
from specula_b200.lib.interp2d import interp_coords_xy
from specula_b200.lib.make_mask import make_xy
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.connections import InputList
from specula_b200.data_objects.electric_field import ElectricField
from specula_b200.data_objects.layer import Layer


class AtmoPropagation(BaseProcessingObj):
    def __init__(self, simul_params, source_dict: dict, doFresnel: bool = False, wavelengthInNm: float = 500.0,
                 pupil_position=None, mergeLayersContrib=True, target_device_idx=None, precision=None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if doFresnel:
            raise NotImplementedError('Fresnel propagation is not implemented')
        if not len(source_dict) > 0:
            raise ValueError('No sources have been set')
        if not simul_params.pixel_pupil > 0:
            raise ValueError('Pixel pupil must be >0')
        if not mergeLayersContrib:
            raise NotImplementedError('AtmoPropagation: mergeLayersContrib=False is not on the specula_b200 path')
        self.simul_params = simul_params
        self.pixel_pupil = simul_params.pixel_pupil
        self.pixel_pitch = simul_params.pixel_pitch
        self.pixel_pupil_size = self.pixel_pupil
        self.source_dict = source_dict
        self.pupil_position = None if pupil_position is None else np.array(pupil_position, dtype=float)
        self.mergeLayersContrib = mergeLayersContrib
        for name, source in source_dict.items():
            ef = ElectricField(self.pixel_pupil, self.pixel_pupil, self.pixel_pitch,
                               target_device_idx=self.target_device_idx, precision=self.precision)
            ef.S0 = source.phot_density()
            self.outputs['out_' + name + '_ef'] = ef
        self.inputs['atmo_layer_list'] = InputList(type=Layer, optional=True)
        self.inputs['common_layer_list'] = InputList(type=Layer)
        self.airmass = 1. / np.cos(np.radians(simul_params.zenithAngleInDeg or 0.0))

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        atmo = self.inputs['atmo_layer_list'].get(self.target_device_idx) or []
        common = self.inputs['common_layer_list'].get(self.target_device_idx) or []
        self._layers = list(atmo) + list(common)
        if len(self._layers) < 1:
            raise ValueError('At least one layer must be set')
        if len(self._layers) > _lib.SB_MAX_LAYERS:
            raise NotImplementedError(f'AtmoPropagation: at most {_lib.SB_MAX_LAYERS} layers')
        self._coords = {}                  # source name -> [None (crop) or (yy, xx) device tensors] per layer
        for name, source in self.source_dict.items():
            per = []
            for layer in self._layers:
                if layer.size[0] < self.pixel_pupil or layer.size[1] < self.pixel_pupil:
                    raise ValueError(f'AtmoPropagation: layer {layer.size} smaller than the pupil')
                on_axis = layer.height == 0 or (np.isinf(source.height) and source.r == 0)
                plain = (not np.any(layer.shiftXYinPixel) and self.pupil_position is None and
                         layer.rotInDeg == 0 and max(layer.magnification, 1.0) == 1)
                if on_axis and plain:
                    per.append(None)
                elif (source.height - layer.height) * self.airmass > 0:
                    yy, xx = self._layer_coords(source, layer)
                    per.append((torch.as_tensor(yy, device=self.device), torch.as_tensor(xx, device=self.device)))
                else:
                    raise ValueError('Invalid layer/source geometry')
            self._coords[name] = per
        self._interpolated = any(c is not None for per in self._coords.values() for c in per)
        if self._interpolated:
            self._samplings = {name: self._sampling_table(per) for name, per in self._coords.items()}

    def _layer_coords(self, source, layer):
        """Sample coordinates of one layer for one source (atmo_propagation.py:
        169-209, with Interp2D's rounding, rotation and clamping): the source's
        angles and the airmass in float32, the grid in float64."""
        P = self.pixel_pupil
        L = layer.size[0]
        r = np.float32(source.polar_coordinates[0]) * ASEC2RAD
        phi = np.float32(source.polar_coordinates[1]) * (np.pi / 180.)
        airmass = np.float32(1.0) / np.cos(np.radians(self.simul_params.zenithAngleInDeg or 0.0), dtype=np.float32)
        half = np.array([(L - 1) / 2., (L - 1) / 2.]) - layer.shiftXYinPixel
        cos_sin = np.array([np.cos(phi), np.sin(phi)])
        if self.pupil_position is not None and L > P and np.isinf(source.height):
            pos = r * layer.height * airmass / layer.pixel_pitch * cos_sin + self.pupil_position / layer.pixel_pitch
        elif self.pupil_position is not None and L > P:
            sky = r * source.height * airmass / layer.pixel_pitch * cos_sin
            pup = self.pupil_position / layer.pixel_pitch
            pos = (sky - pup) * layer.height / source.height + pup
        else:
            pos = r * layer.height * airmass / layer.pixel_pitch * cos_sin
        pupmeta = P if np.isinf(source.height) else P * (abs(source.height - abs(layer.height)) / source.height)
        mag = max(layer.magnification, 1.0)
        if mag != 1.0:
            pupmeta /= mag
        limit0 = (layer.size[0] - P) / 2
        limit1 = (layer.size[1] - P) / 2
        if not (abs(pos[0]) <= limit0 and abs(pos[1]) <= limit1):
            raise ValueError('FATAL ERROR, the source is not inside the selected FoV for atmosphere layers generation.')
        xx, yy = make_xy(P, pupmeta / 2.)
        xx1 = xx + half[0] + pos[0]
        yy1 = yy + half[1] + pos[1]
        angle = -layer.rotInDeg % 360
        # the reference passes the angle in degrees scaled by 180 / pi once more
        return interp_coords_xy(layer.size, yy1, xx1, rotInDeg=angle * 180.0 / np.pi)

    def _sampling_table(self, per, phase_override=None):
        arr = (_lib.PropSampling * len(self._layers))()
        P = self.pixel_pupil
        for k, (layer, c) in enumerate(zip(self._layers, per)):
            d = arr[k]
            unit = getattr(layer, '_unit_amplitude', False)
            d.A = None if unit else layer.A.data_ptr()
            ph = layer.phaseInNm
            if phase_override and id(layer) in phase_override:
                ph = phase_override[id(layer)]
            d.phase = ph.data_ptr()
            d.ld = layer.phaseInNm.stride(0)
            d.rows, d.cols = layer.size[0], layer.size[1]
            if c is None:
                d.top = (layer.size[0] - P) // 2
                d.left = (layer.size[1] - P) // 2
            else:
                d.yy, d.xx = c[0].data_ptr(), c[1].data_ptr()
        return arr

    def _fill_dark_phase(self):
        """Interpolated layers with zero-amplitude pixels get the mean phase of
        the lit ones there, in place (atmo_propagation.py:128-132)."""
        for k, layer in enumerate(self._layers):
            if getattr(layer, '_unit_amplitude', False):
                continue
            if any(per[k] is not None for per in self._coords.values()):
                lit = layer.A != 0
                mean = torch.sum(torch.where(lit, layer.phaseInNm, torch.zeros_like(layer.phaseInNm))) / \
                    torch.clamp(torch.sum(lit), min=1)
                layer.phaseInNm.copy_(torch.where(lit, layer.phaseInNm, mean.to(layer.phaseInNm.dtype)))

    def _descriptors(self, phase_override=None):
        arr = (_lib.PropLayer * len(self._layers))()
        P = self.pixel_pupil
        for k, layer in enumerate(self._layers):
            d = arr[k]
            unit = getattr(layer, '_unit_amplitude', False)
            d.A = None if unit else layer.A.data_ptr()
            ph = layer.phaseInNm
            if phase_override and id(layer) in phase_override:
                ph = phase_override[id(layer)]
                if ph.shape != layer.phaseInNm.shape or ph.stride() != layer.phaseInNm.stride():
                    raise ValueError('AtmoPropagation: phase override must match the layer layout')
            d.phase = ph.data_ptr()
            d.ld = layer.phaseInNm.stride(0)
            if not unit and layer.A.stride(0) != d.ld:
                raise ValueError('AtmoPropagation: layer amplitude and phase must share a row stride')
            d.top = (layer.size[0] - P) // 2
            d.left = (layer.size[1] - P) // 2
        return arr

    def trigger_code(self, phase_override=None):
        """``phase_override``: {id(layer): tensor} reads another buffer in place
        of a layer's phase (used for the double-buffered DM of the pipelined
        loop graph)."""
        if self._interpolated:
            self._fill_dark_phase()
            for name in self.source_dict:
                ef = self.outputs['out_' + name + '_ef']
                arr = self._samplings[name] if not phase_override else \
                    self._sampling_table(self._coords[name], phase_override)
                _lib.call('sb_propagate', arr, len(self._layers), self.pixel_pupil, ef.A.data_ptr(),
                          ef.phaseInNm.data_ptr(), self.stream_handle())
            return
        arr = self._descriptors(phase_override)
        for name in self.source_dict:
            ef = self.outputs['out_' + name + '_ef']
            _lib.call('sb_propagate_on_axis', arr, len(self._layers), self.pixel_pupil, ef.A.data_ptr(),
                      ef.phaseInNm.data_ptr(), self.stream_handle())

    def post_trigger(self):
        for name in self.source_dict:
            self.outputs['out_' + name + '_ef'].generation_time = self.current_time
