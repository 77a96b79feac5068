"""Atmospheric propagation on the B200 (mirrors
specula/processing_objects/atmo_propagation.py:15-250), on-axis branch.

For an on-axis source (or ground layers) the reference crops every layer
around its centre and multiplies amplitudes / adds phases into the source's
field (:123-125).  Here that is one sb_propagate_on_axis call per source.
Off-axis / LGS interpolation and Fresnel propagation are not on this path
(NotImplementedError at setup).
"""
import numpy as np

from specula_b200 import _lib
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
        for source in self.source_dict.values():
            for layer in self._layers:
                on_axis = layer.height == 0 or (np.isinf(source.height) and source.r == 0)
                plain = (not np.any(layer.shiftXYinPixel) and self.pupil_position is None and
                         layer.rotInDeg == 0 and max(layer.magnification, 1.0) == 1)
                if not (on_axis and plain):
                    raise NotImplementedError('AtmoPropagation: off-axis / shifted / rotated / magnified layers '
                                              '(Interp2D branch) are not on the specula_b200 path')
                if layer.size[0] < self.pixel_pupil or layer.size[1] < self.pixel_pupil:
                    raise ValueError(f'AtmoPropagation: layer {layer.size} smaller than the pupil')

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
        arr = self._descriptors(phase_override)
        for name in self.source_dict:
            ef = self.outputs['out_' + name + '_ef']
            _lib.call('sb_propagate_on_axis', arr, len(self._layers), self.pixel_pupil, ef.A.data_ptr(),
                      ef.phaseInNm.data_ptr(), self.stream_handle())

    def post_trigger(self):
        for name in self.source_dict:
            self.outputs['out_' + name + '_ef'].generation_time = self.current_time
