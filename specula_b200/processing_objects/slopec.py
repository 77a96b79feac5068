"""Slope computer base (mirrors specula/processing_objects/slopec.py:9-101)."""
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.pixels import Pixels
from specula_b200.data_objects.slopes import Slopes


class Slopec(BaseProcessingObj):
    def __init__(self, sn: Slopes = None, use_sn: bool = False, accumulate: bool = False,
                 weight_from_accumulated: bool = False, recmat=None, filt_intmat=None, filt_recmat=None,
                 filtmat=None, accumulation_dt: float = 0, accumulated_pixels: tuple = (0, 0),
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if use_sn and not sn:
            raise ValueError('Slopes null are not valid')
        if weight_from_accumulated and accumulate:
            raise ValueError('weightFromAccumulated and accumulate must not be set together')
        for flag, what in ((recmat is not None, 'slope->mode recmat'), (filtmat is not None, 'slope filtering'),
                           (filt_intmat is not None or filt_recmat is not None, 'slope filtering'),
                           (accumulate, 'accumulation'), (weight_from_accumulated, 'weights from accumulation')):
            if flag:
                raise NotImplementedError(f'{type(self).__name__}: {what} is not on the specula_b200 path')
        self.slopes = Slopes(2, target_device_idx=target_device_idx, precision=precision)
        # slope nulls are stored but never subtracted, as in the reference (slopec.py:37-40)
        self.sn = sn
        self.use_sn = use_sn
        self.flux_per_subaperture_vector = BaseValue(target_device_idx=target_device_idx)
        self.max_flux_per_subaperture_vector = BaseValue(target_device_idx=target_device_idx)
        self.inputs['in_pixels'] = InputValue(type=Pixels)
        self.outputs['out_slopes'] = self.slopes
