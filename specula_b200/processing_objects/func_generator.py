"""Time-series generator (subset of specula/processing_objects/func_generator.py:14-207):
constant values (any type with zero amplitude), 'SIN' and the 'PUSHPULL' modal
push-pull sequence of specula/lib/modal_pushpull_signal.py:35-65."""
import numpy as np
import torch

from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue


class FuncGenerator(BaseProcessingObj):
    def __init__(self, func_type='SIN', nmodes: int = None, time_hist=None, psd=None, fr_psd=None,
                 continuous_psd=None, constant: list = None, amp: list = None, freq: list = None,
                 offset: list = None, vect_amplitude: list = None, nsamples: int = 1, seed: int = None,
                 ncycles: int = 1, vsize: int = 1, target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.type = func_type.upper()
        npdt = np.float32 if self.precision == 1 else np.float64
        self.constant = np.array(constant, dtype=npdt) if constant is not None else npdt(0.0)
        self.amp = np.array(amp, dtype=npdt) if amp is not None else npdt(0.0)
        self.freq = np.array(freq, dtype=npdt) if freq is not None else npdt(0.0)
        self.offset = np.array(offset, dtype=npdt) if offset is not None else npdt(0.0)
        self.time_hist = None
        if self.type == 'PUSHPULL':
            if nmodes is None or vect_amplitude is None:
                raise ValueError('PUSHPULL needs nmodes and vect_amplitude')
            va = np.asarray(vect_amplitude, dtype=float)
            th = np.zeros((2 * nmodes * ncycles, nmodes))
            for i in range(nmodes):
                for j in range(ncycles):
                    th[2 * (ncycles * i + j):2 * (ncycles * i + j) + 2, i] = [va[i], -va[i]]
            self.time_hist = np.repeat(th, nsamples, axis=0).astype(npdt)
        elif self.type not in ('SIN', 'LINEAR', 'RANDOM', 'TIME_HIST'):
            raise NotImplementedError(f'FuncGenerator: type {func_type} is not on the specula_b200 path')
        self.output = BaseValue(target_device_idx=target_device_idx)
        self.outputs['output'] = self.output
        self._iter = 0

    def trigger_code(self):
        if self.type == 'PUSHPULL':
            v = self.time_hist[min(self._iter, len(self.time_hist) - 1)]
            self._iter += 1
        elif self.type == 'SIN':
            t = self.current_time_seconds
            v = self.amp * np.sin(self.freq * 2 * np.pi * t + self.offset) + self.constant
        else:
            v = self.constant
        self.output.value = torch.as_tensor(np.array(v), device=self.device) \
            if self.device.type == 'cuda' else np.array(v)

    def check_ready(self, t):
        self.current_time = t
        self.current_time_seconds = self.t_to_seconds(t)
        self.ready = True
        return True

    def post_trigger(self):
        self.output.generation_time = self.current_time
