"""Time and device bookkeeping shared by data and processing objects
(mirrors specula/base_time_obj.py:6-109).

Times are integer nanoseconds (``_time_resolution = 1e9``); ``seconds_to_t``
converts through the decimal string exactly like the reference, so loop
times are identical integers.
"""
from decimal import Decimal

import torch

import specula_b200 as _g


class BaseTimeObj:
    def __init__(self, target_device_idx=None, precision=None):
        self._time_resolution = int(1e9)
        self.precision = _g.global_precision if precision is None else precision
        self.target_device_idx = _g.default_target_device_idx if target_device_idx is None else target_device_idx
        if self.target_device_idx >= 0:
            self.device = torch.device('cuda', self.target_device_idx)
        else:
            self.device = torch.device('cpu')
        self.dtype = torch.float32 if self.precision == 1 else torch.float64
        self.complex_dtype = torch.complex64 if self.precision == 1 else torch.complex128

    def t_to_seconds(self, t):
        return float(t) / float(self._time_resolution)

    def seconds_to_t(self, seconds):
        if self._time_resolution == 0:
            return 0
        # round to 9 decimals through the string form, as the reference does
        d = Decimal(f'{float(seconds):.9f}')
        return int(d * self._time_resolution)

    def _zeros(self, *shape, dtype=None):
        return torch.zeros(*shape, dtype=self.dtype if dtype is None else dtype, device=self.device)

    def _tensor(self, a, dtype=None):
        """Copy a host array (or tensor) onto this object's device."""
        dt = self.dtype if dtype is None else dtype
        if isinstance(a, torch.Tensor):
            return a.to(device=self.device, dtype=dt).clone()
        return torch.as_tensor(_np_array(a), device=self.device).to(dt).clone()


def _np_array(a):
    import numpy as np
    return np.ascontiguousarray(np.asarray(a))
