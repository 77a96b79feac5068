"""IIR temporal filter on the B200 (mirrors specula/processing_objects/iir_filter.py:9-211)
for filters of up to 8 numerator / denominator taps (the 2-tap integrator
with forgetting factor has a straight-line path).  One sb_integrator call
per step performs the state shift of prepare_trigger, the filter update of
trigger_code and the delayed output of post_trigger, with the reference's
float32 operation order, including NumPy's summation order of the tap
products (bit-exact)."""
import math

import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue


class IirFilter(BaseProcessingObj):
    def __init__(self, simul_params, iir_filter_data, delay: float = 0, integration: bool = True,
                 offset: float = None, og_shaper: float = None, target_device_idx=None, precision=None):
        if integration is False:
            raise NotImplementedError('IirFilter: integration=False is not implemented yet')
        if og_shaper is not None:
            raise NotImplementedError('OG Shaper not implementd yet')
        if offset is not None:
            raise NotImplementedError('Offset not implemented yet')
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.simul_params = simul_params
        self.time_step = simul_params.time_step
        self.iir_filter_data = iir_filter_data
        self._n_num = iir_filter_data.num_np.shape[1]
        self._n_den = iir_filter_data.den_np.shape[1]
        if not (1 <= self._n_num <= 8 and 1 <= self._n_den <= 8):
            raise NotImplementedError('IirFilter: filters of up to 8 taps are on the specula_b200 path')
        self.delay = delay if delay is not None else 0
        if int(np.ceil(self.delay)) + 1 > 8:
            raise NotImplementedError('IirFilter: delays above 7 frames are not on the specula_b200 path')
        self._n = iir_filter_data.nfilter
        self._total_length = int(np.ceil(self.delay)) + 1
        self.state = torch.zeros((self._n, self._total_length), dtype=self.dtype, device=self.device)
        self._ist = torch.zeros((self._n, self._n_num), dtype=self.dtype, device=self.device)
        self._ost = torch.zeros((self._n, self._n_den), dtype=self.dtype, device=self.device)
        self.out_comm = BaseValue(value=torch.zeros(self._n, dtype=self.dtype, device=self.device),
                                  target_device_idx=target_device_idx)
        self.inputs['delta_comm'] = InputValue(type=BaseValue)
        self.outputs['out_comm'] = self.out_comm

    @property
    def last_state(self):
        return self.state[:, 0]

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        rem = self.delay % 1
        k_out = int(self.delay) if rem == 0 else int(math.ceil(self.delay))
        self._num = self.iir_filter_data.num.to(self.device, torch.float32).contiguous()
        self._den = self.iir_filter_data.den.to(self.device, torch.float32).contiguous()
        self._plan = _lib.IirPlan(n=self._n, total=self._total_length, shift=int(self.delay > 0), k_out=k_out,
                                  rem=float(np.float32(rem)), one_minus_rem=float(np.float32(1 - rem)),
                                  num=self._num.data_ptr(), den=self._den.data_ptr(), ist=self._ist.data_ptr(),
                                  ost=self._ost.data_ptr(), state=self.state.data_ptr(), out_next=None,
                                  n_num=self._n_num, n_den=self._n_den)

    @property
    def next_output_available(self):
        """True when the next step's output is known one step ahead
        (integer delay >= 1), see trigger_code(out_next=...)."""
        return self.delay % 1 == 0 and self.delay >= 1

    def next_output(self):
        """The output the next step will emit, from the current state."""
        return self.state[:, int(self.delay) - 1]

    def trigger_code(self, out_next=None):
        """One filter step; with ``out_next`` (a float32 device vector) the
        kernel also writes the output of the following step."""
        d = self.local_inputs['delta_comm'].value
        if not isinstance(d, torch.Tensor) or d.device != self.device or d.dtype != torch.float32:
            d = torch.as_tensor(d, dtype=torch.float32, device=self.device)
        self._plan.out_next = None if out_next is None else out_next.data_ptr()
        try:
            _lib.call('sb_integrator', _byref(self._plan), d.contiguous().data_ptr(),
                      self.out_comm.value.data_ptr(), self.stream_handle())
        finally:
            self._plan.out_next = None

    def post_trigger(self):
        self.out_comm.generation_time = self.current_time


def _byref(s):
    import ctypes
    return ctypes.byref(s)
