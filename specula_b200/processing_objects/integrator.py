"""Integrator (mirrors specula/processing_objects/integrator.py:7-52): an
IirFilter with num=[0, gain], den=[-ff, 1] per mode."""
from specula_b200.data_objects.iir_filter_data import IirFilterData
from specula_b200.processing_objects.iir_filter import IirFilter


class Integrator(IirFilter):
    def __init__(self, simul_params, int_gain, ff: list = None, n_modes: int = None, delay: float = 0,
                 offset: float = None, og_shaper=None, target_device_idx: int = None, precision: int = None):
        if n_modes is not None:
            if isinstance(n_modes, int):
                n_modes = [n_modes]
            if len(n_modes) != len(int_gain):
                raise ValueError(f'When n_modes is a list, length of n_modes {len(n_modes)} must match '
                                 f'length of int_gain {len(int_gain)}')
            int_gain = [v for i, v in enumerate(int_gain) for _ in range(n_modes[i])]
            if ff is not None:
                if isinstance(ff, (int, float)):
                    ff = [ff]
                if len(n_modes) != len(ff):
                    raise ValueError(f'When n_modes is a list, length of n_modes {len(n_modes)} must match '
                                     f'length of ff {len(ff)}')
                ff = [v for i, v in enumerate(ff) for _ in range(n_modes[i])]
        data = IirFilterData.from_gain_and_ff(int_gain, ff=ff, target_device_idx=target_device_idx,
                                              precision=precision)
        super().__init__(simul_params, data, delay=delay, offset=offset, og_shaper=og_shaper,
                         target_device_idx=target_device_idx, precision=precision)
