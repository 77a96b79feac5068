"""Time-series storage of loop outputs (mirrors
specula/processing_objects/data_store.py:19-116).

Every input connected to the store (a BaseValue, Slopes, Pixels or
ElectricField output) is recorded at each step where it was refreshed,
keyed by the step time.  The reference copies each value to the host every
step (a device synchronisation per step); here the values are cloned on
the device and moved to pinned host memory in batches of ``flush_steps``
with non-blocking copies, so the loop never waits for the store.
``finalize()`` writes, under ``store_dir/<YYYYmmdd_HHMMSS>``, one file per
input in the reference's layout:

* ``fits``: primary image = the stacked values (steps first, the object
  precision), extension 1 = the step times (ns, same dtype);
* ``pickle``: {'data', 'times', 'hdr'};

plus ``params.yml`` / ``replay_params.yml`` when setParams /
setReplayParams were called (the reference requires them).
"""
import os
import pickle
import time
from collections import OrderedDict, defaultdict

import numpy as np
import torch

from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.electric_field import ElectricField
from specula_b200.data_objects.pixels import Pixels
from specula_b200.data_objects.slopes import Slopes
from specula_b200.lib import fits_io


class DataStore(BaseProcessingObj):
    def __init__(self, store_dir: str, data_format: str = 'fits', flush_steps: int = 256,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if data_format not in ('fits', 'pickle'):
            raise TypeError(f'Error: unsupported file format {data_format}')
        self.data_filename = ''
        self.tn_dir = store_dir
        self.data_format = data_format
        self.flush_steps = int(flush_steps)
        self.params = None
        self.replay_params = None
        self._pending = defaultdict(list)        # name -> [(time, device tensor)]
        self._host = defaultdict(list)           # name -> [(times, pinned host tensor of stacked values)]
        self._events = []

    def setParams(self, params):
        self.params = params

    def setReplayParams(self, replay_params):
        self.replay_params = replay_params

    @staticmethod
    def _value_of(item):
        if isinstance(item, BaseValue):
            return torch.as_tensor(item.value)
        if isinstance(item, Slopes):
            return item.slopes
        if isinstance(item, Pixels):
            return item.pixels
        if isinstance(item, ElectricField):
            return torch.stack((item.A, item.phaseInNm))
        raise TypeError(f"Error: don't know how to save an object of type {type(item)}")

    def trigger_code(self):
        for name, inp in self.inputs.items():
            item = inp.get(self.target_device_idx)
            if item is not None and item.generation_time == self.current_time:
                v = self._value_of(item)
                self._pending[name].append((self.current_time, v.detach().clone()))
                if len(self._pending[name]) >= self.flush_steps:
                    self._flush(name)

    def _flush(self, name):
        """Stack the pending device copies and start their copy to pinned host memory."""
        pend = self._pending.pop(name, [])
        if not pend:
            return
        times = [t for t, _ in pend]
        stacked = torch.stack([v for _, v in pend])
        host = torch.empty(stacked.shape, dtype=stacked.dtype, device='cpu',
                           pin_memory=stacked.is_cuda)
        host.copy_(stacked, non_blocking=True)
        if stacked.is_cuda:
            ev = torch.cuda.Event()
            ev.record()
            self._events.append(ev)
        self._host[name].append((times, host))

    def _series(self):
        for name in list(self._pending):
            self._flush(name)
        for ev in self._events:
            ev.synchronize()
        self._events = []
        npdt = np.float32 if self.precision == 1 else np.float64
        out = OrderedDict()
        for name, chunks in self._host.items():
            times = np.array([t for ts, _ in chunks for t in ts], dtype=npdt)
            data = np.concatenate([h.numpy() for _, h in chunks], axis=0).astype(npdt)
            out[name] = (times, data)
        return out

    def create_TN_folder(self):
        today = time.strftime('%Y%m%d_%H%M%S')
        prefix = os.path.join(self.tn_dir, today)
        k = 1
        while os.path.exists(prefix):
            prefix = os.path.join(self.tn_dir, f'{today}_{k}')
            k += 1
        os.makedirs(prefix)
        self.tn_dir = prefix

    def save_params(self):
        import yaml
        if self.params is not None:
            with open(os.path.join(self.tn_dir, 'params.yml'), 'w') as f:
                yaml.dump(self.params, f, default_flow_style=False, sort_keys=False)
        if self.replay_params is not None:
            self.replay_params.setdefault('data_source', {})['store_dir'] = self.tn_dir
            with open(os.path.join(self.tn_dir, 'replay_params.yml'), 'w') as f:
                yaml.dump(self.replay_params, f, default_flow_style=False, sort_keys=False)

    def save_fits(self):
        for name, (times, data) in self._series().items():
            fits_io.write_hdus(os.path.join(self.tn_dir, name + '.fits'), [(data, {}), (times, {})], overwrite=True)

    def save_pickle(self):
        for name, (times, data) in self._series().items():
            with open(os.path.join(self.tn_dir, name + '.pickle'), 'wb') as f:
                pickle.dump({'data': data, 'times': times, 'hdr': {}}, f, protocol=pickle.HIGHEST_PROTOCOL)

    def finalize(self):
        self.create_TN_folder()
        self.save_params()
        if self.data_format == 'pickle':
            self.save_pickle()
        else:
            self.save_fits()
