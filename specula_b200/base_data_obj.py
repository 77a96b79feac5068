"""Base of every data object: a generation time stamp plus device placement
(mirrors specula/base_data_obj.py:11-186).

All objects of one loop live on the same CUDA device here, so the
cross-device clone path of the reference (copyTo / transferDataTo) reduces to
returning the object itself or moving its tensors.
"""
import torch

from specula_b200.base_time_obj import BaseTimeObj


class BaseDataObj(BaseTimeObj):
    def __init__(self, target_device_idx=None, precision=None):
        super().__init__(target_device_idx, precision)
        self._generation_time = -1

    @property
    def generation_time(self):
        return self._generation_time

    @generation_time.setter
    def generation_time(self, value):
        self._generation_time = value

    def copyTo(self, target_device_idx):
        """Same object if already there, else a shallow clone whose tensors
        are moved to the target device (base_data_obj.py:80-106)."""
        if target_device_idx == self.target_device_idx:
            return self
        import copy
        cloned = copy.copy(self)
        dev = torch.device('cuda', target_device_idx) if target_device_idx >= 0 else torch.device('cpu')
        for k, v in vars(self).items():
            if isinstance(v, torch.Tensor):
                setattr(cloned, k, v.to(dev))
        cloned.target_device_idx = target_device_idx
        cloned.device = dev
        return cloned

    def transferDataTo(self, destobj):
        for k, v in vars(self).items():
            if isinstance(v, torch.Tensor) and isinstance(getattr(destobj, k, None), torch.Tensor):
                getattr(destobj, k).copy_(v)
        destobj.generation_time = self.generation_time
        return destobj
