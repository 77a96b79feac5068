"""Slope vector, non-interleaved [sx..., sy...] by default
(mirrors specula/data_objects/slopes.py:8-159)."""
import torch

from specula_b200.base_data_obj import BaseDataObj


class Slopes(BaseDataObj):
    def __init__(self, length: int = None, slopes=None, interleave: bool = False,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if slopes is not None:
            self.slopes = self._tensor(slopes)
        else:
            self.slopes = torch.zeros(length, dtype=self.dtype, device=self.device)
        self.interleave = interleave
        self.single_mask = None
        self.display_map = None
        self._set_indices()

    def _set_indices(self):
        n = self.size // 2
        if self.interleave:
            self.indicesX = torch.arange(0, n, device=self.device) * 2
            self.indicesY = self.indicesX + 1
        else:
            self.indicesX = torch.arange(0, n, device=self.device)
            self.indicesY = self.indicesX + n

    def resize(self, new_size):
        self.slopes = torch.zeros(new_size, dtype=self.dtype, device=self.device)
        self._set_indices()

    @property
    def size(self):
        return self.slopes.numel()

    @property
    def xslopes(self):
        return self.slopes[self.indicesX]

    @xslopes.setter
    def xslopes(self, value):
        self.slopes[self.indicesX] = torch.as_tensor(value, dtype=self.dtype, device=self.device)

    @property
    def yslopes(self):
        return self.slopes[self.indicesY]

    @yslopes.setter
    def yslopes(self, value):
        self.slopes[self.indicesY] = torch.as_tensor(value, dtype=self.dtype, device=self.device)

    def indx(self):
        return self.indicesX

    def indy(self):
        return self.indicesY

    def sum(self, s2, factor):
        self.slopes.add_(s2.slopes * factor)

    def subtract(self, s2):
        self.slopes.sub_(s2.slopes if isinstance(s2, Slopes) else torch.as_tensor(s2.value, device=self.device))
