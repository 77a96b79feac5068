"""Intensity image (mirrors specula/data_objects/intensity.py:5-33)."""
import torch

from specula_b200.base_data_obj import BaseDataObj


class Intensity(BaseDataObj):
    def __init__(self, dimx: int, dimy: int, target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.i = torch.zeros((dimx, dimy), dtype=self.dtype, device=self.device)

    @property
    def size(self):
        return tuple(self.i.shape)

    def sum(self, i2, factor=1.0):
        self.i.add_(i2.i * factor)
