"""Detector frame (mirrors specula/data_objects/pixels.py:7-95).  Values are
stored in the object dtype; with photon noise they are integers, as the
reference's int64 frames are."""
import torch

from specula_b200.base_data_obj import BaseDataObj


class Pixels(BaseDataObj):
    def __init__(self, dimx: int, dimy: int, bits: int = 16, signed: int = 0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if bits > 64:
            raise ValueError('Cannot create pixel object with more than 64 bits per pixel')
        self.signed = signed
        self.bpp = bits
        self.bytespp = (bits + 7) // 8
        self.pixels = torch.zeros((dimx, dimy), dtype=self.dtype, device=self.device)

    def set_value(self, v):
        self.pixels.copy_(torch.as_tensor(v, dtype=self.dtype))

    @property
    def size(self):
        return tuple(self.pixels.shape)

    def multiply(self, factor):
        self.pixels.mul_(factor)

    def set_size(self, size):
        self.pixels = torch.zeros(size, dtype=self.dtype, device=self.device)
