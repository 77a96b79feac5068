"""Electric field: amplitude A and phase in nm on a square grid
(mirrors specula/data_objects/electric_field.py:8-167)."""
import math

import torch

from specula_b200.base_data_obj import BaseDataObj


class ElectricField(BaseDataObj):
    def __init__(self, dimx: int, dimy: int, pixel_pitch: float, S0: float = 0.0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        dimx, dimy = int(dimx), int(dimy)
        self.pixel_pitch = pixel_pitch
        self.S0 = S0
        self.A = torch.ones((dimx, dimy), dtype=self.dtype, device=self.device)
        self.phaseInNm = torch.zeros((dimx, dimy), dtype=self.dtype, device=self.device)

    def set_value(self, v):
        """Overwrite amplitude and phase in place (no reallocation)."""
        self.A.copy_(torch.as_tensor(v[0], dtype=self.dtype))
        self.phaseInNm.copy_(torch.as_tensor(v[1], dtype=self.dtype))

    def reset(self):
        self.A.fill_(1.0)
        self.phaseInNm.zero_()

    @property
    def size(self):
        return tuple(self.A.shape)

    def phi_at_lambda(self, wavelengthInNm):
        return self.phaseInNm * ((2 * math.pi) / wavelengthInNm)

    def ef_at_lambda(self, wavelengthInNm):
        """Complex field A*exp(i*2*pi*phase/lambda) (electric_field.py:67-75)."""
        return torch.polar(self.A, self.phi_at_lambda(wavelengthInNm))

    def product(self, ef2, subrect=None):
        if subrect is None:
            subrect = [0, 0]
        x2 = subrect[0] + self.size[0]
        y2 = subrect[1] + self.size[1]
        self.A.mul_(ef2.A[subrect[0]:x2, subrect[1]:y2])
        self.phaseInNm.add_(ef2.phaseInNm[subrect[0]:x2, subrect[1]:y2])

    def area(self):
        return self.A.numel() * (self.pixel_pitch ** 2)

    def masked_area(self):
        return (self.pixel_pitch ** 2) * float(torch.sum(self.A))

    def square_modulus(self, wavelengthInNm):
        ef = self.ef_at_lambda(wavelengthInNm)
        return (ef * ef.conj()).real
