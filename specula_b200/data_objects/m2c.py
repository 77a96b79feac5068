"""Modes-to-commands matrix (mirrors specula/data_objects/m2c.py:7-44)."""
from specula_b200.base_data_obj import BaseDataObj


class M2C(BaseDataObj):
    def __init__(self, m2c, nmodes: int = None, norm_factor: float = None,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.m2c = self._tensor(m2c)
        if nmodes is not None:
            self.set_nmodes(nmodes)
        self.norm_factor = norm_factor

    @property
    def nmodes(self):
        return self.m2c.shape[1]

    def set_nmodes(self, nmodes):
        self.m2c = self.m2c[:, :nmodes].contiguous()
