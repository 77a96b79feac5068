"""Reconstruction matrix, (n_modes x n_slopes) as used by Modalrec
(mirrors specula/data_objects/recmat.py:8-68)."""
from specula_b200.base_data_obj import BaseDataObj


class Recmat(BaseDataObj):
    def __init__(self, recmat, modes2recLayer=None, norm_factor: float = 0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.recmat = self._tensor(recmat)
        self.norm_factor = norm_factor
        self.proj_list = []
        self.modes2recLayer = None

    def reduce_size(self, nModesToBeDiscarded):
        n = self.recmat.shape[1]
        if nModesToBeDiscarded >= n:
            raise ValueError(f'nModesToBeDiscarded should be less than nmodes (<{n})')
        self.recmat = self.recmat[:, :n - nModesToBeDiscarded].contiguous()
