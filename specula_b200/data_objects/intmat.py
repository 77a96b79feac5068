"""Interaction matrix (n_modes x n_slopes) and its pseudo-inverse
(mirrors specula/data_objects/intmat.py:8-111).  The pseudo-inverse runs in
float64 on the device (torch.linalg.pinv)."""
import torch

from specula_b200.base_data_obj import BaseDataObj
from specula_b200.data_objects.recmat import Recmat


class Intmat(BaseDataObj):
    def __init__(self, intmat, slope_mm=None, slope_rms=None, pupdata_tag: str = '', norm_factor: float = 0.0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.intmat = self._tensor(intmat)
        self.slope_mm = slope_mm
        self.slope_rms = slope_rms
        self.pupdata_tag = pupdata_tag
        self.norm_factor = norm_factor

    @property
    def size(self):
        return tuple(self.intmat.shape)

    def reduce_size(self, n_modes_to_be_discarded):
        n = self.intmat.shape[0]
        if n_modes_to_be_discarded >= n:
            raise ValueError(f'nModesToBeDiscarded should be less than nmodes (<{n})')
        self.intmat = self.intmat[:n - n_modes_to_be_discarded, :]

    def reduce_slopes(self, n_slopes_to_be_discarded):
        n = self.intmat.shape[1]
        if n_slopes_to_be_discarded >= n:
            raise ValueError(f'nSlopesToBeDiscarded should be less than nslopes (<{n})')
        self.intmat = self.intmat[:, :n - n_slopes_to_be_discarded]

    def generate_rec(self, nmodes=None, cut_modes=0, w_vec=None, interactive=False):
        im = self.intmat if nmodes is None else self.intmat[:nmodes, :]
        rec = self.pseudo_invert(im)
        return Recmat(rec, target_device_idx=self.target_device_idx, precision=self.precision)

    def pseudo_invert(self, matrix, n_modes_to_drop=0, w_vec=None, interactive=False):
        return torch.linalg.pinv(matrix.to(torch.float64)).to(self.dtype)
