"""Valid sub-aperture pixel tables (mirrors specula/data_objects/subap_data.py:10-79).
``idxs`` are flattened row-major detector indices, one row per sub-aperture."""
import math

import numpy as np
import torch

from specula_b200.base_data_obj import BaseDataObj


class SubapData(BaseDataObj):
    def __init__(self, idxs, display_map, nx: int, ny: int, energy_th: float = 0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.idxs = np.asarray(idxs.cpu() if isinstance(idxs, torch.Tensor) else idxs).astype(np.int64)
        self.display_map = np.asarray(display_map.cpu() if isinstance(display_map, torch.Tensor)
                                      else display_map).astype(np.int64)
        self.nx = int(nx)
        self.ny = int(ny)
        self.energy_th = float(energy_th)

    @property
    def n_subaps(self):
        return self.idxs.shape[0]

    @property
    def np_sub(self):
        return int(math.sqrt(self.idxs.shape[1]))

    def single_mask(self):
        f = np.zeros(self.nx * self.ny, dtype=np.float32)
        f[self.display_map] = 1
        return f.reshape((self.nx, self.ny))

    def subap_idx(self, n):
        return self.idxs[n, :]

    def display_map_idx(self, n):
        return self.display_map[n]
