"""IIR filter coefficients (mirrors specula/data_objects/iir_filter_data.py:9-120,264-292
for the integrator case).  num/den are (n_filters x 2): num = [0, gain],
den = [-ff, 1]."""
import numpy as np

from specula_b200.base_data_obj import BaseDataObj


class IirFilterData(BaseDataObj):
    def __init__(self, ordnum, ordden, num, den, target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        npdt = np.float32 if self.precision == 1 else np.float64
        self.ordnum = np.array(ordnum, dtype=int)
        self.ordden = np.array(ordden, dtype=int)
        self.num_np = self._normalise(np.array(num, dtype=npdt), self.ordnum)
        self.den_np = self._normalise(np.array(den, dtype=npdt), self.ordden)
        self.gain = self.num_np[:, -1].copy()
        self.num = self._tensor(self.num_np)
        self.den = self._tensor(self.den_np)

    @staticmethod
    def _normalise(c, order):
        # right-align coefficient rows shorter than the array (set_num/set_den)
        c = c.copy()
        w = c.shape[1]
        for i in range(len(c)):
            if order[i] < w and np.sum(np.abs(c[i, int(order[i]):])) == 0:
                c[i, :] = np.roll(c[i, :], w - int(order[i]))
        return c

    @property
    def nfilter(self):
        return len(self.num_np)

    @staticmethod
    def from_gain_and_ff(gain, ff=None, target_device_idx=None, precision=None):
        gain = np.array(gain, dtype=float)
        n = len(gain)
        if ff is None:
            ff = np.ones(n)
        elif np.ndim(ff) == 0 or len(ff) != n:
            ff = np.full(n, ff)
        else:
            ff = np.array(ff, dtype=float)
        num = np.zeros((n, 2))
        den = np.zeros((n, 2))
        num[:, 1] = gain
        den[:, 0] = -ff
        den[:, 1] = 1
        return IirFilterData(np.full(n, 2), np.full(n, 2), num, den,
                             target_device_idx=target_device_idx, precision=precision)
