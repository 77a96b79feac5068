"""Oracle: reconstructor, integrator, DM and push-pull calibration
(test infrastructure only).

Restates specula/processing_objects/modalrec.py:114-162 (non-POLC branch),
specula/processing_objects/iir_filter.py:100-211 with
specula/data_objects/iir_filter_data.py:264-292 (Integrator),
specula/processing_objects/dm.py:72-86 and the push-pull interaction matrix of
specula/processing_objects/im_rec_calibrator.py:42-71 with
specula/lib/modal_pushpull_signal.py:35-65 and
specula/data_objects/intmat.py:75-87.
"""
import numpy as np


def modalrec(recmat, slopes):
    """modes = R @ s (modalrec.py:159)."""
    return recmat @ slopes


class IntegratorOracle:
    """IIR integrator num=[0, g], den=[-ff, 1] with an integer or fractional
    output delay (iir_filter.py:100-211, iir_filter_data.py:278-292)."""

    def __init__(self, gains, ff=None, delay=0, precision=1):
        dt = np.float32 if precision == 1 else np.float64
        g = np.asarray(gains, dtype=float)
        n = len(g)
        ff = np.ones(n) if ff is None else np.broadcast_to(np.asarray(ff, dtype=float), (n,))
        self.num = np.zeros((n, 2), dtype=dt)
        self.num[:, 1] = g
        self.den = np.zeros((n, 2), dtype=dt)
        self.den[:, 0] = -ff
        self.den[:, 1] = 1
        self.delay = delay
        self.total = int(np.ceil(delay)) + 1
        self.state = np.zeros((n, self.total), dtype=dt)
        self.ist = np.zeros_like(self.num)
        self.ost = np.zeros_like(self.den)

    def step(self, delta):
        # prepare_trigger: shift the state buffer (iir_filter.py:100-108)
        if self.delay > 0:
            self.state[:, 1:self.total] = self.state[:, 0:self.total - 1]
        # trigger_code (iir_filter.py:171-197)
        no = self.den.shape[1]
        ni = self.num.shape[1]
        self.ost[:, :-1] = self.ost[:, 1:]
        self.ost[:, -1] = 0
        self.ist[:, :-1] = self.ist[:, 1:]
        self.ist[:, -1] = 0
        self.ist[:, ni - 1] = delta
        factor = 1 / self.den[:, no - 1]
        num_c = np.sum(self.num * self.ist, axis=1)
        den_c = np.sum(self.den[:, :no - 1] * self.ost[:, :no - 1], axis=1)
        self.ost[:, no - 1] = factor * (num_c - den_c)
        self.state[:, 0] = self.ost[:, no - 1]
        # post_trigger (iir_filter.py:199-211)
        rem = self.delay % 1
        if rem == 0:
            return self.state[:, int(self.delay)].copy()
        k = int(np.ceil(self.delay))
        return rem * self.state[:, k] + (1 - rem) * self.state[:, k - 1]


def dm_phase(ifunc, mask, commands, sign=-1, m2c=None, precision=1, idx=None):
    """DM layer phase: phase[mask] = (sign * m2c @ c) @ IF (dm.py:72-86).
    ``idx``: np.where(mask), when the caller keeps it (the reference computes
    it once at construction, ifunc.py:66-73)."""
    dt = np.float32 if precision == 1 else np.float64
    cmd = np.asarray(commands, dtype=dt)
    if m2c is not None:
        cmd = np.asarray(m2c, dtype=dt) @ cmd
    ifc = np.zeros(ifunc.shape[0], dtype=dt)
    ifc[:len(cmd)] = sign * cmd
    out = np.zeros(mask.shape, dtype=dt)
    out[np.where(mask) if idx is None else idx] = ifc @ ifunc
    return out


def pushpull_intmat(slopes_fn, nmodes, amplitudes):
    """Push-pull IM: row k accumulates s(+a_k)/a_k + s(-a_k)/(-a_k), i.e. twice
    the central difference (im_rec_calibrator.py:58-63,
    modal_pushpull_signal.py:35-65).  ``slopes_fn(k, a)`` returns the slopes
    with mode k commanded to amplitude a."""
    rows = []
    for k in range(nmodes):
        a = amplitudes[k]
        rows.append(slopes_fn(k, a) / a + slopes_fn(k, -a) / (-a))
    return np.array(rows)
