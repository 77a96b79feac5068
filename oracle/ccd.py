"""Oracle: CCD detector (test infrastructure only).

Restates specula/processing_objects/ccd.py:198-287 (the start_time gate,
integration, binning,
QE, background/dark, Poisson photon noise, Gaussian readout noise, ADU
quantisation), and the deterministic detector-structure options: the
charge-transfer matrices (ccd.py:223-224), pixel gains (:239-240) and the
per-pixel QE map with its normalisation (:242-245, 285-287).  The random
EMCCD (excess) and CIC draws are checked by their statistics instead.

Binning follows the reference's intended arithmetic (ccd.py:264-280: b x b
block sums of the full-resolution integrated frame, scaled by
b^2 * sum(frame) / sum(blocks)).  The reference itself cannot run it: its
integrated frame is sized with `Pixels.size * binning` (ccd.py:113), a
tuple repetition, so the frame has the binned shape and apply_binning fails.

Noise draws use the same NumPy generators as the reference CPU path
(``default_rng(photon_seed)``, ``default_rng(readout_seed)``), so with equal
seeds this oracle reproduces the reference CPU CCD bit for bit.
"""
import numpy as np


class CCDOracle:
    def __init__(self, size, dt_s, loop_dt_s, bandw, binning=1, photon_noise=False,
                 readout_noise=False, background_noise=False, darkcurrent_noise=False,
                 readout_level=0.0, background_level=0.0, darkcurrent_level=0.0,
                 quantum_eff=1.0, photon_seed=1, readout_seed=2, ADU_gain=8, ADU_bias=400,
                 precision=1, cte_mat=None, pixel_gains=None, qe_map=None, qe_map_normalise=False):
        self.dtype = np.float32 if precision == 1 else np.float64
        self.size = (size[0] // binning, size[1] // binning)
        self.binning = binning
        self.integrated = np.zeros((self.size[0] * binning, self.size[1] * binning), dtype=self.dtype)
        self.dt_ratio = loop_dt_s * bandw
        self.frames_per_read = int(round(dt_s / loop_dt_s))
        self.count = 0
        self.photon_noise = photon_noise
        self.readout_noise = readout_noise
        self.background_noise = background_noise
        self.darkcurrent_noise = darkcurrent_noise
        self.readout_level = readout_level
        self.background_level = background_level
        self.darkcurrent_level = darkcurrent_level
        self.qe = quantum_eff
        self.gain = ADU_gain
        self.bias = ADU_bias
        self.photon_rng = np.random.default_rng(photon_seed)
        self.readout_rng = np.random.default_rng(readout_seed)
        self.cte_mat = None if cte_mat is None else np.asarray(cte_mat, dtype=self.dtype)
        self.pixel_gains = None if pixel_gains is None else np.asarray(pixel_gains, dtype=self.dtype)
        self.qe_map = None if qe_map is None else np.asarray(qe_map, dtype=self.dtype)
        self.qe_map_normalise = qe_map_normalise

    def step(self, intensity):
        """One loop step; returns the frame when a read-out happens, else None
        (ccd.py:198-216 with start_time 0)."""
        self.integrated += intensity * self.dt_ratio
        self.count += 1
        if self.count % self.frames_per_read:
            return None
        return self._read()

    def step_at(self, intensity, t, start=0):
        """The loop step at time t with the start_time gate and read-out rule
        of ccd.py:199-207 (times in loop steps, start a multiple of them):
        nothing before ``start``; the frame closes when
        (t + 1 - D - start) is a multiple of D, D = frames_per_read.  Returns
        the frame when one closes, else None."""
        if start > 0 and t < start:
            return None
        self.integrated += intensity * self.dt_ratio
        D = self.frames_per_read
        if (t + 1 - D - start) % D:
            return None
        return self._read()

    def _read(self):
        frame = self._binning()
        if self.qe != 1:
            frame = frame * self.qe
        if self.qe_map is not None:
            frame = frame * self.qe_map
        frame = self._noise(frame)
        self.integrated *= 0.0
        return frame

    def _binning(self):
        # ccd.py:264-280
        f = self.integrated.copy()
        if self.binning > 1:
            tot = np.sum(f)
            b = self.binning
            f = f.reshape(self.size[0], b, self.size[1], b).sum(axis=(1, 3))
            f = f * b ** 2 * (tot / np.sum(f))
        return f

    def _noise(self, f):
        # ccd.py:218-262
        if self.background_noise or self.darkcurrent_noise:
            f += (self.background_level + self.darkcurrent_level)
        if self.cte_mat is not None:
            f = np.dot(np.dot(self.cte_mat[:, :, 0], f), self.cte_mat[:, :, 1])
        if self.photon_noise:
            f = self.photon_rng.poisson(f)                      # int64 from here on
        if self.readout_noise:
            ron = self.readout_rng.standard_normal(size=f.size)
            f += (ron.reshape(f.shape) * self.readout_level).astype(f.dtype)
        if self.pixel_gains is not None:
            f *= self.pixel_gains
        if self.qe_map is not None and self.qe_map_normalise:
            f *= 1 / self.qe_map
        if self.photon_noise:
            f = np.round(f * self.gain) + self.bias
            np.maximum(f, 0, out=f)                             # clamp < 0 -> 0, in place
            f -= self.bias
            f = (f / self.gain).astype(f.dtype)
            if self.darkcurrent_noise:
                f -= self.darkcurrent_level
        return f
