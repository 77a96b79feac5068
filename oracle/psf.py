"""Oracle (test infrastructure only): PSF and Strehl ratio of an electric
field, restated from specula/processing_objects/psf.py.

calc_psf follows PSF.calc_psf (psf.py:56-96): the complex field A*exp(i*phi)
zero-padded into the top-left corner of an imwidth x imwidth array, FFT,
fftshift, |.|^2, optionally normalised to its sum.  The Strehl ratio is the
centre pixel of the normalised PSF over that of the flat-phase reference
(psf.py:111-124).  PSFOracle mirrors the object's integration after
start_time (psf.py:126-137).
"""
import numpy as np


def out_size(dim, nd):
    """Padded PSF size (psf.py:46-52): round(dim * nd / 2) * 2."""
    return int(np.around(dim * nd / 2) * 2)


def calc_psf(phase, amp, imwidth=None, normalize=False, nocenter=False, precision=1):
    cdt = np.complex64 if precision == 1 else np.complex128
    result = amp * np.exp(1j * phase, dtype=cdt)
    if imwidth is not None:
        u = np.zeros((imwidth, imwidth), dtype=cdt)
        u[:result.shape[0], :result.shape[1]] = result
    else:
        u = result
    fp = np.fft.fft2(u)
    if not nocenter:
        fp = np.fft.fftshift(fp)
    psf = np.real(fp * np.conj(fp))
    if normalize:
        psf /= np.sum(psf)
    return psf


class PSFOracle:
    def __init__(self, shape, wavelength_nm, nd=1, start_time=0.0, precision=1):
        self.lam = wavelength_nm
        self.n = out_size(shape[0], nd)
        self.start_time = start_time
        self.precision = precision
        self.dtype = np.float32 if precision == 1 else np.float64
        self.ref = None
        self.int_psf = np.zeros((self.n, self.n), dtype=self.dtype)
        self.intsr = 0.0
        self.count = 0

    def step(self, A, phase_nm, t_seconds):
        """One trigger + post_trigger: returns (psf, sr)."""
        A = np.asarray(A, dtype=self.dtype)
        phase_nm = np.asarray(phase_nm, dtype=self.dtype)
        if self.ref is None:
            self.ref = calc_psf(A * 0.0, A, imwidth=self.n, normalize=True, precision=self.precision)
        phi = phase_nm * ((2 * np.pi) / self.lam)
        psf = calc_psf(phi, A, imwidth=self.n, normalize=True, precision=self.precision)
        c = self.n // 2
        sr = psf[c, c] / self.ref[c, c]
        if t_seconds >= self.start_time:
            self.count += 1
            self.intsr += sr
            self.int_psf += psf
        return psf, sr

    @property
    def int_sr(self):
        return self.intsr / self.count if self.count else 0.0
