"""Sodium laser-guide-star kernels of the SH (mirrors
specula/data_objects/convolution_kernel.py:134-380 and
specula/data_objects/gaussian_convolution_kernel.py:5-109).

``real_kernels`` (dimx*dimy, dimension, dimension) float32: the geometric
beacon images (specula_b200.lib.lgs.lgs_map_sh, computed on the device);
``kernels``: per lenslet (row-major) the normalised map or, with
``return_fft`` (what the SH uses), its normalised inverse FFT in complex64.
Both tensors keep their device addresses when the kernels are recomputed,
so a captured SH graph reads the new values.  ``prepare_for_sh``
recomputes only when a parameter changed.  The reference also caches the
maps in a FITS file named after a hash in the working directory; here they
are recomputed instead (a few milliseconds on the device), and
``save`` / ``restore`` read and write the reference's file layout.
"""
import hashlib
import json

import numpy as np
import torch

from specula_b200.base_data_obj import BaseDataObj
from specula_b200.lib import fits_io
from specula_b200.lib.lgs import kernel_spectra, lgs_map_sh


class ConvolutionKernel(BaseDataObj):
    def __init__(self, dimx: int, dimy: int, pxscale: float, pupil_size_m: float, dimension: int,
                 launcher_pos: list = (0.0, 0.0, 0.0), seeing: float = 0.0, launcher_size: float = 0.0,
                 zfocus: float = 90e3, theta: list = (0.0, 0.0), airmass: float = 1.0, oversampling: int = 1,
                 return_fft: bool = True, positive_shift_tt: bool = True, target_device_idx: int = None,
                 precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if len(launcher_pos) != 3:
            raise ValueError('Launcher position must be a three-elements vector [m]')
        if dimx != dimy:
            raise NotImplementedError('ConvolutionKernel: square lenslet arrays only')
        self.dimx = dimx
        self.dimy = dimy
        self.pxscale = pxscale
        self.pupil_size_m = pupil_size_m
        self.dimension = dimension
        self.seeing = seeing
        self.launcher_size = launcher_size
        self.spot_size = float(np.sqrt(seeing ** 2 + launcher_size ** 2))
        self.zlayer = None
        self.zprofile = None
        self.zfocus = zfocus
        self.theta = np.asarray(theta, dtype=np.float64)
        self.airmass = airmass
        self.oversampling = oversampling
        self.launcher_pos = np.asarray(launcher_pos, dtype=np.float64)
        self.return_fft = return_fft
        self.positive_shift_tt = positive_shift_tt
        n, d = dimx * dimy, dimension
        self.real_kernels = torch.zeros((n, d, d), dtype=torch.float32, device=self.device)
        self.kernels = torch.zeros((n, d, d), dtype=torch.complex64 if return_fft else torch.float32,
                                   device=self.device)
        self._kernel_fn = None

    def _tt(self):
        return np.array([0.5, 0.5] if self.positive_shift_tt else [-0.5, -0.5]) * self.pxscale

    def calculate_focus(self):
        z = np.asarray(self.zlayer, dtype=np.float64)
        p = np.asarray(self.zprofile, dtype=np.float64)
        return float(np.sum(z * p) / np.sum(p))

    def _params(self):
        zfocus = self.zfocus if self.zfocus != -1 else self.calculate_focus()
        return [self.dimx, self.pupil_size_m, self.launcher_pos.tolist(), zfocus * self.airmass,
                (np.asarray(self.zlayer, dtype=np.float64) * self.airmass).tolist(),
                np.asarray(self.zprofile, dtype=np.float64).tolist(),
                float(np.sqrt(self.seeing ** 2 + self.launcher_size ** 2)), self.pxscale, self.dimension,
                self.oversampling, (self._tt() + self.theta).tolist()]

    def build(self):
        """Name identifying the current kernel parameters (changes when any does)."""
        if self.zlayer is None or len(self.zlayer) != len(self.zprofile):
            raise ValueError('Number of elements of zlayer and zprofile must be the same')
        return 'ConvolutionKernel' + hashlib.sha1(json.dumps(self._params()).encode()).hexdigest()

    def calculate_lgs_map(self):
        if len(self.zlayer) != len(self.zprofile):
            raise ValueError('Number of elements of zlayer and zprofile must be the same')
        self.spot_size = float(np.sqrt(self.seeing ** 2 + self.launcher_size ** 2))
        if self.spot_size <= 0:
            raise ValueError('Spot size must be greater than zero')
        zfocus = (self.zfocus if self.zfocus != -1 else self.calculate_focus()) * self.airmass
        heights = np.asarray(self.zlayer, dtype=np.float64) * self.airmass
        maps = lgs_map_sh(self.dimx, self.pupil_size_m, self.launcher_pos, zfocus, heights - zfocus,
                          np.asarray(self.zprofile, dtype=np.float64), self.spot_size, self.pxscale,
                          self.dimension, overs=self.oversampling, theta=self._tt() + self.theta, device=self.device)
        self.real_kernels.copy_(maps)
        self.process_kernels(return_fft=self.return_fft)

    def process_kernels(self, return_fft=False):
        if not bool(torch.isfinite(self.real_kernels).all()):
            raise ValueError('Kernel contains non-finite values!')
        if return_fft:
            kernel_spectra(self.real_kernels, self.dimx, out=self.kernels)
        else:
            rk = self.real_kernels.to(torch.float64)
            tot = rk.sum(dim=(1, 2), keepdim=True)
            rk = torch.where(tot > 0, rk / torch.where(tot > 0, tot, torch.ones_like(tot)), rk)
            n, d = self.dimx, self.dimension
            self.kernels.copy_(rk.view(n, n, d, d).transpose(0, 1).reshape(n * n, d, d).to(self.kernels.dtype))

    def prepare_for_sh(self, sodium_altitude=None, sodium_intensity=None, current_time=None):
        if sodium_altitude is not None:
            self.zlayer = np.asarray(torch.as_tensor(sodium_altitude).cpu(), dtype=np.float64)
        if sodium_intensity is not None:
            self.zprofile = np.asarray(torch.as_tensor(sodium_intensity).cpu(), dtype=np.float64)
        fn = self.build()
        if fn != self._kernel_fn:
            self._kernel_fn = fn
            self.calculate_lgs_map()
        if current_time is not None:
            self.generation_time = current_time

    # FITS layout of the reference's save / restore (primary header + kernel maps in extension 1)
    def _header(self):
        return {'VERSION': 1.1, 'PXSCALE': float(self.pxscale), 'DIM': int(self.dimension),
                'OVERSAMP': int(self.oversampling), 'POSTT': bool(self.positive_shift_tt),
                'SPOTSIZE': float(self.spot_size), 'DIMX': int(self.dimx), 'DIMY': int(self.dimy)}

    def save(self, filename, hdr=None):
        h = dict(hdr or {})
        h.update(self._header())
        fits_io.write_hdus(filename, [(None, h), (self.real_kernels.cpu().numpy(), {})], overwrite=True)

    @classmethod
    def restore(cls, filename, target_device_idx=None, kernel_obj=None, return_fft=False):
        hdr = fits_io.getheader(filename, ext=0)
        if hdr['VERSION'] != 1.1:
            raise ValueError(f"Unknown version {hdr['VERSION']}. Only version=1.1 is supported")
        if kernel_obj is None:
            kernel_obj = cls._from_header(hdr, target_device_idx, return_fft)
        elif kernel_obj.dimx != hdr['DIMX'] or kernel_obj.dimy != hdr['DIMY']:
            raise ValueError('Provided kernel object dimensions do not match the FITS file dimensions')
        kernel_obj.pxscale = hdr['PXSCALE']
        kernel_obj.oversampling = hdr['OVERSAMP']
        kernel_obj.positive_shift_tt = hdr['POSTT']
        kernel_obj.spot_size = hdr['SPOTSIZE']
        data = torch.as_tensor(np.asarray(fits_io.getdata(filename, ext=1), dtype=np.float32),
                               device=kernel_obj.device)
        kernel_obj.real_kernels.copy_(data)
        kernel_obj.process_kernels(return_fft=kernel_obj.return_fft)
        return kernel_obj

    @classmethod
    def _from_header(cls, hdr, target_device_idx, return_fft):
        obj = cls(dimx=hdr['DIMX'], dimy=hdr['DIMY'], pxscale=hdr['PXSCALE'], pupil_size_m=0.0,
                  dimension=hdr['DIM'], launcher_size=hdr['SPOTSIZE'], oversampling=hdr['OVERSAMP'],
                  return_fft=return_fft, positive_shift_tt=hdr['POSTT'], target_device_idx=target_device_idx)
        obj.spot_size = hdr['SPOTSIZE']
        return obj


class GaussianConvolutionKernel(ConvolutionKernel):
    """Gaussian spot of ``spot_size`` arcsec on axis (no launcher position,
    no elongation): lgs_map_sh with the launcher at the origin, the beacon at
    90 km and one layer (gaussian_convolution_kernel.py:38-57)."""

    def __init__(self, dimx: int, dimy: int, pxscale: float, dimension: int, spot_size: float,
                 pupil_size_m: float = 0.0, oversampling: int = 1, return_fft: bool = True,
                 positive_shift_tt: bool = True, airmass: float = 1.0, target_device_idx: int = None,
                 precision: int = None):
        super().__init__(dimx=dimx, dimy=dimy, pxscale=pxscale, pupil_size_m=pupil_size_m, dimension=dimension,
                         airmass=airmass, oversampling=oversampling, return_fft=return_fft,
                         positive_shift_tt=positive_shift_tt, target_device_idx=target_device_idx,
                         precision=precision)
        self.spot_size = spot_size

    def build(self):
        params = [self.dimx, self.pupil_size_m, 90e3, self.spot_size, self.pxscale, self.dimension,
                  self._tt().tolist()]
        return 'ConvolutionKernel' + hashlib.sha1(json.dumps(params).encode()).hexdigest()

    def calculate_lgs_map(self):
        maps = lgs_map_sh(self.dimx, self.pupil_size_m, 0.0, 90e3, [0.0], [1.0], self.spot_size, self.pxscale,
                          self.dimension, overs=1, theta=self._tt(), device=self.device)
        self.real_kernels.copy_(maps)
        self.process_kernels(return_fft=self.return_fft)

    def prepare_for_sh(self, sodium_altitude=None, sodium_intensity=None, current_time=None):
        fn = self.build()
        if fn != self._kernel_fn:
            self._kernel_fn = fn
            self.calculate_lgs_map()
        if current_time is not None:
            self.generation_time = current_time

    @classmethod
    def _from_header(cls, hdr, target_device_idx, return_fft):
        return cls(dimx=hdr['DIMX'], dimy=hdr['DIMY'], pxscale=hdr['PXSCALE'], dimension=hdr['DIM'],
                   spot_size=hdr['SPOTSIZE'], oversampling=hdr['OVERSAMP'], return_fft=return_fft,
                   positive_shift_tt=hdr['POSTT'], target_device_idx=target_device_idx)
