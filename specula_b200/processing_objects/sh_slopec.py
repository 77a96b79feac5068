"""Shack-Hartmann slope computer on the B200 (mirrors
specula/processing_objects/sh_slopec.py:25-445).

``trigger_code()`` is one sb_slopec call implementing calc_slopes_nofor
(sh_slopec.py:308-438): gather each valid sub-aperture through
``SubapData.idxs``, subtract the threshold and clamp at 0, weighted CoG with
the weights of computeXYweights (:86-132), factor zeroed where the
sub-aperture flux is below 1e-3 of the mean.  Output layout [sx..., sy...].

The option attributes the reference sets after construction (:48-60) are
read at each trigger: thr_pedestal, thr_ratio_value, winMatWindowed,
mult_factor; quadcell_mode, weightedPixRad and windowing act through
set_xy_weights(), and vecWeiPixRadT switches weightedPixRad in time
(:136-143).  thr_ratio_value is each sub-aperture's fraction of its largest
windowed pixel, as the reference's per-sub-aperture loop computes it
(:231-232); the array form at :375-377 indexes a scalar and raises.  The
weighted CoG mask without windowing is the Gaussian of psf_gaussian
(:440-445) with FWHM weightedPixRad, the call :121 means to make (it passes
three arguments to a two-argument method and raises).  Templates,
correlation and two-step CoG (the reference's calc_slopes_for branch) are
not on this path.
"""
import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.subap_data import SubapData
from specula_b200.lib.make_mask import make_mask
from specula_b200.processing_objects.slopec import Slopec


class _LazyReduction(BaseValue):
    """BaseValue whose value is a reduction of the flux vector, computed on access."""

    def __init__(self, source, fn, **kw):
        super().__init__(**kw)
        self._source = source
        self._fn = fn

    @property
    def value(self):
        v = self._source.value
        return None if v is None else self._fn(v)


class ShSlopec(Slopec):
    def __init__(self,
                 subapdata: SubapData,
                 sn=None,
                 thr_value: float = -1,
                 exp_weight: float = 1.0,
                 filtmat=None,
                 corr_template=None,
                 target_device_idx: int = None,
                 precision: int = None):
        super().__init__(sn=sn, filtmat=filtmat, target_device_idx=target_device_idx, precision=precision)
        if corr_template is not None:
            raise NotImplementedError('ShSlopec: correlation templates are not on the specula_b200 path')
        self.thr_value = thr_value
        self.exp_weight = exp_weight
        self.subapdata = subapdata
        self.thr_ratio_value = 0.0
        self.thr_pedestal = False
        self.mult_factor = 0.0
        self.winMatWindowed = None
        self.quadcell_mode = False
        self.weightedPixRad = 0.0
        self.windowing = False
        self.vecWeiPixRadT = None
        self._win_src = None
        self._win = None
        self.xweights = None
        self.slopes.resize(subapdata.n_subaps * 2)
        self.total_counts = _LazyReduction(self.flux_per_subaperture_vector, torch.sum,
                                           target_device_idx=target_device_idx)
        self.subap_counts = _LazyReduction(self.flux_per_subaperture_vector, torch.mean,
                                           target_device_idx=target_device_idx)
        self.set_xy_weights()
        self.outputs['out_subapdata'] = self.subapdata

    @property
    def subap_idx(self):
        return self.subapdata.idxs

    def computeXYweights(self, np_sub, exp_weight, weightedPixRad=0.0, quadcell_mode=False, windowing=False):
        """x/y CoG weights on linspace(-1, 1) (sh_slopec.py:86-132): the
        exponential law, or the signs in quad-cell mode; xc/yc the two-step
        centroid weights; a weighted mask for weightedPixRad != 0 (a window
        of diameter 2 * weightedPixRad pixels, or the Gaussian of FWHM
        weightedPixRad normalised to its peak), entries below 1e-6 zeroed and
        the x/y weights multiplied by it."""
        v = np.linspace(-1, 1, np_sub)
        x, y = np.meshgrid(v, v)
        if quadcell_mode:
            x = np.where(x > 0, 1.0, -1.0)
            y = np.where(y > 0, 1.0, -1.0)
            xc, yc = x, y
        else:
            xc, yc = x, y
            x = np.where(x > 0, np.power(x, exp_weight), -np.power(np.abs(x), exp_weight))
            y = np.where(y > 0, np.power(y, exp_weight), -np.power(np.abs(y), exp_weight))
        xc = np.where(x > 0, xc, -np.abs(xc))
        yc = np.where(y > 0, yc, -np.abs(yc))
        if weightedPixRad != 0:
            if windowing:
                mask = make_mask(np_sub, diaratio=2.0 * weightedPixRad / np_sub).astype(np.float64)
            else:
                mask = self.psf_gaussian(np_sub, [weightedPixRad, weightedPixRad])
                mask = mask / np.max(mask)
            mask[mask < 1e-6] = 0.0
            x = x * mask.astype(np.float32)
            y = y * mask.astype(np.float32)
        else:
            mask = np.ones((np_sub, np_sub))
        return {'x': x, 'y': y, 'xc': xc, 'yc': yc, 'mask_weighted': mask}

    @staticmethod
    def psf_gaussian(np_sub, fwhm):
        """Gaussian on the [-1, 1] grid with FWHM fwhm[0] (sh_slopec.py:440-445)."""
        v = np.linspace(-1, 1, np_sub)
        x, y = np.meshgrid(v, v)
        return np.exp(-4 * np.log(2) * (x ** 2 + y ** 2) / fwhm[0] ** 2, dtype=np.float32)

    def set_xy_weights(self):
        """Recomputes the weights from the option attributes.  After setup the
        device buffers are rewritten in place, so a captured step graph sees
        the new weights at its next replay."""
        w = self.computeXYweights(self.subapdata.np_sub, self.exp_weight, self.weightedPixRad, self.quadcell_mode,
                                  self.windowing)
        new = {k: self._tensor(np.asarray(w[k]).ravel()) for k in ('x', 'y', 'xc', 'yc', 'mask_weighted')}
        if self.xweights is not None and self.xweights.device == new['x'].device:
            for name, k in (('xweights', 'x'), ('yweights', 'y'), ('xcweights', 'xc'), ('ycweights', 'yc'),
                            ('mask_weighted', 'mask_weighted')):
                getattr(self, name).copy_(new[k])
        else:
            self.xweights, self.yweights = new['x'], new['y']
            self.xcweights, self.ycweights = new['xc'], new['yc']
            self.mask_weighted = new['mask_weighted']

    def options_plain(self):
        """True when no option beyond thr_value and the weights is on."""
        return (not self.thr_pedestal and not self.thr_ratio_value > 0 and self.winMatWindowed is None and
                not self.mult_factor)

    def _sync_options(self):
        """Copies the option attributes into the launch plan (calc_slopes_nofor
        reads them at every call, sh_slopec.py:326-418)."""
        if self.thr_value > 0 and self.thr_ratio_value > 0:
            raise ValueError('Only one between _thr_value and _thr_ratio_value can be set.')
        pl = self._plan
        pl.thr = float(self.thr_value) if self.thr_value > 0 else 0.0
        pl.thr_pedestal = 1 if self.thr_pedestal else 0
        pl.thr_ratio = float(self.thr_ratio_value) if self.thr_ratio_value > 0 else 0.0
        pl.mult = float(self.mult_factor)
        if self.winMatWindowed is not self._win_src:
            n, npx2 = self.subapdata.idxs.shape
            if self.winMatWindowed is None:
                self._win = None
            else:
                w = np.asarray(self.winMatWindowed, dtype=np.float32)
                if w.size != npx2 * n:
                    raise ValueError(f'ShSlopec: winMatWindowed has {w.size} values, the sub-apertures '
                                     f'{npx2} x {n}')
                self._win = torch.as_tensor(w.reshape(npx2, n), device=self.device).contiguous()
            self._win_src = self.winMatWindowed
        pl.window = None if self._win is None else self._win.data_ptr()
        pl.xw, pl.yw, pl.mw = self.xweights.data_ptr(), self.yweights.data_ptr(), self.mask_weighted.data_ptr()

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        sd = self.subapdata
        n, npx2 = sd.idxs.shape
        pix = self.inputs['in_pixels'].get(self.target_device_idx)
        npix = pix.pixels.numel()
        if sd.idxs.min() < 0 or sd.idxs.max() >= npix:
            raise ValueError(f'ShSlopec: sub-aperture indices outside the {pix.size} frame')
        self._idxs = torch.as_tensor(sd.idxs.astype(np.int32), device=self.device).contiguous()
        self._flux = torch.zeros(n, dtype=self.dtype, device=self.device)
        self.flux_per_subaperture_vector.value = self._flux
        self._plan = _lib.SlopecPlan(n_subaps=n, npx2=npx2, idxs=self._idxs.data_ptr())
        self._sync_options()
        nb = _lib.load().sb_slopec_scratch_bytes(self._plan)
        self._scratch = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self._pix = pix
        self._target = self._setup_products(2 * n)
        self.slopes.single_mask = sd.single_mask()
        self.slopes.display_map = sd.display_map

    def trigger_code(self):
        if self.vecWeiPixRadT is not None:
            # rows (weightedPixRad, start time [s]): the last row whose time has passed
            vec = np.asarray(self.vecWeiPixRadT, dtype=np.float64)
            idx = np.where(self.current_time_seconds > vec[:, 1])[0]
            if len(idx) > 0 and vec[idx[-1], 0] != self.weightedPixRad:
                self.weightedPixRad = float(vec[idx[-1], 0])
                self.set_xy_weights()
        self._sync_options()
        st = self.stream_handle()
        _lib.call('sb_slopec', _byref(self._plan), self._pix.pixels.data_ptr(), self._target.data_ptr(),
                  self._flux.data_ptr(), self._scratch.data_ptr(), self._scratch.numel(), st)
        self._apply_products(st)

    def post_trigger(self):
        t = self.current_time
        self.slopes.generation_time = t
        self.flux_per_subaperture_vector.generation_time = t
        self.total_counts.generation_time = t
        self.subap_counts.generation_time = t


def _byref(s):
    import ctypes
    return ctypes.byref(s)
