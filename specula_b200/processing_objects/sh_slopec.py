"""Shack-Hartmann slope computer on the B200 (mirrors
specula/processing_objects/sh_slopec.py:25-445).

``trigger_code()`` is one sb_slopec call implementing calc_slopes_nofor
(sh_slopec.py:308-438): gather each valid sub-aperture through
``SubapData.idxs``, subtract the threshold and clamp at 0, weighted CoG with
the weights of computeXYweights (:86-132), factor zeroed where the
sub-aperture flux is below 1e-3 of the mean.  Output layout [sx..., sy...].
Templates, correlation, windowing and two-step CoG (the reference's
calc_slopes_for branch) are not on this path.
"""
import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.subap_data import SubapData
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

    def computeXYweights(self, np_sub, exp_weight):
        """x/y CoG weights on linspace(-1, 1) with the exponential law of
        sh_slopec.py:98-113; mask weights are ones (no windowing)."""
        v = np.linspace(-1, 1, np_sub)
        x, y = np.meshgrid(v, v)
        x = np.where(x > 0, np.power(x, exp_weight), -np.power(np.abs(x), exp_weight))
        y = np.where(y > 0, np.power(y, exp_weight), -np.power(np.abs(y), exp_weight))
        return {'x': x, 'y': y, 'mask_weighted': np.ones((np_sub, np_sub))}

    def set_xy_weights(self):
        w = self.computeXYweights(self.subapdata.np_sub, self.exp_weight)
        self.xweights = self._tensor(w['x'].ravel())
        self.yweights = self._tensor(w['y'].ravel())
        self.mask_weighted = self._tensor(w['mask_weighted'].ravel())

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
        self._plan = _lib.SlopecPlan(n_subaps=n, npx2=npx2, thr=float(self.thr_value) if self.thr_value > 0 else 0.0,
                                     idxs=self._idxs.data_ptr(), xw=self.xweights.data_ptr(),
                                     yw=self.yweights.data_ptr(), mw=self.mask_weighted.data_ptr())
        nb = _lib.load().sb_slopec_scratch_bytes(self._plan)
        self._scratch = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self._pix = pix
        self._target = self._setup_products(2 * n)
        self.slopes.single_mask = sd.single_mask()
        self.slopes.display_map = sd.display_map

    def trigger_code(self):
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
