"""Slope computer base (mirrors specula/processing_objects/slopec.py:9-101)."""
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.pixels import Pixels
from specula_b200.data_objects.slopes import Slopes


class Slopec(BaseProcessingObj):
    def __init__(self, sn: Slopes = None, use_sn: bool = False, accumulate: bool = False,
                 weight_from_accumulated: bool = False, recmat=None, filt_intmat=None, filt_recmat=None,
                 filtmat=None, accumulation_dt: float = 0, accumulated_pixels: tuple = (0, 0),
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if use_sn and not sn:
            raise ValueError('Slopes null are not valid')
        if weight_from_accumulated and accumulate:
            raise ValueError('weightFromAccumulated and accumulate must not be set together')
        for flag, what in ((accumulate, 'accumulation'), (weight_from_accumulated, 'weights from accumulation')):
            if flag:
                raise NotImplementedError(f'{type(self).__name__}: {what} is not on the specula_b200 path')
        self.recmat = recmat
        if filtmat is not None:
            if filt_intmat:
                raise ValueError('filt_intmat must not be set if "filtmat" is set')
            if filt_recmat:
                raise ValueError('filt_recmat must not be set if "filtmat" is set')
            from specula_b200.data_objects.intmat import Intmat
            from specula_b200.data_objects.recmat import Recmat
            filt_intmat = Intmat(filtmat[0], target_device_idx=target_device_idx)
            filt_recmat = Recmat(filtmat[1], target_device_idx=target_device_idx)
        elif (filt_intmat is not None) != (filt_recmat is not None):
            raise ValueError('Both filt_intmat and filt_recmat must be set for slopes filtering')
        self.filt_intmat = filt_intmat
        self.filt_recmat = filt_recmat
        self.slopes = Slopes(2, target_device_idx=target_device_idx, precision=precision)
        # slope nulls are stored but never subtracted, as in the reference (slopec.py:37-40)
        self.sn = sn
        self.use_sn = use_sn
        self.flux_per_subaperture_vector = BaseValue(target_device_idx=target_device_idx)
        self.max_flux_per_subaperture_vector = BaseValue(target_device_idx=target_device_idx)
        self.inputs['in_pixels'] = InputValue(type=Pixels)
        self.outputs['out_slopes'] = self.slopes

    # -- post-trigger products of slopec.py:92-101, on the device ------------
    def _setup_products(self, n_slopes):
        """Buffers of the optional slope products; returns the vector the slope
        kernel must write (the output slopes, or a raw buffer when a
        slope->mode reconstructor replaces them)."""
        import torch
        f32 = dict(device=self.device, dtype=torch.float32)
        self._raw = None
        self._RmT = None
        length = n_slopes
        if self.recmat is not None:
            Rm = torch.as_tensor(self.recmat.recmat).to(**f32)          # n_slopes x n_out: slopes @ recmat
            if Rm.shape[0] != n_slopes:
                raise ValueError(f'{type(self).__name__}: recmat {tuple(Rm.shape)} for {n_slopes} slopes')
            self._RmT = Rm.t().contiguous()
            self._raw = torch.zeros(n_slopes, **f32)
            length = Rm.shape[1]
            self.slopes.resize(length)
        self._RfT = self._IMf = None
        if self.filt_recmat is not None:
            Rf = torch.as_tensor(self.filt_recmat.recmat).to(**f32)      # length x n_filt
            IMf = torch.as_tensor(self.filt_intmat.intmat).to(**f32)     # length x n_filt
            if Rf.shape[0] != length or IMf.shape != Rf.shape:
                raise ValueError(f'{type(self).__name__}: filtering matrices {tuple(Rf.shape)} / '
                                 f'{tuple(IMf.shape)} for {length} slopes')
            self._RfT = Rf.t().contiguous()
            self._IMf = IMf.contiguous()
            self._filt_modes = torch.zeros(Rf.shape[1], **f32)
            self._filt_slopes = torch.zeros(length, **f32)
        return self._raw if self._raw is not None else self.slopes.slopes

    def _apply_products(self, stream):
        """slopes @ recmat, then slopes -= (slopes @ R_f) @ IM_f^T, as GEMVs."""
        from specula_b200 import _lib
        out = self.slopes.slopes
        if self._RmT is not None:
            R = self._RmT
            _lib.call('sb_modalrec', R.data_ptr(), R.shape[0], R.shape[1], R.stride(0), self._raw.data_ptr(),
                      out.data_ptr(), stream)
        if self._RfT is not None:
            R, IM = self._RfT, self._IMf
            _lib.call('sb_modalrec', R.data_ptr(), R.shape[0], R.shape[1], R.stride(0), out.data_ptr(),
                      self._filt_modes.data_ptr(), stream)
            _lib.call('sb_modalrec', IM.data_ptr(), IM.shape[0], IM.shape[1], IM.stride(0),
                      self._filt_modes.data_ptr(), self._filt_slopes.data_ptr(), stream)
            out.sub_(self._filt_slopes)
