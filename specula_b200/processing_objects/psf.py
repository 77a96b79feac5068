"""PSF and Strehl ratio on the B200 (mirrors specula/processing_objects/psf.py:17-137).

Same constructor, input (``in_ef``) and outputs (``out_sr``, ``out_psf``) as
the reference, plus the ``int_sr`` / ``int_psf`` values it integrates after
``start_time``.

* Strehl ratio: sb_strehl, one fused reduction over the pupil
  (|sum A e^{i phi}|^2 / (sum A)^2, which is exactly the reference's centre
  pixel of the normalised PSF over that of the flat-phase reference).
* PSF image: the reference zero-pads the field to N = round(M nd / 2) * 2,
  FFTs and fftshifts it.  Here the padding never materialises:
  F = W u W^T with the N x M pruned DFT matrix W whose rows are already in
  fftshift order, as two real GEMMs on the tensor cores (sb_psf_tc:
  tcgen05 with split-BF16 operands and FP32 accumulation), the field built
  in the first launch, |F|^2 / total (Parseval's total N^2 sum |u|^2) and
  the integration in the last GEMM's epilogue.
"""
import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.electric_field import ElectricField


def psf_size(dim, nd):
    """Padded PSF size (psf.py:46-52): round(dim * nd / 2) * 2."""
    return int(np.around(dim * nd / 2) * 2)


class PSF(BaseProcessingObj):
    def __init__(self, wavelengthInNm: float, nd: float = 1, start_time: float = 0.0, target_device_idx: int = None,
                 precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if wavelengthInNm <= 0:
            raise ValueError('PSF wavelength must be >0')
        self.nd = nd
        self.start_time = start_time
        self.wavelengthInNm = wavelengthInNm
        self.sr = BaseValue(target_device_idx=target_device_idx)
        self.int_sr = BaseValue(target_device_idx=target_device_idx)
        self.psf = BaseValue(target_device_idx=target_device_idx)
        self.int_psf = BaseValue(target_device_idx=target_device_idx)
        self.inputs['in_ef'] = InputValue(type=ElectricField)
        self.outputs['out_sr'] = self.sr
        self.outputs['out_psf'] = self.psf
        self._integrating = False

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        in_ef = self.inputs['in_ef'].get(self.target_device_idx)
        m = in_ef.size[0]
        if in_ef.size[0] != in_ef.size[1]:
            raise NotImplementedError('PSF: square electric fields only')
        n = psf_size(m, self.nd)
        if n < m:
            raise ValueError(f'PSF: padded size {n} smaller than the field ({m})')
        dev = self.device
        self.out_size = [n, n]
        self._m, self._n = m, n
        lib = _lib.load()
        # the DFT operand (split-BF16, pre-tiled for the tensor cores), built once on the device
        self._dft = torch.empty(lib.sb_psf_tc_dft_bytes(m, n), dtype=torch.uint8, device=dev)
        _lib.call('sb_psf_tc_prepare', m, n, self._dft.data_ptr(), self._dft.numel(),
                  torch.cuda.current_stream(dev).cuda_stream)
        self._tc_scratch = torch.zeros(lib.sb_psf_tc_scratch_bytes(m, n), dtype=torch.uint8, device=dev)
        self.psf.value = torch.zeros((n, n), dtype=torch.float32, device=dev)
        self.int_psf.value = torch.zeros((n, n), dtype=torch.float32, device=dev)
        self.sr.value = torch.zeros((), dtype=torch.float32, device=dev)
        self._int_sr = torch.zeros(2, dtype=torch.float64, device=dev)     # running sum, count
        self.int_sr.value = torch.zeros((), dtype=torch.float64, device=dev)
        self._scratch = torch.zeros(_lib.load().sb_psf_scratch_bytes(), dtype=torch.uint8, device=dev)
        self._k = float(np.float32((2 * np.pi) / self.wavelengthInNm))
        self._in_ef = in_ef

    def reset_integration(self):
        self.int_psf.value.zero_()
        self._int_sr.zero_()

    def prepare_trigger(self, t):
        super().prepare_trigger(t)
        self._integrating = self.current_time_seconds >= self.start_time

    def trigger_code(self):
        ef = self._in_ef
        st = self.stream_handle()
        npx = ef.A.numel()
        _lib.call('sb_strehl', ef.A.data_ptr(), ef.phaseInNm.data_ptr(), npx, self._k, self.sr.value.data_ptr(),
                  self._int_sr.data_ptr(), int(self._integrating), self._scratch.data_ptr(), self._scratch.numel(), st)
        _lib.call('sb_psf_tc', ef.A.data_ptr(), ef.phaseInNm.data_ptr(), self._m, self._n, self._k,
                  self._dft.data_ptr(), self.psf.value.data_ptr(),
                  self.int_psf.value.data_ptr() if self._integrating else None, self._tc_scratch.data_ptr(),
                  self._tc_scratch.numel(), st)
        if self._integrating:
            torch.div(self._int_sr[0], self._int_sr[1], out=self.int_sr.value)

    def post_trigger(self):
        super().post_trigger()
        t = self.current_time
        self.psf.generation_time = t
        self.sr.generation_time = t
        if self._integrating:
            self.int_psf.generation_time = t
            self.int_sr.generation_time = t
