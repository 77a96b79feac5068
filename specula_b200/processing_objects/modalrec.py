"""Modal reconstructor on the B200 (mirrors specula/processing_objects/modalrec.py:9-186).

Non-POLC path: ``modes = R @ slopes`` with R (n_modes x n_slopes), one
sb_modalrec call (HBM-streaming GEMV).  ``in_slopes_list`` inputs are
concatenated into a device buffer first.  POLC and projection matrices are
not on this path.
"""
import torch

from specula_b200 import _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputList, InputValue
from specula_b200.data_objects.recmat import Recmat
from specula_b200.data_objects.slopes import Slopes


class Modalrec(BaseProcessingObj):
    def __init__(self, nmodes: int = None, recmat: Recmat = None, projmat: Recmat = None, intmat=None,
                 polc: bool = False, filtmat=None, identity: bool = False, ncutmodes: int = None,
                 nSlopesToBeDiscarded: int = None, dmNumber: int = 0, noProj: bool = False,
                 input_modes_index: list = None, input_modes_slice: list = None, output_slice: list = None,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if polc or projmat is not None:
            raise NotImplementedError('Modalrec: POLC / projection matrices are not on the specula_b200 path')
        if recmat is None:
            if identity:
                if nmodes is None:
                    raise ValueError('modalrec nmodes key must be set!')
                recmat = Recmat(torch.eye(nmodes), target_device_idx=target_device_idx, precision=precision)
            elif intmat is not None:
                if nmodes:
                    intmat.reduce_size(intmat.size[0] - nmodes)
                if nSlopesToBeDiscarded:
                    intmat.reduce_slopes(nSlopesToBeDiscarded)
                recmat = Recmat(intmat.intmat, target_device_idx=target_device_idx, precision=precision)
        if ncutmodes and recmat is not None:
            recmat.reduce_size(ncutmodes)
        if filtmat is not None and recmat is not None:
            recmat.recmat = recmat.recmat @ torch.as_tensor(filtmat, dtype=recmat.recmat.dtype,
                                                            device=recmat.recmat.device)
        self.recmat = recmat
        self.intmat = intmat
        self.polc = polc
        if output_slice is not None:
            self.output_slice = slice(*output_slice)
        else:
            self.output_slice = slice(None, None, None)
        n_out = len(range(*self.output_slice.indices(self.recmat.recmat.shape[0])))
        self.modes = BaseValue('output modes from modal reconstructor', target_device_idx=target_device_idx)
        self.pseudo_ol_modes = BaseValue('output POL modes from modal reconstructor',
                                         target_device_idx=target_device_idx)
        self.inputs['in_slopes'] = InputValue(type=Slopes, optional=True)
        self.inputs['in_slopes_list'] = InputList(type=Slopes, optional=True)
        self.outputs['out_modes'] = self.modes
        self.outputs['out_pseudo_ol_modes'] = self.pseudo_ol_modes
        self._all_modes = torch.zeros(self.recmat.recmat.shape[0], dtype=self.dtype, device=self.device)
        self.modes.value = self._all_modes[self.output_slice]
        self.pseudo_ol_modes.value = torch.zeros(n_out, dtype=self.dtype, device=self.device)

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        s = self.inputs['in_slopes'].get(self.target_device_idx)
        sl = self.inputs['in_slopes_list'].get(self.target_device_idx)
        if not s and (not sl or not all(sl)):
            raise ValueError("Either 'slopes' or 'slopes_list' must be given as an input")
        if self.recmat is None:
            raise ValueError('Recmat object not valid')
        R = self.recmat.recmat
        if R.dtype != torch.float32 or not R.is_contiguous() or R.device != self.device:
            R = R.to(device=self.device, dtype=torch.float32).contiguous()
        self._R = R
        n_sl = s.size if s is not None else sum(x.size for x in sl)
        if n_sl != R.shape[1]:
            raise ValueError(f'Modalrec: {n_sl} slopes for a {tuple(R.shape)} reconstructor')
        self._slopes_buf = None if s is not None else torch.zeros(n_sl, dtype=self.dtype, device=self.device)

    def trigger_code(self):
        s = self.local_inputs.get('in_slopes')
        if s is not None:
            vec = s.slopes
        else:
            vec = self._slopes_buf
            off = 0
            for x in self.local_inputs['in_slopes_list']:
                vec[off:off + x.size].copy_(x.slopes)
                off += x.size
        _lib.call('sb_modalrec', self._R.data_ptr(), self._R.shape[0], self._R.shape[1], self._R.stride(0),
                  vec.data_ptr(), self._all_modes.data_ptr(), self.stream_handle())

    def post_trigger(self):
        self.modes.generation_time = self.current_time
