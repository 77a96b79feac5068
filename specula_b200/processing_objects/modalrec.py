"""Modal reconstructor on the B200 (mirrors specula/processing_objects/modalrec.py:9-186).

Non-POLC path: ``modes = R @ slopes`` with R (n_modes x n_slopes), one
sb_modalrec call (HBM-streaming GEMV).  ``in_slopes_list`` inputs are
concatenated into a device buffer first.

POLC (modalrec.py:126-156): with the commands c of ``in_commands`` (zeros
until they arrive), the pseudo-open-loop slopes s + IM c (added in place to
the input slopes, as the reference does), their modes R s
(``out_pseudo_ol_modes``; without a projection matrix the reference's
in-place subtraction leaves R s - c there) and the output (P R s or R s) - c,
where P is the optional projection matrix: up to three sb_modalrec GEMVs and
two device axpys.
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
        if polc:
            if identity:
                raise ValueError('identity cannot be set with POLC.')
            if ncutmodes is not None:
                raise ValueError('ncutmodes cannot be set with POLC.')
            if recmat is None or intmat is None:
                raise ValueError('Modalrec: POLC needs recmat and intmat')
        elif recmat is None:
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
        self.projmat = projmat
        self.intmat = intmat
        self.polc = polc
        self.input_modes_index = input_modes_index
        self.input_modes_slice = slice(*input_modes_slice) if input_modes_slice is not None else None
        if output_slice is not None:
            self.output_slice = slice(*output_slice)
        else:
            self.output_slice = slice(None, None, None)
        # the projection matrix only enters the POLC form (modalrec.py:150-154)
        n_all = projmat.recmat.shape[0] if (polc and projmat is not None) else self.recmat.recmat.shape[0]
        n_out = len(range(*self.output_slice.indices(n_all)))
        self.modes = BaseValue('output modes from modal reconstructor', target_device_idx=target_device_idx)
        self.pseudo_ol_modes = BaseValue('output POL modes from modal reconstructor',
                                         target_device_idx=target_device_idx)
        self.inputs['in_slopes'] = InputValue(type=Slopes, optional=True)
        self.inputs['in_slopes_list'] = InputList(type=Slopes, optional=True)
        self.outputs['out_modes'] = self.modes
        self.outputs['out_pseudo_ol_modes'] = self.pseudo_ol_modes
        self._all_modes = torch.zeros(n_all, dtype=self.dtype, device=self.device)
        self.modes.value = self._all_modes[self.output_slice]
        self.pseudo_ol_modes.value = torch.zeros(self.recmat.recmat.shape[0] if polc else n_out, dtype=self.dtype,
                                                 device=self.device)
        if polc:
            self.out_comm = BaseValue('output commands from modal reconstructor', target_device_idx=target_device_idx)
            self.inputs['in_commands'] = InputValue(type=BaseValue, optional=True)
            self.inputs['in_commands_list'] = InputList(type=BaseValue, optional=True)

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
        if self.polc:
            dev32 = dict(device=self.device, dtype=torch.float32)
            self._IM = torch.as_tensor(self.intmat.intmat).to(**dev32).contiguous()
            self._P = None if self.projmat is None else \
                torch.as_tensor(self.projmat.recmat).to(**dev32).contiguous()
            n_cmd = self._IM.shape[1]
            if self._IM.shape[0] != n_sl:
                raise ValueError(f'Modalrec: interaction matrix {tuple(self._IM.shape)} for {n_sl} slopes')
            if self._P is not None and (self._P.shape[1] != R.shape[0] or self._P.shape[0] != n_cmd):
                raise ValueError('Modalrec: projection matrix must be (n_commands x n_modes)')
            if self._P is None and R.shape[0] != n_cmd:
                raise ValueError('Modalrec: the reconstructor must give one mode per command')
            self._cmd = torch.zeros(n_cmd, **dev32)
            self._comm_slopes = torch.zeros(n_sl, **dev32)

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
        st = self.stream_handle()
        if not self.polc:
            _lib.call('sb_modalrec', self._R.data_ptr(), self._R.shape[0], self._R.shape[1], self._R.stride(0),
                      vec.data_ptr(), self._all_modes.data_ptr(), st)
            return
        self._load_commands()
        IM, R = self._IM, self._R
        _lib.call('sb_modalrec', IM.data_ptr(), IM.shape[0], IM.shape[1], IM.stride(0), self._cmd.data_ptr(),
                  self._comm_slopes.data_ptr(), st)
        vec.add_(self._comm_slopes)                      # pseudo-open-loop slopes, in place as the reference
        pol = self.pseudo_ol_modes.value
        _lib.call('sb_modalrec', R.data_ptr(), R.shape[0], R.shape[1], R.stride(0), vec.data_ptr(), pol.data_ptr(),
                  st)
        if self._P is None:
            # the reference subtracts the commands in place from the array it
            # also publishes as the pseudo-open-loop modes (modalrec.py:150-155)
            pol.sub_(self._cmd)
            self._all_modes.copy_(pol)
        else:
            P = self._P
            _lib.call('sb_modalrec', P.data_ptr(), P.shape[0], P.shape[1], P.stride(0), pol.data_ptr(),
                      self._all_modes.data_ptr(), st)
            self._all_modes.sub_(self._cmd)

    def _load_commands(self):
        """The commands of this step (modalrec.py:127-145): zeros until the first
        ones arrive, then optionally indexed / sliced."""
        obj = self.local_inputs.get('in_commands')
        lst = self.local_inputs.get('in_commands_list')
        if obj is not None and obj.value is not None:
            c = torch.as_tensor(obj.value).reshape(-1)
        elif lst and all(x.value is not None for x in lst):
            c = torch.cat([torch.as_tensor(x.value).reshape(-1) for x in lst])
        else:
            self._cmd.zero_()
            return
        if self.input_modes_index is not None:
            c = c[torch.as_tensor(self.input_modes_index, device=c.device)]
        if self.input_modes_slice is not None:
            c = c[self.input_modes_slice]
        if c.numel() != self._cmd.numel():
            raise ValueError(f'Modalrec: {c.numel()} commands for a {tuple(self._IM.shape)} interaction matrix')
        self._cmd.copy_(c.to(device=self.device, dtype=torch.float32))

    def post_trigger(self):
        self.modes.generation_time = self.current_time
        if self.polc:
            self.pseudo_ol_modes.generation_time = self.current_time
