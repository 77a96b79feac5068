"""Deformable mirror on the B200 (mirrors specula/processing_objects/dm.py:10-96).

``phase[mask] = (sign * m2c @ c) @ IF`` is one sb_dm_project call (plus a
sb_modalrec GEMV for m2c when given).  The influence functions are copied
once into a row-padded device layout (row stride a multiple of 32 floats) so
the projection streams them with aligned 16-byte loads.
"""
import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.ifunc import IFunc
from specula_b200.data_objects.layer import Layer


class DM(BaseProcessingObj):
    def __init__(self, simul_params, height: float, ifunc: IFunc = None, m2c=None, type_str: str = None,
                 nmodes: int = None, nzern: int = None, start_mode: int = None, input_offset: int = 0,
                 idx_modes=None, npixels: int = None, obsratio: float = None, diaratio: float = None,
                 pupilstop=None, sign: int = -1, target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.simul_params = simul_params
        self.pixel_pitch = simul_params.pixel_pitch
        mask = None
        if pupilstop:
            mask = pupilstop.A
            if npixels is None:
                npixels = mask.shape[0]
        if not ifunc:
            ifunc = IFunc(type_str=type_str, mask=mask, npixels=npixels, obsratio=obsratio, diaratio=diaratio,
                          nzern=nzern, nmodes=nmodes, start_mode=start_mode, idx_modes=idx_modes,
                          target_device_idx=target_device_idx, precision=precision)
        self._ifunc = ifunc
        s = tuple(ifunc.mask_inf_func.shape)
        nmodes_if = ifunc.size[0]
        self.if_commands = torch.zeros(nmodes_if, dtype=self.dtype, device=self.device)
        self.layer = Layer(s[0], s[1], self.pixel_pitch, height, target_device_idx=target_device_idx,
                           precision=precision)
        self.layer.A = ifunc.mask_inf_func.to(self.dtype)
        if m2c is not None:
            self.m2c = m2c.m2c
            self.m2c_commands = torch.zeros(m2c.m2c.shape[1], dtype=self.dtype, device=self.device)
        else:
            self.m2c = None
            self.m2c_commands = None
        self.input_offset = input_offset
        self.nmodes = nmodes
        self.sign = sign
        self.inputs['in_command'] = InputValue(type=BaseValue)
        self.outputs['out_layer'] = self.layer

    @property
    def ifunc(self):
        return self._ifunc.influence_function

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        IF = self._ifunc.influence_function
        nm, nv = IF.shape
        ld = (nv + 31) // 32 * 32
        buf = torch.zeros((nm, ld), dtype=torch.float32, device=self.device)
        buf[:, :nv] = IF.to(self.device, torch.float32)
        self._IF = buf
        self._ld = ld
        self._idx = torch.as_tensor(self._ifunc.idx_inf_func.astype(np.int32), device=self.device)
        if self._idx.numel() != nv:
            raise ValueError(f'DM: {nv} influence-function columns for {self._idx.numel()} mask pixels')
        if self.m2c is not None:
            self._m2c = self.m2c.to(self.device, torch.float32).contiguous()
            self._cmd = torch.zeros(self._m2c.shape[0], dtype=torch.float32, device=self.device)

    def trigger_code(self):
        self.project(self.local_inputs['in_command'].value, self.layer.phaseInNm)

    def project(self, c, out_phase, columns=None):
        """phase[mask] = (sign * m2c @ c) @ IF into ``out_phase`` (pix x pix).
        ``columns`` = (c0, c1): only influence-function columns c0 .. c1 - 1
        (c0 a multiple of 4), i.e. only those mask pixels."""
        if not isinstance(c, torch.Tensor) or c.device != self.device or c.dtype != torch.float32:
            c = torch.as_tensor(c, dtype=torch.float32, device=self.device)
        if self.nmodes is not None:
            c = c[self.input_offset:self.input_offset + self.nmodes]
        c = c.contiguous()
        st = self.stream_handle()
        if self.m2c is not None:
            self.m2c_commands[:c.numel()].copy_(c)
            _lib.call('sb_modalrec', self._m2c.data_ptr(), self._m2c.shape[0], self._m2c.shape[1],
                      self._m2c.stride(0), self.m2c_commands.data_ptr(), self._cmd.data_ptr(), st)
            c = self._cmd
        if out_phase.shape != self.layer.phaseInNm.shape or not out_phase.is_contiguous():
            raise ValueError('DM.project: output must be a contiguous array shaped like the layer')
        c0, c1 = (0, int(self._idx.numel())) if columns is None else columns
        if c0 % 4 or not 0 <= c0 <= c1 <= self._idx.numel():
            raise ValueError(f'DM.project: columns {columns} outside 0..{self._idx.numel()} or unaligned')
        _lib.call('sb_dm_project', self._IF.data_ptr() + 4 * c0, self._IF.shape[0], c1 - c0, self._ld,
                  c.data_ptr(), int(c.numel()), float(self.sign), self._idx.data_ptr() + 4 * c0,
                  out_phase.data_ptr(), st)

    def post_trigger(self):
        self.layer.generation_time = self.current_time
