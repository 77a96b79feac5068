"""Push-pull interaction-matrix accumulator (mirrors
specula/processing_objects/im_rec_calibrator.py:10-98).

Each step with fresh slopes, the non-zero command k (a FuncGenerator
'PUSHPULL' sequence, modal_pushpull_signal.py:35-65) adds ``slopes /
cmd_k`` to row k - first_mode of the matrix, so a +a / -a pair leaves
``(s(+a) - s(-a)) / a`` (im_rec_calibrator.py:58-63).  The accumulation is a
device axpy; finding the commanded mode reads the command vector back, as
the reference's ``xp.nonzero`` does.

``finalize()`` leaves the interaction matrix in ``self.intmat`` (Intmat,
n_modes x n_slopes) and, when a reconstructor tag is set, its float64
pseudo-inverse in ``self.rec`` in the orientation Modalrec consumes
(n_modes x n_slopes: the reference's saved-and-restored orientation,
recmat.py:40-68).  FITS files are not written.

``ShSlopesAdjoint.intmat`` / ``ShCalibrationSystem.adjoint_intmat`` give the
same matrix (small-amplitude limit) from the adjoint in two launches.
"""
import torch

from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.intmat import Intmat
from specula_b200.data_objects.recmat import Recmat
from specula_b200.data_objects.slopes import Slopes


class ImRecCalibrator(BaseProcessingObj):
    def __init__(self, nmodes: int, data_dir: str = '', rec_tag: str = '', im_tag: str = '', first_mode: int = 0,
                 pupdata_tag: str = None, tag_template: str = None, target_device_idx: int = None,
                 precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self._nmodes = nmodes
        self._first_mode = first_mode
        self._data_dir = data_dir
        if tag_template is None and (rec_tag is None or rec_tag == 'auto'):
            raise ValueError('At least one of tag_template and rec_tag must be set')
        self._rec_filename = tag_template if (rec_tag is None or rec_tag == 'auto') else rec_tag
        self._im_filename = im_tag
        self.pupdata_tag = pupdata_tag
        self._im = None
        self.intmat = None
        self.rec = None
        self.inputs['in_slopes'] = InputValue(type=Slopes)
        self.inputs['in_commands'] = InputValue(type=BaseValue)
        self.output_im = [Slopes(length=2, target_device_idx=target_device_idx) for _ in range(nmodes)]
        self.outputs['out_im'] = self.output_im

    def trigger_code(self):
        # slopes must have been refreshed this step (im_rec_calibrator.py:44-48)
        sl = self.local_inputs['in_slopes']
        if sl.generation_time != self.current_time:
            return
        slopes = sl.slopes
        commands = torch.as_tensor(self.local_inputs['in_commands'].value, device=self.device)
        if self._im is None:
            self._im = torch.zeros((self._nmodes, slopes.numel()), dtype=self.dtype, device=self.device)
            for i in range(self._nmodes):
                self.output_im[i].slopes = self._im[i]
        idx = torch.nonzero(commands.reshape(-1)).reshape(-1)
        if idx.numel() > 0:
            k = int(idx[0])
            mode = k - self._first_mode
            if 0 <= mode < self._nmodes:
                self._im[mode].add_(slopes.to(self.dtype) / commands.reshape(-1)[k].to(self.dtype))
        for o in self.output_im:
            o.single_mask = sl.single_mask
            o.display_map = sl.display_map
            o.generation_time = self.current_time

    def finalize(self):
        if self._im is None:
            return
        self.intmat = Intmat(self._im.clone(), pupdata_tag=self.pupdata_tag or '',
                             target_device_idx=self.target_device_idx, precision=self.precision)
        if self._rec_filename:
            im = self.intmat.intmat[:self._nmodes]
            pinv = torch.linalg.pinv(im.to(torch.float64))        # n_slopes x n_modes
            self.rec = Recmat(pinv.T.to(self.dtype).contiguous(), target_device_idx=self.target_device_idx,
                              precision=self.precision)
