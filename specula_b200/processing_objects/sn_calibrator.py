"""Slope-null calibrator (mirrors specula/processing_objects/sn_calibrator.py:8-37).

Keeps the last slopes it saw (a copy on the device) as ``self.slopes``; the
reference writes them to a FITS file at ``finalize()``, which is not done
here (FITS I/O is outside specula_b200).
"""
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.connections import InputValue
from specula_b200.data_objects.slopes import Slopes


class SnCalibrator(BaseProcessingObj):
    def __init__(self, data_dir: str = '', output_tag: str = None, tag_template: str = None,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self._data_dir = data_dir
        if tag_template is None and (output_tag is None or output_tag == 'auto'):
            raise ValueError('At least one of tag_template and output_tag must be set')
        self._filename = tag_template if (output_tag is None or output_tag == 'auto') else output_tag
        self.slopes = None
        self.inputs['in_slopes'] = InputValue(type=Slopes)

    def trigger_code(self):
        src = self.local_inputs['in_slopes']
        self.slopes = Slopes(slopes=src.slopes.clone(), target_device_idx=self.target_device_idx,
                             precision=self.precision)
        self.slopes.generation_time = src.generation_time
