"""Valid sub-aperture detection (mirrors
specula/processing_objects/sh_subap_calibrator.py:10-92).

From one SH intensity frame: the flux of each lenslet's detector box,
lenslets above ``energy_th`` times the brightest are valid.  Boxes are
scanned lenslet-column first; each valid box contributes its pixels'
flattened row-major indices (rows from the lenslet's x coordinate, columns
from its y coordinate, as the reference's mask slicing does) and
``display_map = j * nx + i``.  The box sums run on the device; the
selection is host work on n_lenses^2 numbers.  The result is kept in
``self.subaps`` (SubapData); no FITS file is written.
"""
import numpy as np
import torch

from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.connections import InputValue
from specula_b200.data_objects.intensity import Intensity
from specula_b200.data_objects.lenslet import Lenslet
from specula_b200.data_objects.subap_data import SubapData


def lenslet_boxes(n_lenses, frame_side):
    """[(r0, r1, c0, c1)] per lenslet (i, j), i-major: the reference's
    round(center -/+ np_sub/2) box of lenslet (i, j) (sh_subap_calibrator.py:47-60)."""
    lens = Lenslet(n_lenses)
    boxes = []
    for i in range(lens.dimx):
        for j in range(lens.dimy):
            lx, ly, size = lens.get(i, j)
            x = frame_side / 2.0 * (1 + lx)
            y = frame_side / 2.0 * (1 + ly)
            np_sub = round(frame_side / 2.0 * size)
            boxes.append((int(np.round(x - np_sub / 2)), int(np.round(x + np_sub / 2)),
                          int(np.round(y - np_sub / 2)), int(np.round(y + np_sub / 2))))
    return boxes, np_sub


class ShSubapCalibrator(BaseProcessingObj):
    def __init__(self, subap_on_diameter: int, energy_th: float, data_dir: str = '', output_tag: str = None,
                 tag_template: str = None, target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self._n = subap_on_diameter
        self._energy_th = energy_th
        self._data_dir = data_dir
        if tag_template is None and (output_tag is None or output_tag == 'auto'):
            raise ValueError('At least one of tag_template and output_tag must be set')
        self._filename = tag_template if (output_tag is None or output_tag == 'auto') else output_tag
        self.subaps = None
        self.inputs['in_i'] = InputValue(type=Intensity)

    def trigger_code(self):
        self.subaps = self.detect_subaps(self.local_inputs['in_i'].i, self._energy_th)

    def detect_subaps(self, image, energy_th):
        image = torch.as_tensor(image)
        side = image.shape[0]
        n = self._n
        boxes, np_sub = lenslet_boxes(n, side)
        flux = torch.stack([image[r0:r1, c0:c1].to(torch.float64).sum() for r0, r1, c0, c1 in boxes])
        flux = flux.cpu().numpy().reshape(n, n)
        sel = flux > energy_th * flux.max()
        idxs, dmap = [], []
        for i in range(n):
            for j in range(n):
                if sel[i, j]:
                    r0, r1, c0, c1 = boxes[i * n + j]
                    rr, cc = np.meshgrid(np.arange(r0, r1), np.arange(c0, c1), indexing='ij')
                    idxs.append((rr * image.shape[1] + cc).ravel())
                    dmap.append(j * n + i)
        if not idxs:
            raise ValueError('Error: no subapertures selected')
        return SubapData(idxs=np.array(idxs, dtype=np.int64), display_map=np.array(dmap, dtype=np.int64),
                         nx=n, ny=n, energy_th=energy_th, target_device_idx=self.target_device_idx,
                         precision=self.precision)
