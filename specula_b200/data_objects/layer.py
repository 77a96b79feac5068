"""Phase layer at a given height (mirrors specula/data_objects/layer.py:6-52)."""
import numpy as np

from specula_b200.data_objects.electric_field import ElectricField


class Layer(ElectricField):
    def __init__(self, dimx: int, dimy: int, pixel_pitch: float, height: float,
                 shiftXYinPixel: tuple = (0.0, 0.0), rotInDeg: float = 0.0, magnification: float = 1.0,
                 target_device_idx: int = None, precision: int = None):
        super().__init__(dimx, dimy, pixel_pitch, target_device_idx=target_device_idx, precision=precision)
        self.height = height
        self.shiftXYinPixel = np.array(shiftXYinPixel, dtype=np.float32 if self.precision == 1 else np.float64)
        self.rotInDeg = rotInDeg
        self.magnification = magnification
