"""Laser launch telescope (mirrors specula/data_objects/laser_launch_telescope.py:3-33).

spot_size: laser spot size [arcsec]; tel_position: x, y, z of the launcher
with respect to the telescope [m] (empty: a Gaussian spot on axis);
beacon_focus: distance from the pupil to the beacon focus [m]; beacon_tt:
beacon tip and tilt [arcsec].
"""
from specula_b200.base_data_obj import BaseDataObj


class LaserLaunchTelescope(BaseDataObj):
    def __init__(self, spot_size: float = 0.0, tel_position: list = (), beacon_focus: float = 90e3,
                 beacon_tt: list = (0.0, 0.0), target_device_idx: int = None, precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self.spot_size = spot_size
        self.tel_pos = list(tel_position)
        self.beacon_focus = beacon_focus
        self.beacon_tt = list(beacon_tt)
