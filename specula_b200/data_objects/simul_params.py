"""Global simulation parameters (mirrors specula/data_objects/simul_params.py)."""
from dataclasses import dataclass


@dataclass
class SimulParams:
    pixel_pupil: int = None
    pixel_pitch: float = None
    root_dir: str = '.'
    total_time: float = 0.1
    time_step: float = 0.001
    zenithAngleInDeg: float = 0
    display_server: bool = False
