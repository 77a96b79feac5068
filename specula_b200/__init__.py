"""specula_b200 — B200-native closed-loop Shack-Hartmann step with SPECULA's
processing-object API.

The package mirrors the module layout of the reference
(``specula.processing_objects.<snake_case>``, ``specula.data_objects.<...>``)
so YAML-style class lookup finds the same class names.  Device arrays are
torch tensors on a CUDA device; every ``trigger_code`` calls the C ABI of
``libspecula_b200.so`` (hand-written sm_100a kernels) on the current torch
stream.  There is no CPU fallback.

Global defaults follow specula/__init__.py:36-95: ``init(device_idx,
precision)``; ``precision=0`` is float64 and ``precision=1`` float32.  The GPU
hot path computes in float32 (precision=1); float64 is accepted by the data
containers but the processing objects reject it.
"""
import numpy as np

ASEC2RAD = np.pi / (3600 * 180)
RAD2ASEC = 1.0 / ASEC2RAD

global_precision = 1
default_target_device_idx = 0


def init(device_idx=0, precision=1):
    """Set the default CUDA device index and precision (0: float64, 1: float32)."""
    global global_precision, default_target_device_idx
    if precision not in (0, 1):
        raise ValueError('precision must be 0 (float64) or 1 (float32)')
    global_precision = precision
    default_target_device_idx = device_idx


def cpuArray(v):
    """Host NumPy copy of a tensor / array / scalar (specula/__init__.py:97-102)."""
    try:
        import torch
        if isinstance(v, torch.Tensor):
            return v.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return np.array(v)
