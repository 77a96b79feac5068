import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200) and the built libspecula_b200.so')


@pytest.fixture(scope='session')
def golden():
    """Golden fixtures written by tests/golden/make_golden.py from the reference."""
    import json
    out = {}
    for name in ('ref_fits', 'sh_fp32', 'sh_fp64', 'chain_fp32', 'zernike_fp32', 'psf_fp32'):
        with np.load(os.path.join(GOLDEN, name + '.npz')) as z:
            out[name] = {k: z[k] for k in z.files}
    with open(os.path.join(GOLDEN, 'sh_geometry.json')) as f:
        out['geometry'] = json.load(f)
    return out


@pytest.fixture(scope='session')
def lgs():
    """Laser-guide-star fixtures (make_golden.py --lgs)."""
    with np.load(os.path.join(GOLDEN, 'lgs_fp32.npz')) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope='session')
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    from specula_b200 import _lib
    _lib.load()
    return torch.device('cuda', 0)
