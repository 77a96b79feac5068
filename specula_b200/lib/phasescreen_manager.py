"""Phase-screen cache (specula/lib/phasescreen_manager.py:8-58): one FITS file
per seed under ``directory``, named

    ps_seed{seed}_dim{dimension}_pixpit{pitch:.3f}_L0{L0:.4f}_{single|double}.fits

with the reference's three other spellings of the same name accepted when
reading (seed and L0 written as integers or floats).  A missing screen is
synthesised on the GPU (specula_b200.lib.phasescreen, float64) and written in
the object precision (float32 for 'single'), so caches are shared with the
reference in both directions.
"""
import os

import numpy as np
import torch

from specula_b200.lib import fits_io
from specula_b200.lib.phasescreen import calc_phasescreen


def _int_str(x):
    return str(int(np.around(x)))


def phasescreen_names(seed, dimension, pixel_pitch, L0, precision):
    """The file name the reference writes, then the alternatives it reads."""
    p = 'single' if precision == 1 else 'double'
    dim = _int_str(dimension)
    s_int, s_flt = _int_str(seed), str(float(seed))
    l_flt, l_int = f'{float(L0):.4f}', f'{float(np.around(L0)):.4f}'
    return [f'ps_seed{s_int}_dim{dim}_pixpit{pixel_pitch:.3f}_L0{l_flt}_{p}.fits',
            f'ps_seed{s_int}_dim{dim}_pixpit{pixel_pitch:.3f}_L0{l_int}_{p}.fits',
            f'ps_seed{s_flt}_dim{dim}_pixpit{pixel_pitch:.3f}_L0{l_flt}_{p}.fits',
            f'ps_seed{s_flt}_dim{dim}_pixpit{pixel_pitch:.3f}_L0{l_int}_{p}.fits']


def phasescreens_manager(L0, dimension, pixel_pitch, directory, precision=1, seed=(0,), device='cuda'):
    """Square screens for every seed: read from ``directory`` when cached,
    else synthesised and written there.  Returns device tensors (float32 for
    precision 1, float64 otherwise)."""
    L0 = np.atleast_1d(np.asarray(L0, dtype=np.float64))
    seeds = list(np.atleast_1d(seed))
    if len(L0) not in (1, len(seeds)):
        raise ValueError('The number of elements in L0 must be 1 or the same as the number of seeds!')
    os.makedirs(directory, exist_ok=True)
    dtype = torch.float32 if precision == 1 else torch.float64
    out = []
    for i, s in enumerate(seeds):
        L0i = float(L0[i] if len(L0) == len(seeds) else L0[0])
        names = phasescreen_names(s, dimension, pixel_pitch, L0i, precision)
        hit = next((n for n in names if os.path.exists(os.path.join(directory, n))), None)
        if hit is not None:
            screen = torch.as_tensor(fits_io.getdata(os.path.join(directory, hit)), device=device).to(dtype)
        else:
            screen = calc_phasescreen(L0i, dimension, pixel_pitch, seed=int(s), device=device).to(dtype)
            fits_io.writeto(os.path.join(directory, names[0]), screen.cpu().numpy(), overwrite=True)
        out.append(screen)
    return out
