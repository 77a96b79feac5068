"""Von Karman phase-screen synthesis, float64 on the GPU.

Same construction as specula/lib/calc_phasescreen.py:6-105: uniform draws
from NumPy's RandomState(seed) (host, so the random stream is the
reference's), Box-Muller Gaussians, a Hermitian-symmetric spectrum
arrangement, the von Karman amplitude (f^2 + 1/L0^2)^(-11/12) times the
normalisation constant, and an inverse 2-D FFT (norm='forward').  The
arithmetic after the draws runs in float64 on the device (the reference
computes in the object precision); the inverse FFT is cuFFT through
torch.fft, a setup-time library call outside the loop.
"""
import math

import numpy as np
import torch


def calc_phasescreen(L0, dimension, pixel_pitch, seed=0, device='cuda'):
    n = int(math.ceil(math.log2(float(dimension))))
    dim = 2 ** n
    h = dim // 2
    m_dim = dim * pixel_pitch
    rng = np.random.RandomState(seed)
    draws = [torch.as_tensor(rng.random((h + 1, 2 * h + 1)), device=device) for _ in range(4)]
    u1, v1, u2, v2 = draws
    re = torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * v1)
    im = torch.sqrt(-2.0 * torch.log(u2)) * torch.cos(2.0 * math.pi * v2)
    del draws, u1, v1, u2, v2
    ps = torch.zeros((dim, dim), dtype=torch.complex128, device=device)
    ps[h:2 * h, 0:2 * h] = torch.complex(re[1:h + 1, 1:2 * h + 1], im[1:h + 1, 1:2 * h + 1])
    re_r = torch.flip(re, (0, 1))
    im_r = torch.flip(im, (0, 1))
    ps[0:h - 1, 0:2 * h] = torch.complex(re_r[1:h, 1:2 * h + 1], -im_r[1:h, 1:2 * h + 1])
    ps[h, 0:h] = torch.complex(re[0, 1:h + 1], im[0, 1:h + 1])
    ps[h, h:2 * h] = torch.complex(torch.flip(re, (0,))[0, 0:h], -torch.flip(im, (0,))[0, 0:h])
    ps[2 * h - 1, :] = 0
    ps[:, 2 * h - 1] = 0
    c = torch.arange(dim, dtype=torch.float64, device=device) - (h - 1)
    f2 = (c[:, None] ** 2 + c[None, :] ** 2) / m_dim ** 2
    ps *= (f2 + 1.0 / float(L0) ** 2) ** (-11. / 12.)
    ps *= math.sqrt(0.033 / 2. / m_dim ** 2) * (2 * math.pi) ** (2. / 3.) * math.sqrt(0.06) * \
        (1 / pixel_pitch) ** (5. / 6.)
    ps = torch.roll(ps, (-h + 1, -h + 1), dims=(0, 1))
    ps = torch.fft.ifft2(ps, norm='forward')
    ps = torch.roll(ps, (h - 1, h - 1), dims=(0, 1))
    return ps.real.contiguous()
