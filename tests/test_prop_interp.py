"""Propagation through interpolated layers (atmo_propagation.py:104-209),
host side on CPU: the sample coordinates AtmoPropagation builds for an LGS at
90 km (cone effect), an off-axis NGS and an off-axis LGS over shifted,
rotated and magnified layers, bilinearly interpolated here with SciPy's
RegularGridInterpolator (the reference's CPU path), give the reference's
fields (tests/golden/prop_fp32.npz, make_golden.py --prop) within 1e-6."""
import numpy as np
import pytest
from scipy.interpolate import RegularGridInterpolator

from tests.cases import rel_max_err

SPECS = [(0.0, (0.0, 0.0), 0.0, 1.0), (4000.0, (1.5, -2.0), 0.0, 1.0), (9000.0, (0.0, 0.0), 10.0, 1.0),
         (12000.0, (0.0, 0.0), 0.0, 1.3)]
SOURCES = {'lgs': ([0.0, 0.0], 90e3, 589.0), 'ngs_off': ([30.0, 45.0], float('inf'), 750.0),
           'lgs_off': ([20.0, -60.0], 90e3, 589.0)}


@pytest.fixture(scope='module')
def prop_golden():
    import os
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'prop_fp32.npz')) as z:
        return {k: z[k] for k in z.files}


def build(device_idx, g):
    import torch
    from specula_b200.data_objects.simul_params import SimulParams
    from specula_b200.data_objects.layer import Layer
    from specula_b200.data_objects.pupilstop import Pupilstop
    from specula_b200.data_objects.source import Source
    from specula_b200.processing_objects.atmo_propagation import AtmoPropagation
    sp = SimulParams(pixel_pupil=64, pixel_pitch=0.05, time_step=0.001)
    layers = []
    for k, (h, sh, rot, mag) in enumerate(SPECS):
        lay = Layer(160, 160, 0.05, h, shiftXYinPixel=sh, rotInDeg=rot, magnification=mag,
                    target_device_idx=device_idx)
        lay.phaseInNm.copy_(torch.as_tensor(g['prop/layer%d/phase' % k]))
        lay.A.copy_(torch.as_tensor(g['prop/layer%d/A' % k]))
        layers.append(lay)
    pup = Pupilstop(sp, mask_diam=1.0, obs_diam=0.14, target_device_idx=device_idx)
    sources = {n: Source(pc, 8.0, lam, height=h, phot_density_value=1.0) for n, (pc, h, lam) in SOURCES.items()}
    prop = AtmoPropagation(sp, sources, target_device_idx=device_idx)
    prop.inputs['atmo_layer_list'].set(layers)
    prop.inputs['common_layer_list'].set([pup])
    return prop, layers, pup, sources


def test_coordinates_and_bilinear_match_reference(prop_golden):
    g = prop_golden
    prop, layers, pup, sources = build(-1, g)
    assert np.array_equal(pup.A.numpy(), g['prop/pupil_A'])
    for name, src in sources.items():
        A = np.ones((64, 64), np.float32)
        P = np.zeros((64, 64), np.float32)
        for k, lay in enumerate(layers + [pup]):
            on_axis = lay.height == 0 or (np.isinf(src.height) and src.r == 0)
            plain = not np.any(lay.shiftXYinPixel) and lay.rotInDeg == 0 and max(lay.magnification, 1.0) == 1
            a, p = lay.A.numpy().astype(np.float32), lay.phaseInNm.numpy().astype(np.float32)
            if on_axis and plain:
                t = (lay.size[0] - 64) // 2
                A *= a[t:t + 64, t:t + 64]
                P += p[t:t + 64, t:t + 64]
                continue
            p = p.copy()
            p[a == 0] = np.mean(p[a != 0])
            yy, xx = prop._layer_coords(src, lay)
            pts = (np.arange(lay.size[0], dtype=np.float32), np.arange(lay.size[1], dtype=np.float32))
            for v, out in ((a, 'A'), (p, 'P')):
                val = RegularGridInterpolator(pts, v, method='linear')((yy, xx)).reshape(64, 64).astype(np.float32)
                if out == 'A':
                    A *= val
                else:
                    P += val
        assert rel_max_err(A, g['prop/%s/A' % name]) <= 1e-6, name
        assert rel_max_err(P, g['prop/%s/phase' % name]) <= 1e-6, name


def test_source_outside_the_layers_is_rejected(prop_golden):
    from specula_b200.data_objects.source import Source
    prop, layers, pup, sources = build(-1, prop_golden)
    with pytest.raises(ValueError, match='FoV'):
        prop._layer_coords(Source([200.0, 0.0], 8.0, 750.0, phot_density_value=1.0), layers[3])
