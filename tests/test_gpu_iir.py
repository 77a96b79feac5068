"""General IIR filters (1 to 8 taps) through sb_integrator against the
reference's IirFilter (tests/golden/iir_fp32.npz, make_golden.py --iir):
integer and fractional delays, a lower-order row right-aligned by
IirFilterData, 6 steps; bit-exact (the reference's float32 operation order,
NumPy's summation order of the tap products)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu

CASES = [('taps3x3_d2', 2.0), ('taps4x2_d1.5', 1.5), ('taps8x8_d0', 0.0), ('taps1x1_d1', 1.0)]


@pytest.mark.parametrize('name,delay', CASES)
def test_general_iir_is_bit_exact(cuda, name, delay):
    from specula_b200.processing_objects.iir_filter import IirFilter
    from specula_b200.data_objects.iir_filter_data import IirFilterData
    from specula_b200.data_objects.simul_params import SimulParams
    from specula_b200.base_value import BaseValue
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'iir_fp32.npz')) as z:
        g = {k: z[k] for k in z.files}
    key = 'iir/' + name
    fd = IirFilterData(g[key + '/ordnum'], g[key + '/ordden'], g[key + '/num'], g[key + '/den'], target_device_idx=0)
    sp = SimulParams(pixel_pupil=8, pixel_pitch=0.1, time_step=0.001)
    filt = IirFilter(sp, fd, delay=delay, target_device_idx=0)
    n = g[key + '/num'].shape[0]
    d = BaseValue(value=torch.zeros(n, device='cuda'), target_device_idx=0)
    filt.inputs['delta_comm'].set(d)
    filt.setup()
    for t in range(6):
        d.value = torch.as_tensor(g[key + '/in%d' % t], device='cuda')
        d.generation_time = (t + 1) * 1000000
        filt.check_ready((t + 1) * 1000000)
        filt.trigger()
        filt.post_trigger()
        got = filt.out_comm.value.cpu().numpy()
        assert np.array_equal(got, g[key + '/out%d' % t]), (name, t, got, g[key + '/out%d' % t])
