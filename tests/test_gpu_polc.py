"""Modalrec POLC on the GPU against the reference (tests/golden/polc_fp32.npz,
make_golden.py --polc): pseudo-open-loop slopes added in place to the input,
pseudo-open-loop modes and output modes over three steps (zeros for the
commands before they arrive), without and with a projection matrix; within
1e-5 (three float32 GEMVs)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('case', ['plain', 'proj'])
def test_polc_matches_reference(cuda, case):
    from specula_b200.processing_objects.modalrec import Modalrec
    from specula_b200.data_objects.recmat import Recmat
    from specula_b200.data_objects.intmat import Intmat
    from specula_b200.data_objects.slopes import Slopes
    from specula_b200.base_value import BaseValue
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'polc_fp32.npz')) as z:
        g = {k: z[k] for k in z.files}
    R, P, IM = g['polc/R'], g['polc/P'], g['polc/%s/IM' % case]
    rec = Modalrec(recmat=Recmat(R, target_device_idx=0), intmat=Intmat(IM, target_device_idx=0), polc=True,
                   projmat=Recmat(P, target_device_idx=0) if case == 'proj' else None, target_device_idx=0)
    sl = Slopes(R.shape[1], target_device_idx=0)
    cmd = BaseValue(target_device_idx=0)
    rec.inputs['in_slopes'].set(sl)
    rec.inputs['in_commands'].set(cmd)
    for t in range(3):
        sl.slopes.copy_(torch.as_tensor(g['polc/%s/slopes_in%d' % (case, t)]))
        sl.generation_time = t + 1
        if t > 0:
            cmd.value = torch.as_tensor(g['polc/%s/commands%d' % (case, t)], device='cuda')
            cmd.generation_time = t + 1
        if t == 0:
            rec.setup()
        rec.check_ready(t + 1)
        rec.trigger()
        rec.post_trigger()
        torch.cuda.synchronize()
        for got, key in ((sl.slopes, 'slopes_after'), (rec.modes.value, 'modes'), (rec.pseudo_ol_modes.value, 'pol')):
            ref = g['polc/%s/%s%d' % (case, key, t)]
            assert rel_max_err(got.cpu().numpy(), ref) <= 1e-5, (case, key, t)
