"""ShSlopec slope filtering (slopec.py:92-101 through filtmat) on the GPU
against the reference (tests/golden/slopec_filt_fp32.npz, make_golden.py
--slopec-filter): the reference's own 8x8 sub-aperture table, two random
frames, slopes within 1e-4 of the largest; and the base class's
slope->mode reconstructor against a float64 product."""
import os

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(golden, **kw):
    from specula_b200.processing_objects.sh_slopec import ShSlopec
    from specula_b200.data_objects.subap_data import SubapData
    from specula_b200.data_objects.pixels import Pixels
    ref = golden['ref_fits']
    sd = SubapData(idxs=ref['subaps/idxs'], display_map=ref['subaps/display_map'], nx=8, ny=8, target_device_idx=0)
    sc = ShSlopec(sd, target_device_idx=0, **kw)
    pix = Pixels(64, 64, target_device_idx=0)
    sc.inputs['in_pixels'].set(pix)
    sc.setup()
    return sc, pix


def _step(sc, pix, frame, t):
    pix.pixels.copy_(torch.as_tensor(frame))
    pix.generation_time = t
    sc.check_ready(t)
    sc.trigger()
    sc.post_trigger()
    return sc.slopes.slopes.cpu().numpy()


def test_filtmat_matches_reference(golden, cuda):
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'slopec_filt_fp32.npz')) as z:
        g = {k: z[k] for k in z.files}
    sc, pix = _run(golden, filtmat=g['slopec_filt/filtmat'])
    for t in range(2):
        got = _step(sc, pix, g['slopec_filt/frame%d' % t], t + 1)
        assert rel_max_err(got, g['slopec_filt/slopes%d' % t]) <= 1e-4, t


def test_slope_to_mode_recmat(golden, cuda):
    from specula_b200.data_objects.recmat import Recmat
    rng = np.random.default_rng(4)
    plain, pix0 = _run(golden)
    frame = (rng.random((64, 64)) * 100).astype(np.float32)
    s = _step(plain, pix0, frame, 1).astype(np.float64)
    Rm = rng.standard_normal((s.size, 7)).astype(np.float32)
    sc, pix = _run(golden)
    sc.recmat = Recmat(Rm, target_device_idx=0)     # the slope->mode product is a Slopec base option
    sc.setup()
    got = _step(sc, pix, frame, 1)
    assert got.shape == (7,)
    assert rel_max_err(got, s @ Rm.astype(np.float64)) <= 1e-5
