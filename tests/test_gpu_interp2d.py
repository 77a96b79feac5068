"""sb_interp2d_field against the reference's Interp2D fixture
(test_interp2d.py:19-43: input_phase.fits -> ref_phase.fits, rtol 4e-2 with
its one known outlier pixel) and the oracle's float64 bilinear (<= 1e-6), and
the reference's boundary check (test_interp2d.py:45-60): a slice of a larger
array is never read beyond its rows."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from oracle import sh as osh  # noqa: E402
from tests.cases import rel_max_err  # noqa: E402
from tests.test_oracle_golden import _interp_fits_case  # noqa: E402

pytestmark = pytest.mark.gpu


def _interp(A, P, rows, cols, yy, xx):
    from specula_b200 import _lib
    yy_t = torch.as_tensor(yy, device='cuda').contiguous()
    xx_t = torch.as_tensor(xx, device='cuda').contiguous()
    Ao = torch.empty(yy.size, dtype=torch.float32, device='cuda')
    Po = torch.empty(yy.size, dtype=torch.float32, device='cuda')
    _lib.call('sb_interp2d_field', A.data_ptr(), P.data_ptr(), rows, cols, yy_t.data_ptr(), xx_t.data_ptr(),
              yy.size, Ao.data_ptr(), Po.data_ptr(), None)
    torch.cuda.synchronize()
    return Ao.cpu().numpy(), Po.cpu().numpy()


def test_interp2d_matches_reference_fits(cuda):
    phase, ref, yy, xx = _interp_fits_case()
    P = torch.as_tensor(phase, device='cuda').contiguous()
    _, got = _interp(P, P, phase.shape[0], phase.shape[1], yy, xx)
    got = got.reshape(ref.shape)
    assert rel_max_err(got, osh.interp2d(phase, yy, xx, ref.shape)) <= 1e-6
    got[394, 365] = ref[394, 365]
    np.testing.assert_allclose(got, ref, rtol=4e-2)


def test_interp2d_reads_only_its_rows(cuda):
    from specula_b200.lib.interp2d import interp_coords
    big = torch.full((20, 20), float('nan'), dtype=torch.float32, device='cuda')
    big[:10] = 1.0
    yy, xx = interp_coords((10, 20), (5, 5), rotInDeg=45)
    A, P = _interp(big, big, 10, 20, yy, xx)
    assert not np.isnan(A).any() and not np.isnan(P).any()
