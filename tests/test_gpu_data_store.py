"""DataStore on the GPU: device-side copies, batched non-blocking moves to
pinned host memory, same files as on CPU."""
import os

import numpy as np
import pytest

from tests.golden import fits_min
from tests.test_data_store import run_store

pytestmark = pytest.mark.gpu


def test_store_on_gpu(cuda, tmp_path):
    ds, want, times = run_store(tmp_path, 'fits', 0, steps=7, flush_steps=3)
    for name, arr in want.items():
        (h0, d0), (h1, d1) = fits_min.read_hdus(os.path.join(ds.tn_dir, name + '.fits'))
        assert np.array_equal(d0, arr) and np.array_equal(d1, times)
