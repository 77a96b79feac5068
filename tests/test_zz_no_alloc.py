"""The no-allocation SH entry point (sb_sh_forward_static).

It exists for callers that cannot allocate device memory, such as a
real-time control thread that must not allocate once the loop runs, or a
foreign-language binding that owns its input and output buffers but has no
CUDA allocator.  Its scratch is a fixed-size device array inside the library.
This file is collected last so that a failure here stops a ``-x`` run only
after every other test has run; it must also pass alone in a fresh process
(the first call on the device resolves the array's address).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import SH_CASES, rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

INTENSITY_TOL = 1e-5   # same tolerance as the SH parity tests


def _setup(case):
    from specula_b200.processing_objects.sh import SH
    from specula_b200.data_objects.electric_field import ElectricField
    name, pix, pitch, lam, fov, pxs, n, npx, coeff = case
    sh = SH(wavelengthInNm=lam, subap_wanted_fov=fov, sensor_pxscale=pxs, subap_on_diameter=n, subap_npx=npx,
            fov_ovs_coeff=coeff, target_device_idx=0)
    ef = ElectricField(pix, pix, pitch, S0=3.0, target_device_idx=0)
    from oracle.masks import make_mask
    ef.A.copy_(torch.as_tensor(make_mask(pix, 0.14, 1.0).astype(np.float32)))
    ef.generation_time = 1
    sh.inputs['in_ef'].set(ef)
    sh.setup()
    return sh, ef


@pytest.mark.parametrize('case', [c for c in SH_CASES if c[8] == 1.0], ids=lambda c: c[0])
def test_static_scratch_entry_matches_caller_scratch_entry(case, cuda):
    from specula_b200 import _lib
    sh, ef = _setup(case)
    st = torch.cuda.current_stream().cuda_stream
    plan = ctypes.byref(sh._plan)
    out_ref = torch.empty_like(sh.outputs['out_i'].i)
    out_new = torch.empty_like(out_ref)
    rng = np.random.default_rng(42)
    for call in range(2):       # two calls in a row, each with a new phase
        ph = (rng.standard_normal(ef.phaseInNm.shape) * 80).astype(np.float32)
        ef.phaseInNm.copy_(torch.as_tensor(ph, device=ef.A.device) * ef.A)
        out_new.fill_(float('nan'))
        _lib.call('sb_sh_forward', plan, ef.A.data_ptr(), ef.phaseInNm.data_ptr(), ef.A.data_ptr(), ef.A.numel(),
                  sh._photon_scale, out_ref.data_ptr(), sh._scratch.data_ptr(), sh._scratch.numel(), st)
        _lib.call('sb_sh_forward_static', plan, ef.A.data_ptr(), ef.phaseInNm.data_ptr(), ef.A.data_ptr(),
                  ef.A.numel(), sh._photon_scale, out_new.data_ptr(), st)
        torch.cuda.synchronize()
        a, b = out_new.cpu().numpy(), out_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call
        assert rel_max_err(a, b) <= INTENSITY_TOL, call


def test_static_scratch_rejects_oversized_geometry(cuda):
    from specula_b200 import _lib
    sh, ef = _setup([c for c in SH_CASES if c[0] == 'n16_fft16'][0])
    big = _lib.ShPlan.from_buffer_copy(sh._plan)
    big.n_lenses = 2048                   # far beyond the static array; nothing is launched
    lib = _lib.load()
    rc = lib.sb_sh_forward_static(ctypes.byref(big), ef.A.data_ptr(), ef.phaseInNm.data_ptr(), ef.A.data_ptr(),
                                  ef.A.numel(), ctypes.c_float(1.0), sh.outputs['out_i'].i.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == -4
    assert b'static array' in lib.sb_last_error()
