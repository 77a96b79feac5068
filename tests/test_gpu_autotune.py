"""Tile-shape variants and the autotuner on the GPU.

Every variant of a tunable family computes the same result as variant 0:
bit-identical where only the tiling changes (realisations per pass of the
batched mirror with one mode-row group, and its register-blocked forms,
which keep every column's mode order; sub-apertures per CTA of the FP32
SH); every batched-mirror variant within 1e-5 of the largest value of a
float64 product (two mode-row groups change the FP32 summation order: about
1e-6 with 500 random modes).  The autotuner registers one
of them and its JSON cache is reused by a second tuner.
"""
import ctypes
import json

import numpy as np
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu


def _dm_problem(nm, nv, L, B, seed):
    gen = torch.Generator(device='cuda').manual_seed(seed)
    ld = (nv + 31) // 32 * 32
    IF = torch.zeros((nm, ld), device='cuda')
    IF[:, :nv] = torch.randn((nm, nv), device='cuda', generator=gen)
    idx = torch.as_tensor(np.random.default_rng(seed).permutation(L * L)[:nv].astype(np.int32), device='cuda')
    C = torch.randn((B, nm), device='cuda', generator=gen)
    return IF, ld, idx, C


# batched-mirror variants that sum every column's modes in order from 0
MODE_ORDER_VARIANTS = (0, 2, 4, 6, 7, 8, 9, 10, 11)


@pytest.mark.parametrize('nm,nv,B', [(37, 5003, 3), (500, 40000, 7), (300, 20011, 16), (54, 9000, 19)])
def test_dm_batched_variants_agree(cuda, nm, nv, B):
    from specula_b200 import _lib
    lib = _lib.load()
    L = 256
    IF, ld, idx, C = _dm_problem(nm, nv, L, B, seed=nm + B)
    key = lib.sb_tune_key(nm, nv, B)
    st = torch.cuda.current_stream().cuda_stream
    outs = []
    try:
        for v in range(lib.sb_tune_variants(_lib.SB_TUNE_DM_BATCHED)):
            _lib.call('sb_tune_set', _lib.SB_TUNE_DM_BATCHED, key, v)
            ph = torch.zeros((B, L * L), device='cuda')
            _lib.call('sb_dm_project_batched', IF.data_ptr(), nm, nv, ld, C.data_ptr(), nm, B, -1.0, idx.data_ptr(),
                      ph.data_ptr(), L * L, st)
            torch.cuda.synchronize()
            outs.append(ph)
    finally:
        _lib.call('sb_tune_set', _lib.SB_TUNE_DM_BATCHED, key, -1)
    _lib.call('sb_device_status')
    ref64 = (-(C.double() @ IF[:, :nv].double()))
    scale = float(ref64.abs().max())
    for v, o in enumerate(outs):
        assert float((o[:, idx.long()].double() - ref64).abs().max()) <= 1e-5 * scale, v
        if v in MODE_ORDER_VARIANTS:
            assert torch.equal(o, outs[0]), v


@pytest.mark.parametrize('nm,nsl,B', [(54, 496, 28), (500, 8618, 7), (37, 5003, 19)])
def test_modalrec_batched_variants_bit_identical(cuda, nm, nsl, B):
    """Rows per CTA change only which CTA computes a row: every variant gives
    the same bits, within 1e-5 of float64 (odd slope counts take the scalar loads)."""
    from specula_b200 import _lib
    lib = _lib.load()
    gen = torch.Generator(device='cuda').manual_seed(nm)
    R = torch.randn((nm, nsl), device='cuda', generator=gen)
    S = torch.randn((B, nsl), device='cuda', generator=gen)
    key = lib.sb_tune_key(nm, nsl, B)
    outs = []
    try:
        for v in range(lib.sb_tune_variants(_lib.SB_TUNE_MODALREC_BATCHED)):
            _lib.call('sb_tune_set', _lib.SB_TUNE_MODALREC_BATCHED, key, v)
            M = torch.full((B, nm), float('nan'), device='cuda')
            _lib.call('sb_modalrec_batched', R.data_ptr(), nm, nsl, nsl, S.data_ptr(), nsl, B, M.data_ptr(), nm,
                      torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            outs.append(M)
    finally:
        _lib.call('sb_tune_set', _lib.SB_TUNE_MODALREC_BATCHED, key, -1)
    ref = S.double() @ R.double().t()
    assert float((outs[0].double() - ref).abs().max()) <= 1e-5 * float(ref.abs().max())
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


@pytest.mark.parametrize('which', ['elt80', 'c1_plain16', 'n16_fft16'])
def test_sh_fp32_variants_bit_identical(cuda, which):
    """The TMA-staged SB_TUNE_SH_FP32 variants (0-2) give the frames of the
    variants reading the field directly with the same sub-apertures per CTA
    (3-5) bit for bit; the CTA sizes agree to 1e-6 (the photon normalisation sums per-CTA
    partials, so its last rounding can follow the CTA size).  20 lenslets
    leave a partial last column block for 8 per CTA."""
    from specula_b200 import _lib
    from tests.cases import SH_CASES, rel_max_err
    from tests.test_gpu_sh_split_bf16 import _sh, _elt_case, _turbulent_phase
    from oracle.masks import make_mask
    lib = _lib.load()
    case = _elt_case(16) if which == 'elt80' else next(c for c in SH_CASES if c[0] == which)
    pix = case[1]
    A = make_mask(pix, 0.14, 1.0).astype(np.float32)
    _, sh = _sh(case, A, np.zeros_like(A), 'fp32')
    At = torch.as_tensor(A, device='cuda')
    ph = torch.as_tensor(_turbulent_phase(pix, 3, 1.5, case[3]), device='cuda') * At
    side = case[6] * case[7]
    nbytes = lib.sb_sh_scratch_bytes(ctypes.byref(sh._plan))
    scratch = torch.zeros(nbytes, dtype=torch.uint8, device='cuda')
    key = lib.sb_tune_key(sh._plan.n_lenses, sh._plan.cutsize, 1)
    outs = []
    try:
        for v in range(lib.sb_tune_variants(_lib.SB_TUNE_SH_FP32)):
            _lib.call('sb_tune_set', _lib.SB_TUNE_SH_FP32, key, v)
            out = torch.empty((side, side), device='cuda')
            _lib.call('sb_sh_forward', ctypes.byref(sh._plan), At.data_ptr(), ph.data_ptr(), At.data_ptr(), pix * pix,
                      7.0 * case[2] ** 2, out.data_ptr(), scratch.data_ptr(), nbytes, 0)
            torch.cuda.synchronize()
            outs.append(out)
    finally:
        _lib.call('sb_tune_set', _lib.SB_TUNE_SH_FP32, key, -1)
    assert len(outs) == 6
    for v in range(3):
        assert torch.equal(outs[v + 3], outs[v]), v
        assert rel_max_err(outs[v].cpu().numpy(), outs[0].cpu().numpy()) <= 1e-6, v
    assert float(outs[0].abs().max()) > 0
    _lib.call('sb_device_status')


def test_autotuner_registers_and_caches(cuda, tmp_path):
    from specula_b200 import _lib
    from specula_b200.autotune import Autotuner
    lib = _lib.load()
    nm, nv, L, B = 200, 30000, 256, 7
    IF, ld, idx, C = _dm_problem(nm, nv, L, B, seed=5)
    ph = torch.zeros((B, L * L), device='cuda')
    cache = tmp_path / 'tune.json'
    key = lib.sb_tune_key(nm, nv, B)
    try:
        t1 = Autotuner('cuda:0', cache_path=str(cache), reps=2, launches=3)
        r1 = t1.tune_dm_batched(IF, nm, nv, ld, C, nm, B, 1.0, idx, ph, L * L)
        assert not r1['cached'] and all(r1['agrees_with_variant0'])
        assert lib.sb_tune_get(_lib.SB_TUNE_DM_BATCHED, key) == r1['variant']
        assert r1['times_us'][r1['variant']] == min(t for t in r1['times_us'] if t is not None)
        saved = json.loads(cache.read_text())
        assert len(saved) == 1
        _lib.call('sb_tune_set', _lib.SB_TUNE_DM_BATCHED, key, -1)
        t2 = Autotuner('cuda:0', cache_path=str(cache))
        r2 = t2.tune_dm_batched(IF, nm, nv, ld, C, nm, B, 1.0, idx, ph, L * L)
        assert r2['cached'] and r2['variant'] == r1['variant']
        assert lib.sb_tune_get(_lib.SB_TUNE_DM_BATCHED, key) == r1['variant']
    finally:
        _lib.call('sb_tune_set', _lib.SB_TUNE_DM_BATCHED, key, -1)
