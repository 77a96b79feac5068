"""Batched Monte-Carlo realisations (specula_b200.batched): one CUDA graph
for every realisation with the group-shared reconstructor and mirror run as
batched launches (sb_modalrec_batched, sb_dm_project_batched, one integrator
call), against the same realisations run the plain way (each its own step
graph, reconstructor and mirror).  Noise included (counter-based RNG keyed by
each realisation's seeds).

Tolerance: slopes max|d|/max <= 1e-4 per realisation per step (the batched
reconstructor sums in another order).
"""
from dataclasses import replace

import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu


def _groups(noise=True):
    from specula_b200.scao import ScaoConfig
    base = ScaoConfig(heights=[0.0, 4000.0], cn2=[0.7, 0.3], wind_speed=[10.0, 25.0],
                      wind_direction=[30.0, 212.7], n_modes=20, photon_noise=noise,
                      readout_noise=3.0 if noise else 0.0)
    groups = []
    k = 0
    for lam, n in ((589.0, 3), (750.0, 5)):
        reals = []
        for i in range(n):
            reals.append(replace(base, wavelength_nm=lam, r0=0.09 + 0.02 * i, screen_seed=10 + k, noise_seed=500 + 7 * k))
            k += 1
        groups.append((replace(base, wavelength_nm=lam), reals))
    return groups


@pytest.mark.parametrize('noise', [False, True])
def test_batched_graph_matches_plain_realisations(cuda, noise):
    """Noise-free: slopes within 1e-4 over 6 steps.  With photon and read-out
    noise: the first graph step (inputs still identical) bit-identical; later
    steps differ once a Poisson draw flips on the last-bit differences of the
    batched reconstructor's summation order, so they are not compared."""
    from specula_b200.batched import BatchedScao
    plain = BatchedScao(_groups(noise))
    plain.start()
    plain.capture_plain()
    bat = BatchedScao(_groups(noise))
    bat.start()
    bat.capture()          # one eager batched step, as capture_plain() ran one per loop
    torch.cuda.synchronize()
    for step in range(5 if not noise else 1):
        ref = plain.slopes()
        got = bat.slopes()
        for gi, (a, b) in enumerate(zip(ref, got)):
            for r in range(a.shape[0]):
                assert float(a[r].abs().max()) > 0
                if noise:
                    assert torch.equal(a[r], b[r]), (step, gi, r)
                else:
                    assert rel_max_err(b[r].cpu().numpy(), a[r].cpu().numpy()) <= 1e-4, (step, gi, r)
        plain.replay_plain()
        bat.replay()
        torch.cuda.synchronize()


def test_batched_split_bf16_matches_plain_fp32(cuda):
    """The batched graph with the split-BF16 tensor-core SH against the plain
    FP32 realisations, noise-free: slopes within 1e-4 over 6 closed-loop
    steps (the SH alone is within 2e-5 of float64)."""
    from specula_b200.batched import BatchedScao
    plain = BatchedScao(_groups(False))
    plain.start()
    plain.capture_plain()
    bat = BatchedScao(_groups(False), dft='split_bf16')
    bat.start()
    bat.capture()
    torch.cuda.synchronize()
    worst = 0.0
    for step in range(5):
        for a, b in zip(plain.slopes(), bat.slopes()):
            for r in range(a.shape[0]):
                e = rel_max_err(b[r].cpu().numpy(), a[r].cpu().numpy())
                worst = max(worst, e)
                assert e <= 1e-4, (step, r, e)
        plain.replay_plain()
        bat.replay()
        torch.cuda.synchronize()
    print(f'batched split-BF16 vs plain FP32: worst slope error {worst:.2e}')
    with pytest.raises(ValueError):
        bat.set_dft('fp64')


def test_batched_dm_projection_matches_single(cuda):
    """sb_dm_project_batched row b equals sb_dm_project with command b
    (bit-identical: same per-column summation order), for 1..19 rows."""
    import numpy as np
    from specula_b200 import _lib
    nm, nv, L = 37, 5003, 80
    ld = (nv + 31) // 32 * 32
    gen = torch.Generator(device='cuda').manual_seed(3)
    IF = torch.zeros((nm, ld), device='cuda')
    IF[:, :nv] = torch.randn((nm, nv), device='cuda', generator=gen)
    idx = torch.as_tensor(np.random.default_rng(1).permutation(L * L)[:nv].astype(np.int32), device='cuda')
    st = torch.cuda.current_stream().cuda_stream
    for B in (1, 4, 7, 16, 19):
        C = torch.randn((B, nm), device='cuda', generator=gen)
        out = torch.zeros((B, L, L), device='cuda')
        _lib.call('sb_dm_project_batched', IF.data_ptr(), nm, nv, ld, C.data_ptr(), nm, B, -1.0, idx.data_ptr(),
                  out.data_ptr(), L * L, st)
        for b in range(B):
            ref = torch.zeros((L, L), device='cuda')
            _lib.call('sb_dm_project', IF.data_ptr(), nm, nv, ld, C[b].contiguous().data_ptr(), nm, -1.0,
                      idx.data_ptr(), ref.data_ptr(), st)
            assert torch.equal(out[b], ref), (B, b)
        # reconstructor: slope rows of odd length (scalar loads) and padded to 16 bytes (vector loads)
        for lds in (nv, ld):
            M = torch.empty((B, nm), device='cuda')
            S = torch.randn((B, lds), device='cuda', generator=gen)
            _lib.call('sb_modalrec_batched', IF.data_ptr(), nm, nv, ld, S.data_ptr(), lds, B, M.data_ptr(), nm, st)
            ref = S[:, :nv].double() @ IF[:, :nv].double().t()
            assert rel_max_err(M.cpu().numpy(), ref.cpu().numpy()) <= 1e-5, (B, lds)
    _lib.call('sb_device_status')


def test_fused_atmosphere_propagation_matches_two_launches(cuda):
    """sb_atmo_propagate_batched (layers and field in one launch) against
    sb_atmo_evolve_batched + sb_propagate_batched: layers and field
    bit-identical over three steps, with more realisations than one launch
    of 64 layers holds (2 layers x 40 realisations)."""
    from specula_b200.batched import BatchedScao
    from specula_b200.scao import ScaoConfig
    base = ScaoConfig(heights=[0.0, 4000.0], cn2=[0.7, 0.3], wind_speed=[10.0, 25.0],
                      wind_direction=[30.0, 212.7], n_modes=20, photon_noise=False, readout_noise=0.0)
    reals = [replace(base, r0=0.08 + 0.003 * i, screen_seed=10 + i, noise_seed=100 + i) for i in range(40)]
    systems = []
    for fused in (True, False):
        b = BatchedScao([(base, reals)])
        b.groups[0].fuse_atmo = fused
        b.start()
        systems.append(b)
    for step in range(3):
        for b in systems:
            b.step_eager()
        torch.cuda.synchronize()
        f, t = systems[0].groups[0], systems[1].groups[0]
        assert float(t.EP.abs().max()) > 0
        assert torch.equal(f.ATM, t.ATM), step
        assert torch.equal(f.EA, t.EA), step
        assert torch.equal(f.EP, t.EP), step
