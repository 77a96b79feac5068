"""Loop gradient through the closed SCAO loop (specula_b200.lib.loop_gradient):
checkpointed reverse mode against the same without checkpoints (bit-identical),
against central finite differences of the loop metric along random gain and
reconstructor directions, and the functional forward loop against the
object-by-object loop (noise-free detector).

Tolerances: gradient . direction vs central differences <= 1e-3 relative
(steps 2e-2 on unit gain directions, 0.25 on the reconstructor direction;
measured errors on these seeded directions 2e-5 .. 5e-5 and 3e-5: the
differences' truncation and the float32 loss set the floor); slopes of the
two forward loops <= 1e-4 (max|d|/max).
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

FD_TOL = 1e-3


def _cfg():
    from specula_b200.scao import ScaoConfig
    return ScaoConfig(heights=[0.0, 4000.0], cn2=[0.7, 0.3], wind_speed=[10.0, 25.0], wind_direction=[30.0, 212.7],
                      photon_noise=False, readout_noise=0.0, r0=0.12)


def _lg(T, K):
    from specula_b200.scao import ScaoLoop
    from specula_b200.lib.loop_gradient import LoopGradient
    loop = ScaoLoop(_cfg(), device_idx=0)
    return LoopGradient(loop, T, checkpoint_every=K), loop


def test_checkpointed_gradient_equals_unchecked(cuda):
    lg1, loop = _lg(24, 5)
    lg2, _ = _lg(24, 24)
    g = torch.full((lg1.nm,), 0.45, device='cuda')
    R = loop.rec._R.clone()
    L1, dg1, dR1 = lg1.gradient(g, R)
    L2, dg2, dR2 = lg2.gradient(g, R)
    assert L1 == L2
    assert torch.equal(dg1, dg2) and torch.equal(dR1, dR2)
    assert float(dg1.abs().max()) > 0


def test_gradient_matches_finite_differences(cuda):
    T = 40
    lg, loop = _lg(T, 10)
    rng = np.random.default_rng(5)
    g = torch.as_tensor(0.3 + 0.2 * rng.random(lg.nm), dtype=torch.float32, device='cuda')
    R = loop.rec._R.clone()
    L, dg, dR = lg.gradient(g, R)
    assert L == pytest.approx(lg.loss(g, R), rel=1e-12)
    for k in range(3):
        d = torch.as_tensor(rng.standard_normal(lg.nm), dtype=torch.float32, device='cuda')
        d /= d.norm()
        eps = 2e-2
        fd = (lg.loss(g + eps * d, R) - lg.loss(g - eps * d, R)) / (2 * eps)
        ad = float((dg.double() * d.double()).sum())
        assert abs(ad - fd) <= FD_TOL * abs(fd), (k, ad, fd)
    D = torch.as_tensor(rng.standard_normal(tuple(R.shape)), dtype=torch.float32, device='cuda')
    D *= 0.05 * float(R.norm()) / float(D.norm())
    eps = 0.25
    fd = (lg.loss(g, R + eps * D) - lg.loss(g, R - eps * D)) / (2 * eps)
    ad = float((dR.double() * D.double()).sum())
    assert abs(ad - fd) <= FD_TOL * abs(fd), (ad, fd)


def test_functional_forward_matches_object_loop(cuda):
    from specula_b200.scao import ScaoLoop
    T = 12
    lg, loop = _lg(T, 4)
    ref = ScaoLoop(_cfg(), device_idx=0)
    ref.start()
    slopes = []
    for _ in range(T):
        ref.step_eager()
        slopes.append(ref.slopec.slopes.slopes.clone())
    g = torch.full((lg.nm,), float(_cfg().gain), device='cuda')
    _, S, _ = lg.trajectory(g, ref.rec._R)
    for t in range(T):
        assert rel_max_err(S[t].cpu().numpy(), slopes[t].cpu().numpy()) <= 1e-4, t
