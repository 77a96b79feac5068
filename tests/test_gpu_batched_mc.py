"""Monte-Carlo step over geometry groups (sb_mc_step): six launches per step,
each over every realisation of every group, against the group-by-group
graph of the same realisations (BatchedScao.capture), bit for bit, with the
FP32 and the split-BF16 SH.  The mix is the Monte-Carlo benchmark's three
geometries (20x20 / 160 px, 40x40 / 320 px, 74x74 / 592 px) at two
wavelengths, nine realisations in six groups."""
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu

N_REAL = (4, 3, 2)
STEPS = 3


def _state(sys_b):
    out = []
    for g in sys_b.groups:
        st = {k: getattr(g, k).clone() for k in ('ATM', 'EA', 'EP', 'I', 'INT', 'PIX', 'S', 'FLUX', 'M', 'dm_phase')}
        st['commands'] = g.integ.out_comm.value.clone()
        st['integ_state'] = g.integ.state.clone()
        st['positions'] = torch.cat([lp.atmo._positions.clone() for lp in g.loops])
        st['ccd_state'] = g.loops[0].ccd._state.clone()
        out.append(st)
    return out


def _run(dft, mc, pipelined=False, steps=STEPS):
    from specula_b200.batched import BatchedScao, mc_groups
    sys_b = BatchedScao(mc_groups(n_real=N_REAL), device_idx=0, dft=dft)
    sys_b.start()
    if mc:
        sys_b.capture_mc(pipelined=pipelined)
    else:
        sys_b.capture()
    assert steps % sys_b.steps_per_replay == 0
    for _ in range(steps // sys_b.steps_per_replay):
        sys_b.replay()
    torch.cuda.synchronize()
    from specula_b200 import _lib
    _lib.call('sb_device_status')
    return sys_b, _state(sys_b)


@pytest.mark.parametrize('dft', ['fp32', 'split_bf16'])
def test_mc_step_equals_group_graph(cuda, dft):
    ref_sys, ref = _run(dft, mc=False)
    mc_sys, got = _run(dft, mc=True)
    assert len(mc_sys.groups) == 6
    assert mc_sys.launches_per_step == 6
    assert ref_sys.launches_per_step > 8
    for gi, (a, b) in enumerate(zip(ref, got)):
        for k in a:
            assert torch.equal(a[k], b[k]), (dft, gi, k, float((a[k].double() - b[k].double()).abs().max()))
    # the loop moved: slopes and mirror non-trivial
    assert all(float(st['S'].abs().max()) > 0 for st in got)
    assert all(float(st['dm_phase'].abs().max()) > 0 for st in got)
    mc_sys.release_mc()


def test_pipelined_mc_step_equals_group_graph(cuda):
    """The mirror projection of each step on a second stream (two steps per
    replay, sb_mc_stage): the same bits after four steps."""
    ref_sys, ref = _run('split_bf16', mc=False, steps=4)
    mc_sys, got = _run('split_bf16', mc=True, pipelined=True, steps=4)
    assert mc_sys.steps_per_replay == 2 and mc_sys.launches_per_step == 6
    for gi, (a, b) in enumerate(zip(ref, got)):
        for k in a:
            assert torch.equal(a[k], b[k]), (gi, k, float((a[k].double() - b[k].double()).abs().max()))
    mc_sys.release_mc()


def test_mc_step_rejects_unfusable_groups(cuda):
    """A slope option the fused detector / slope stage does not implement
    keeps the Monte-Carlo step from being built."""
    from specula_b200.batched import BatchedScao, mc_groups
    sys_b = BatchedScao(mc_groups(n_real=(2, 0, 0)), device_idx=0)
    sys_b.start()
    sys_b.groups[0].loops[0].slopec.thr_pedestal = True
    with pytest.raises(NotImplementedError, match='fused detector'):
        sys_b.capture_mc()


def test_single_system_step_through_the_c_abi(cuda):
    """One group of one realisation: sb_mc_step is the whole loop step of one
    SCAO system behind the C ABI (six launches).  Noise-free, against the
    system's own sequential step graph (its single-vector reconstructor and
    mirror kernels sum in another order): slopes and mirror phase within 1e-4
    of their largest values over six steps."""
    from specula_b200.batched import BatchedScao
    from specula_b200.scao import ScaoConfig
    from tests.cases import rel_max_err
    cfg = ScaoConfig(photon_noise=False, readout_noise=0.0)
    a = BatchedScao([(cfg, [cfg])], device_idx=0)
    a.start()
    a.capture_plain()
    b = BatchedScao([(cfg, [cfg])], device_idx=0)
    b.start()
    b.capture_mc()
    assert b.launches_per_step == 6
    for _ in range(6):
        a.replay_plain()
        b.replay()
        torch.cuda.synchronize()
        ga, gb = a.groups[0], b.groups[0]
        assert rel_max_err(gb.S.cpu().numpy(), ga.S.cpu().numpy()) <= 1e-4
        assert rel_max_err(gb.dm_phase.cpu().numpy(), ga.dm_phase.cpu().numpy()) <= 1e-4
    assert float(gb.S.abs().max()) > 0
    b.release_mc()
