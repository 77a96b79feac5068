"""The whole-step CUDA graphs of ScaoLoop (sequential and pipelined) give
bit-identical results to the object-by-object loop (LoopControl), including
photon and read-out noise (counter-based RNG keyed by frame and pixel)."""
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu


def _row_padded(t, pad=4):
    """The same values as ``t`` in a view whose rows are ``pad`` floats longer."""
    big = torch.zeros((t.shape[0], t.shape[1] + pad), dtype=t.dtype, device=t.device)
    big[:, :t.shape[1]].copy_(t)
    return big[:, :t.shape[1]]


def _loop(mode, n_steps, cfg_kw=None, strided_stop=False):
    from specula_b200.scao import ScaoConfig, ScaoLoop
    cfg = ScaoConfig(heights=[0.0, 4000.0], cn2=[0.7, 0.3], wind_speed=[10.0, 25.0],
                     wind_direction=[30.0, 212.7], **(cfg_kw or {}))
    loop = ScaoLoop(cfg, device_idx=0)
    if strided_stop:
        # a pupil stop held in row-padded storage: the two-launch propagation
        # reads it through its row stride, the fused kernel cannot
        loop.pupilstop.A = _row_padded(loop.pupilstop.A)
        loop.pupilstop.phaseInNm = _row_padded(loop.pupilstop.phaseInNm)
    loop.start()
    loop.step_eager()
    done = 1
    if mode == 'eager':
        while done < n_steps:
            loop.step_eager()
            done += 1
    else:
        if mode == 'pipelined_default':
            loop.capture()
        elif mode == 'pipelined_early':
            loop.capture(early_atmo=True)
        elif mode == 'pipelined_unfused_chain':
            loop.capture(fuse_chain=False)
        else:
            loop.capture(pipelined=mode.startswith('pipelined'), fuse_atmo=(mode == 'pipelined_fused'),
                         early_atmo=False)
        done += 1
        while done < n_steps:
            loop.replay()
            done += loop.steps_per_replay
    assert done == n_steps
    torch.cuda.synchronize()
    return loop


@pytest.mark.parametrize('mode', ['sequential', 'pipelined', 'pipelined_fused', 'pipelined_unfused_chain',
                                  'pipelined_early'])
def test_graph_step_matches_object_loop(mode, cuda):
    """pipelined_fused: AtmoEvolution and AtmoPropagation as one launch;
    every mode but pipelined_unfused_chain runs SH, CCD and ShSlopec as the
    two launches of sb_sh_ccd_slopec; pipelined_early also runs the
    atmosphere early, on a stream of its own, with the mirror applied in the
    SH's field read."""
    n = 10
    ref = _loop('eager', n)
    got = _loop(mode, n)
    if mode.startswith('pipelined'):
        assert got.pipelined and got.steps_per_replay == 2
    assert got.fused_chain == (mode != 'pipelined_unfused_chain')
    assert got.early_atmo == (mode == 'pipelined_early')
    for name, a, b in (('slopes', ref.slopec.slopes.slopes, got.slopec.slopes.slopes),
                       ('dm phase', ref.dm.layer.phaseInNm, got.dm.layer.phaseInNm),
                       ('commands', ref.integ.out_comm.value, got.integ.out_comm.value),
                       ('integrator state', ref.integ.state, got.integ.state),
                       ('pixels', ref.ccd.outputs['out_pixels'].pixels, got.ccd.outputs['out_pixels'].pixels),
                       ('layers', ref.atmo.layer_list[1].phaseInNm, got.atmo.layer_list[1].phaseInNm),
                       ('field phase', ref.prop.outputs['out_on_axis_source_ef'].phaseInNm,
                        got.prop.outputs['out_on_axis_source_ef'].phaseInNm),
                       ('field amplitude', ref.prop.outputs['out_on_axis_source_ef'].A,
                        got.prop.outputs['out_on_axis_source_ef'].A),
                       ('intensity', ref.sh.outputs['out_i'].i, got.sh.outputs['out_i'].i)):
        assert torch.equal(a, b), name
    assert float(ref.dm.layer.phaseInNm.abs().max()) > 0


def _assert_same_loop_state(ref, got):
    for name, a, b in (('slopes', ref.slopec.slopes.slopes, got.slopec.slopes.slopes),
                       ('dm phase', ref.dm.layer.phaseInNm, got.dm.layer.phaseInNm),
                       ('commands', ref.integ.out_comm.value, got.integ.out_comm.value),
                       ('pixels', ref.ccd.outputs['out_pixels'].pixels, got.ccd.outputs['out_pixels'].pixels)):
        assert torch.equal(a, b), name


def test_default_capture_fuses_the_atmosphere(cuda):
    """capture() with no arguments picks the fused atmosphere and the fused
    SH / CCD / slope chain for the SCAO layout: 6 kernels per step, the same
    bits as the object loop."""
    n = 6
    ref = _loop('eager', n)
    got = _loop('pipelined_default', n)
    assert got.pipelined and got.fused_atmo and got.fused_chain and not got.early_atmo and got.kernels_per_step == 6
    _assert_same_loop_state(ref, got)


def test_default_capture_falls_back_for_a_strided_stop(cuda):
    """A pupil stop that is not a dense L x L array keeps the two atmosphere
    launches (7 kernels per step with the fused chain), with the same bits as
    the object loop."""
    n = 6
    ref = _loop('eager', n, strided_stop=True)
    got = _loop('pipelined_default', n, strided_stop=True)
    assert got.pipelined and not got.fused_atmo and got.fused_chain and got.kernels_per_step == 7
    _assert_same_loop_state(ref, got)
    plain = _loop('eager', n)
    assert torch.equal(ref.slopec.slopes.slopes, plain.slopec.slopes.slopes)


def test_fractional_delay_falls_back_to_sequential_graph(cuda):
    loop = _loop('pipelined', 4, cfg_kw=dict(delay=1.5))
    assert not loop.pipelined and loop.steps_per_replay == 1


@pytest.mark.parametrize('slots', [1, 2])
def test_io_graph_follows_per_step_inputs(cuda, slots):
    """capture(io=True): every replayed step reads its own seeing / wind row
    from io_inputs and leaves its slopes and commands in io_outputs; the
    results equal the object-by-object loop fed the same per-step inputs."""
    from specula_b200.scao import ScaoConfig, ScaoLoop
    cfg = ScaoConfig(heights=[0.0, 4000.0], cn2=[0.7, 0.3], wind_speed=[10.0, 25.0],
                     wind_direction=[30.0, 212.7])
    n_in = 5

    def inputs(t):
        # step-dependent seeing, wind speed and (fractional-degree) direction
        return [0.7 + 0.05 * t, 10.0 + t, 25.0 - 0.5 * t, 30.0 + 0.37 * t, 212.7 - 0.61 * t]

    ref = ScaoLoop(cfg, device_idx=0)
    got = ScaoLoop(cfg, device_idx=0)
    ref.start()
    got.start()
    outs_ref = []
    # steps 0 and 1 eager in both (capture() runs one eager step itself)
    for t in range(2):
        ref._inputs.copy_(torch.tensor(inputs(t), dtype=torch.float64))
        ref.step_eager()
    got._inputs.copy_(torch.tensor(inputs(0), dtype=torch.float64))
    got.step_eager()
    got._inputs.copy_(torch.tensor(inputs(1), dtype=torch.float64))
    got.capture(io=True, io_slots=slots)
    assert tuple(got.io_inputs.shape) == (2, n_in)
    nsl = got.slopec.slopes.slopes.numel()
    for t in range(2, 8):
        ref._inputs.copy_(torch.tensor(inputs(t), dtype=torch.float64))
        ref.step_eager()
        outs_ref.append(torch.cat([ref.slopec.slopes.slopes, ref.integ.out_comm.value]).clone())
    outs_got = []
    for r in range(3):
        # with two slots the replays alternate between the slots' graphs
        j = r % slots
        for s in range(2):
            got.io_inputs_slots[j][s].copy_(torch.tensor(inputs(2 + 2 * r + s), dtype=torch.float64))
        got.replay(j)
        outs_got.extend([got.io_outputs_slots[j][0].clone(), got.io_outputs_slots[j][1].clone()])
    torch.cuda.synchronize()
    for t, (a, b) in enumerate(zip(outs_ref, outs_got)):
        assert torch.equal(a[:nsl], b[:nsl]), ('slopes', t)
        assert torch.equal(a[nsl:], b[nsl:]), ('commands', t)
    assert torch.equal(ref.atmo.layer_list[1].phaseInNm, got.atmo.layer_list[1].phaseInNm)
