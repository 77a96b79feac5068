"""The headline workloads end to end: the captured, pipelined step graph of
ScaoLoop (the default capture: fused atmosphere, SH / CCD / slopes in two
launches) against the oracle chain
run on the same system, step by step, with no re-synchronisation of the
two loops.

Systems (noise-free detector so both loops see the same frames):
- ELT: 39 m, 640 px, 80x80 sub-apertures of 8x8 px, FFT 16 (cut 4) onto
  6x6 px, 7 layers with random winds, 500 Zernike modes;
- config 1 geometry (ii): 8 m, 160 px, 20x20 sub-apertures, FFT 16 (cut 2)
  onto 8x8 px at 0.875 lambda/d, one layer, 54 Zernike modes.
The reconstructor is the pseudo-inverse of the adjoint interaction matrix
(calibrated with the mirror sign flipped, as the reference's calibration
configuration does), so the loop is a stable negative-feedback loop and
float32 rounding differences stay bounded instead of growing.  The oracle
uses the GPU loop's screens, influence functions, reconstructor and
sub-aperture tables.  Every step: slopes and mirror commands within 1e-4,
the mirror phase within 1e-4 (max |d| / max |ref|).
"""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

SLOPE_TOL = 1e-4
DM_TOL = 1e-4


def _calibrated_loop(cfg, dev):
    """ScaoLoop on Zernike influence functions with the adjoint-calibrated
    reconstructor, started (objects set up), no step taken yet."""
    from specula_b200.data_objects.intmat import Intmat
    from specula_b200.lib.make_mask import make_mask
    from specula_b200.lib.sh_adjoint import ShSlopesAdjoint
    from specula_b200.lib.zernike import compute_zern_ifunc
    from specula_b200.scao import ScaoLoop
    pupil = make_mask(cfg.pixel_pupil, cfg.obsratio, 1.0)
    ifunc, _ = compute_zern_ifunc(cfg.pixel_pupil, cfg.n_modes, mask=pupil)
    loop = ScaoLoop(cfg, device_idx=dev.index, ifunc=torch.as_tensor(ifunc, device=dev))
    loop.start()
    adj = ShSlopesAdjoint(loop.sh, loop.slopec)
    A = torch.as_tensor(pupil.astype(np.float32), device=dev)
    im = adj.intmat(A, torch.zeros_like(A), loop.dm) * (-1.0)
    R = Intmat(im, target_device_idx=dev.index).pseudo_invert(im).t().contiguous().float()
    loop.rec._R.copy_(R)
    torch.cuda.synchronize(dev)
    return loop


def _oracle(loop):
    from oracle.loop import OracleScaoLoop
    strips = [s.cpu().numpy() for s in loop.atmo.phasescreens]
    IF = loop.dm._ifunc.influence_function.cpu().numpy()
    R = loop.rec._R.cpu().numpy()
    S0 = loop.prop.outputs['out_on_axis_source_ef'].S0
    return OracleScaoLoop(loop.cfg, IF, R, loop.subapdata.idxs, loop.pupil, S0, strips=strips)


def _run_against_oracle(cfg, n_steps):
    dev = torch.device('cuda', 0)
    loop = _calibrated_loop(cfg, dev)
    orc = _oracle(loop)
    nsl = loop.slopec.slopes.slopes.numel()
    errs = []

    def check(step, slopes, comm, dm_phase):
        s_ref = orc.step()
        e_s = rel_max_err(slopes, s_ref)
        e_c = rel_max_err(comm, orc.comm) if np.any(orc.comm) else float(np.abs(comm).max())
        e_d = rel_max_err(dm_phase, orc.dm_phase) if np.any(orc.dm_phase) else float(np.abs(dm_phase).max())
        errs.append((step, e_s, e_c, e_d))
        assert e_s <= SLOPE_TOL, (step, 'slopes', e_s)
        assert e_c <= SLOPE_TOL, (step, 'commands', e_c)
        assert e_d <= DM_TOL, (step, 'dm phase', e_d)

    # step 0 object by object, step 1 inside capture(), then the graph (two steps per replay)
    loop.step_eager()
    check(0, loop.slopec.slopes.slopes.cpu().numpy(), loop.integ.out_comm.value.cpu().numpy(),
          loop.dm.layer.phaseInNm.cpu().numpy())
    loop.capture(io=True)
    assert loop.pipelined and loop.fused_atmo and loop.fused_chain and loop.kernels_per_step == 6
    check(1, loop.slopec.slopes.slopes.cpu().numpy(), loop.integ.out_comm.value.cpu().numpy(),
          loop.dm.layer.phaseInNm.cpu().numpy())
    dm_buf = loop._bufs[0]
    step = 2
    while step < n_steps:
        loop.replay()
        torch.cuda.synchronize(dev)
        out = loop.io_outputs.cpu().numpy()
        # the replay's first step writes the mirror into buffer 1, its second into buffer 0
        for k, buf in ((0, dm_buf[1]), (1, dm_buf[0])):
            check(step + k, out[k, :nsl], out[k, nsl:], buf.cpu().numpy())
        step += 2
    assert np.abs(loop.dm.layer.phaseInNm.cpu().numpy()).max() > 0
    from specula_b200 import _lib
    _lib.call('sb_device_status')
    worst = max(errs, key=lambda e: e[1])
    print(f'{n_steps} steps: worst slopes {worst[1]:.2e} (step {worst[0]}), commands '
          f'{max(e[2] for e in errs):.2e}, dm phase {max(e[3] for e in errs):.2e}')
    return errs


def test_elt_pipelined_graph_matches_oracle_loop(cuda):
    from specula_b200.scao import elt_config
    cfg = elt_config()
    cfg.photon_noise = False
    cfg.readout_noise = 0.0
    errs = _run_against_oracle(cfg, 22)
    assert len(errs) == 22


def test_config1_plain16_pipelined_graph_matches_oracle_loop(cuda):
    from specula_b200.scao import ScaoConfig
    cfg = ScaoConfig(photon_noise=False, readout_noise=0.0)     # 160 px, 20x20, 0.875 lambda/d, FFT 16, 54 modes
    errs = _run_against_oracle(cfg, 30)
    assert len(errs) == 30
