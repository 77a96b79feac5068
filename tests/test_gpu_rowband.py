"""One SCAO system split by bands of lenslet rows (specula_b200.rowband) on
one GPU: two and three ranks held in one process (each its own copy of the
system, run one after the other, the exchanges summed by the test) against
the one-process sequential step graph with the fused chain, with photon and
read-out noise: slopes, flux, commands, detector pixels and each rank's
mirror rows bit-identical over six steps."""
import pytest

torch = pytest.importorskip('torch')

pytestmark = pytest.mark.gpu


def _loop(cfg):
    from specula_b200.scao import ScaoLoop
    loop = ScaoLoop(cfg, device_idx=0)
    loop.start()
    return loop


@pytest.mark.parametrize('world', [2, 3])
@pytest.mark.parametrize('dft', ['fp32', 'split_bf16'])
def test_row_bands_equal_one_process(cuda, world, dft):
    from specula_b200.scao import ScaoConfig
    from specula_b200.rowband import RowBandLoop, step_together
    cfg = ScaoConfig(sh_dft=dft)                      # photon + read-out noise on
    ref = _loop(cfg)
    ref.capture(pipelined=False)                      # one eager step, then the graph
    assert ref.fused_chain
    bands = []
    for r in range(world):
        lp = _loop(cfg)
        lp.step_eager()
        bands.append(RowBandLoop(lp, r, world))
    p = ref.sh._plan.np_sub
    npx = ref.sh._plan.subap_npx
    for t in range(6):
        ref.replay()
        step_together(bands)
        torch.cuda.synchronize()
        for b in bands:
            lp = b.loop
            assert torch.equal(lp.slopec.slopes.slopes, ref.slopec.slopes.slopes), (t, b.rank)
            assert torch.equal(lp.slopec._flux, ref.slopec._flux), (t, b.rank)
            assert torch.equal(lp.integ.out_comm.value, ref.integ.out_comm.value), (t, b.rank)
            rows = slice(b.row0 * p, (b.row0 + b.n_rows) * p)
            assert torch.equal(lp.dm.layer.phaseInNm[rows], ref.dm.layer.phaseInNm[rows]), (t, b.rank)
            prow = slice(b.row0 * npx, (b.row0 + b.n_rows) * npx)
            assert torch.equal(lp.ccd._pixels.pixels[prow], ref.ccd._pixels.pixels[prow]), (t, b.rank)
    assert float(ref.slopec.slopes.slopes.abs().max()) > 0
    from specula_b200 import _lib
    _lib.call('sb_device_status')
