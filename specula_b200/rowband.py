"""One SCAO system split over GPUs by bands of lenslet rows.

The reference steps the whole pupil in one process (loop_control.py:83-123).
Here every rank holds its own copy of the system's objects (a ``ScaoLoop``,
same configuration and seeds) and, per step:

- runs the atmosphere and the on-axis propagation in full (replicated);
- runs the SH forward of its band of lenslet rows only (``sb_sh_forward_rows``),
  leaving the per-CTA partial sums of the photon normalisation in the whole
  grid's layout, zero outside its band;
- exchange 1: the partial sums, summed over the ranks;
- normalisation, detector and CoG of its rows (``sb_ccd_slopec_rows``):
  slopes, flux and the CoG sums of its valid sub-apertures at their places in
  whole-system vectors, zero elsewhere;
- exchange 2: those vectors, summed over the ranks; the flux cut-off on the
  sums (``sb_slopec_cutoff``), then the reconstructor and the integrators on
  the whole slope vector (replicated: R is small);
- the mirror projection of the influence-function columns under its rows only
  (``DM.project(columns=...)``): the influence functions, 95 % of the step's
  bytes at ELT size, are what the split divides.

Both exchanges sum vectors whose supports are disjoint across the ranks, so
the sums are exact and every rank's slopes, commands and mirror rows equal the
one-process step's bit for bit (the CCD draws use the whole frame's pixel
indices).  The mirror phase outside a rank's rows is left from its own earlier
steps: the field there is computed but never read.  ``exchange(t)`` sums a
tensor over the ranks in place: ``torch.distributed.all_reduce`` (NCCL, one
process per GPU, ``from_process_group``) or any other in-place sum.
"""
import ctypes

import numpy as np
import torch

from specula_b200 import _lib


def lenslet_bands(n_lenses, world):
    """(first row, rows) of each rank's band: contiguous, as even as possible."""
    if world < 1 or world > n_lenses:
        raise ValueError(f'lenslet_bands: {world} ranks for {n_lenses} lenslet rows')
    base, extra = divmod(n_lenses, world)
    out, r0 = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((r0, n))
        r0 += n
    return out


def mirror_columns(mask_idx, side, row0, row1):
    """Influence-function columns [c0, c1) of the mirror's mask pixels on pixel
    rows row0 .. row1 - 1 of its side x side grid (the mask is listed
    row-major, so they are contiguous); c0 rounded down to a multiple of 4 for
    16-byte aligned rows (the extra columns project the same values the
    neighbouring rank does)."""
    rows = np.asarray(mask_idx, dtype=np.int64) // side
    sel = np.flatnonzero((rows >= row0) & (rows < row1))
    if sel.size == 0:
        return 0, 0
    c0, c1 = int(sel[0]), int(sel[-1]) + 1
    if c1 - c0 != sel.size:
        raise ValueError('mirror_columns: the mask pixels are not listed row-major')
    return c0 & ~3, c1


class RowBandLoop:
    """This rank's share of a ``ScaoLoop`` step (see the module docstring).
    ``loop`` must have run one eager step (``start()``, ``step_eager()``)."""

    def __init__(self, loop, rank, world, exchange=None):
        self.loop = loop
        self.rank, self.world = rank, world
        self.exchange = exchange
        if not loop._can_fuse_chain():
            raise NotImplementedError('RowBandLoop: the system needs the fused SH / detector / slope chain (plain '
                                      'SH, a detector read every step, slopes with thr_value only)')
        loop._setup_chain()
        # the steps after the first advance the atmosphere by the loop's time step
        loop.atmo.delta_time = loop.atmo.t_to_seconds(loop.loop.dt)
        sh, sl, dm = loop.sh, loop.slopec, loop.dm
        self.mode = 0 if sh._forward == 'sb_sh_forward' else 1
        plan = sh._plan
        self.row0, self.n_rows = lenslet_bands(plan.n_lenses, world)[rank]
        lib = _lib.load()
        self.nparts = lib.sb_sh_rows_parts(ctypes.byref(plan), self.mode)
        nbytes = max(lib.sb_sh_scratch_bytes(ctypes.byref(plan)), 8 * self.nparts)
        dev = loop.device
        # SH scratch: the partial sums at its start, never written outside the band
        self._sh_scratch = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
        self.parts_local = self._sh_scratch[:8 * self.nparts].view(torch.float32)
        self.parts = torch.zeros(2 * self.nparts, dtype=torch.float32, device=dev)
        nv = int(sl._plan.n_subaps)
        self.nv = nv
        # slopes (2 nv), flux, tot, sxn, syn: this band's entries, zero elsewhere
        self.vec_local = torch.zeros(6 * nv, dtype=torch.float32, device=dev)
        self.vec = torch.zeros(6 * nv, dtype=torch.float32, device=dev)
        p = plan.np_sub
        side = dm.layer.phaseInNm.shape[1]
        if plan.field_ld != side:
            raise NotImplementedError('RowBandLoop: the mirror grid must be the SH field grid')
        self.columns = mirror_columns(dm._idx.cpu().numpy(), side, self.row0 * p, (self.row0 + self.n_rows) * p)

    @classmethod
    def from_process_group(cls, loop, group=None):
        """Rank and world of the default (or given) process group, NCCL sums."""
        import torch.distributed as dist
        return cls(loop, dist.get_rank(group), dist.get_world_size(group),
                   exchange=lambda t: dist.all_reduce(t, group=group))

    def _stream(self):
        return torch.cuda.current_stream(self.loop.device).cuda_stream

    def sh_band(self):
        """Atmosphere and propagation (whole pupil), then the band's SH:
        returns the partial sums to be summed over the ranks."""
        loop = self.loop
        sh = loop.sh
        loop.atmo.trigger_code()
        loop.prop.trigger_code()
        ef = sh._in_ef
        _lib.call('sb_sh_forward_rows', ctypes.byref(sh._plan), self.mode, self.row0, self.n_rows, ef.A.data_ptr(),
                  ef.phaseInNm.data_ptr(), ef.A.data_ptr(), ef.A.numel(), sh._out_i.i.data_ptr(),
                  self._sh_scratch.data_ptr(), self._sh_scratch.numel(), self._stream())
        return self.parts_local

    def chain_band(self, parts):
        """Normalisation (from the summed partials), CCD and CoG of the band:
        returns the slope / flux / CoG-sum vector to be summed over the ranks."""
        loop = self.loop
        sh, ccd, sl = loop.sh, loop.ccd, loop.slopec
        nv, v = self.nv, self.vec_local
        _lib.call('sb_ccd_slopec_rows', ctypes.byref(sh._plan), parts.data_ptr(), self.nparts, sh._photon_scale,
                  self.row0, self.n_rows, sh._out_i.i.data_ptr(), ctypes.byref(ccd._params),
                  ccd._integrated_i.i.data_ptr(), ccd._pixels.pixels.data_ptr(), ctypes.byref(sl._plan),
                  loop._lenslet_subap.data_ptr(), v.data_ptr(), v[2 * nv:].data_ptr(), v[3 * nv:].data_ptr(),
                  self._stream())
        return v

    def finish(self, vec):
        """Flux cut-off on the summed vectors, reconstructor + integrators on
        the whole slope vector, the mirror on the band's columns."""
        loop = self.loop
        sl, dm = loop.slopec, loop.dm
        nv, st = self.nv, self._stream()
        _lib.call('sb_slopec_cutoff', vec[3 * nv:].data_ptr(), vec[4 * nv:].data_ptr(), vec[5 * nv:].data_ptr(), nv,
                  vec.data_ptr(), st)
        sl._target.copy_(vec[:2 * nv])
        sl._flux.copy_(vec[2 * nv:3 * nv])
        sl._apply_products(st)
        loop._rec_integ()
        dm.project(dm.local_inputs['in_command'].value, dm.layer.phaseInNm, columns=self.columns)

    def step(self):
        """One loop step with the two sums over the ranks."""
        if self.exchange is None:
            raise ValueError('RowBandLoop.step: no exchange (use sh_band / chain_band / finish and sum yourself)')
        self.parts.copy_(self.sh_band())
        self.exchange(self.parts)
        self.vec.copy_(self.chain_band(self.parts))
        self.exchange(self.vec)
        self.finish(self.vec)


def step_together(bands):
    """One step of ranks held in one process (each a ``RowBandLoop`` on its
    own copy of the system, run one after the other; the sums taken here)."""
    parts = [b.sh_band() for b in bands]
    total = torch.stack([p.to(bands[0].parts.device) for p in parts]).sum(0)
    for b in bands:
        b.parts.copy_(total)
    vecs = [b.chain_band(b.parts) for b in bands]
    total = torch.stack([v.to(bands[0].vec.device) for v in vecs]).sum(0)
    for b in bands:
        b.vec.copy_(total)
        b.finish(b.vec)
