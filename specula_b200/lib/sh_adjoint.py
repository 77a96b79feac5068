"""Adjoint of the noise-free SH -> ShSlopec chain and the interaction matrix
built from it, on the B200.

The reference measures the interaction matrix by push-pull: a FuncGenerator
('PUSHPULL', specula/lib/modal_pushpull_signal.py:35-65) commands +a_k then
-a_k on one mode per loop step and ImRecCalibrator
(specula/processing_objects/im_rec_calibrator.py:42-71) accumulates
``im[k] += slopes / cmd_k``, i.e. ``(s(+a) - s(-a)) / a``: 2 x n_modes full
forward steps.  With a linear detector the slopes of one sub-aperture depend
only on that sub-aperture's phase samples and the photon normalisation
(sh.py:426-427) cancels in the centre of gravity (sh_slopec.py:392-404), so
d(slopes)/d(phase) is a 2 x np_sub^2 block per valid sub-aperture.
``ShSlopesAdjoint`` gets all blocks from one kernel launch
(sb_sh_slopes_jacobian) and contracts them with the mirror's influence
functions (sb_intmat_contract), which reads every influence-function
element once: ``IM = 2 * sign * J @ IF^T`` is the push-pull matrix in the
limit of small amplitudes (DM phase = sign * cmd @ IF, dm.py:72-86).

``ShSlopesAdjoint.pushpull_intmat`` runs the reference's push-pull sequence
on the same CUDA chain (one mode's influence function projected per step,
SH forward, CoG), captured in one CUDA graph: the measured alternative.
"""
import ctypes

import numpy as np
import torch

from specula_b200 import _lib


def lenslet_index(idxs, n_lenses, subap_npx):
    """Lenslet index (row * n_lenses + column) of each valid sub-aperture,
    from the ShSlopec pixel table (first pixel of each row of ``idxs``)."""
    idxs = np.asarray(idxs)
    ncols = n_lenses * subap_npx
    first = idxs[:, 0].astype(np.int64)
    row, col = first // ncols, first % ncols
    if np.any(row % subap_npx) or np.any(col % subap_npx):
        raise ValueError('sub-aperture pixel boxes are not aligned with the lenslet grid')
    return ((row // subap_npx) * n_lenses + col // subap_npx).astype(np.int32)


def pixel_to_column(mask_idx, dm_shape, field_size, top=0, left=0):
    """field pixel -> influence-function column (-1 where the mirror has no
    column).  ``mask_idx`` are the flat indices of the mirror's mask pixels
    in its own (dm_shape) grid; field pixel (r, c) sees mirror pixel
    (r + top, c + left), the crop of the on-axis propagation."""
    mask_idx = np.asarray(mask_idx, dtype=np.int64)
    rows, cols = mask_idx // dm_shape[1], mask_idx % dm_shape[1]
    r, c = rows - top, cols - left
    keep = (r >= 0) & (r < field_size) & (c >= 0) & (c < field_size)
    out = np.full(field_size * field_size, -1, dtype=np.int32)
    out[r[keep] * field_size + c[keep]] = np.flatnonzero(keep).astype(np.int32)
    return out


def row_segments(pix2col, lenslets, n_lenses, np_sub, field, ld_if):
    """Per lenslet row the influence-function columns the contraction reads:
    (start, count) in floats, both multiples of 32, covering every mirror
    column under a valid sub-aperture of that row (columns enumerate the
    mirror's pixels row-major, so np_sub consecutive field rows map to one
    contiguous range).  Returns the (n_lenses, 2) int32 table and the largest
    count."""
    p2c = np.asarray(pix2col).reshape(field, field)
    seg = np.zeros((n_lenses, 2), dtype=np.int32)
    lens = np.asarray(lenslets, dtype=np.int64)
    for li in range(n_lenses):
        cols = [p2c[li * np_sub:(li + 1) * np_sub, lj * np_sub:(lj + 1) * np_sub]
                for lj in (lens[lens // n_lenses == li] % n_lenses)]
        if not cols:
            continue
        c = np.concatenate([x.ravel() for x in cols])
        c = c[c >= 0]
        if c.size == 0:
            continue
        start = int(c.min()) & ~31
        end = min((int(c.max()) + 1 + 31) & ~31, int(ld_if))
        seg[li] = (start, end - start)
    return seg, int(seg[:, 1].max()) if n_lenses else 0


class ShSlopesAdjoint:
    """Jacobian / VJP of the slopes of a set-up ``SH`` + ``ShSlopec`` pair
    with respect to the SH input phase (nm), and the adjoint interaction
    matrix.  Noise-free detector, CoG threshold 0, no field interpolation
    (fov_ovs_coeff giving one phase sample per lenslet pixel)."""

    def __init__(self, sh, slopec):
        g = sh.geometry
        if g.do_interpolation:
            raise NotImplementedError('ShSlopesAdjoint: geometries that resample the field (fov_ovs != 1) '
                                      'are not supported')
        if slopec.thr_value > 0:
            raise ValueError('ShSlopesAdjoint: the thresholded CoG is not differentiable (thr_value must be <= 0)')
        self.sh = sh
        self.slopec = slopec
        self.device = sh.device
        self.n_lenses = g.n_lenses
        self.np_sub = g.ovs_np_sub
        self.subap_npx = g.subap_npx
        self.field = sh._plan.field_ld
        idxs = slopec.subapdata.idxs
        self.n_valid = int(idxs.shape[0])
        lens = lenslet_index(idxs, self.n_lenses, self.subap_npx)
        slot = np.full(self.n_lenses * self.n_lenses, -1, dtype=np.int32)
        slot[lens] = np.arange(self.n_valid, dtype=np.int32)
        self._lenslet = torch.as_tensor(lens, device=self.device)
        self._slot = torch.as_tensor(slot, device=self.device)
        self._tot = torch.empty(self.n_valid, dtype=torch.float32, device=self.device)
        self._frame = torch.empty((self.n_lenses * self.subap_npx,) * 2, dtype=torch.float32, device=self.device)
        self._slopes = torch.empty(2 * self.n_valid, dtype=torch.float32, device=self.device)
        self._flux = torch.empty(self.n_valid, dtype=torch.float32, device=self.device)
        nb = _lib.load().sb_slopec_scratch_bytes(ctypes.byref(self._slopec_plan()))
        self._sc_scratch = torch.empty(max(nb, 1), dtype=torch.uint8, device=self.device)

    # -- plumbing ---------------------------------------------------------
    def _slopec_plan(self):
        sc = self.slopec
        return _lib.SlopecPlan(n_subaps=self.n_valid, npx2=self.subap_npx ** 2, thr=0.0,
                               idxs=sc._idxs.data_ptr(), xw=sc.xweights.data_ptr(), yw=sc.yweights.data_ptr(),
                               mw=sc.mask_weighted.data_ptr())

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _field(self, t, name):
        t = torch.as_tensor(t, dtype=torch.float32, device=self.device)
        if t.shape != (self.field, self.field) or not t.is_contiguous():
            raise ValueError(f'ShSlopesAdjoint: {name} must be a contiguous {self.field}x{self.field} array')
        return t

    def _weights(self):
        sc = self.slopec
        return sc.xweights.data_ptr(), sc.yweights.data_ptr(), sc.mask_weighted.data_ptr()

    # -- forward ----------------------------------------------------------
    def slopes(self, A, phase):
        """Noise-free slopes and per-sub-aperture flux at (A, phase): the
        SH forward (sb_sh_forward) then the CoG (sb_slopec) on its frame.
        Returns views of internal buffers."""
        A = self._field(A, 'A')
        phase = self._field(phase, 'phase')
        st = self._stream()
        sh = self.sh
        _lib.call('sb_sh_forward', ctypes.byref(sh._plan), A.data_ptr(), phase.data_ptr(), A.data_ptr(), A.numel(),
                  1.0, self._frame.data_ptr(), sh._scratch.data_ptr(), sh._scratch.numel(), st)
        _lib.call('sb_slopec', ctypes.byref(self._slopec_plan()), self._frame.data_ptr(), self._slopes.data_ptr(),
                  self._flux.data_ptr(), self._sc_scratch.data_ptr(), self._sc_scratch.numel(), st)
        return self._slopes, self._flux

    def active(self, A, phase):
        """1 where the CoG keeps the sub-aperture at (A, phase):
        1/flux <= 1/(1e-3 * mean flux) (sh_slopec.py:400)."""
        _, flux = self.slopes(A, phase)
        return self.active_from_flux(flux)

    # -- adjoint ----------------------------------------------------------
    def _jacobian(self, A, phase, active):
        jac = torch.empty((2, self.n_valid, self.np_sub ** 2), dtype=torch.float32, device=self.device)
        xw, yw, mw = self._weights()
        _lib.call('sb_sh_slopes_jacobian', ctypes.byref(self.sh._plan), A.data_ptr(), phase.data_ptr(), self.n_valid,
                  self._lenslet.data_ptr(), xw, yw, mw, 0 if active is None else active.data_ptr(), jac.data_ptr(),
                  self._tot.data_ptr(), self._stream())
        return jac

    def active_from_flux(self, tot):
        """The CoG cut-off of sh_slopec.py:400 applied to per-sub-aperture
        fluxes: 1 where 1/tot <= 1/(1e-3 * mean(tot))."""
        t = tot.double()
        return ((t > 0) & ((1.0 / t) <= 1.0 / (t.mean() * 1e-3))).float().contiguous()

    def jacobian(self, A, phase, active=None):
        """(2, n_valid, np_sub^2): d slope / d phase_nm per valid sub-aperture
        (zero for sub-apertures the CoG cuts off at (A, phase), or outside
        ``active`` when given)."""
        A = self._field(A, 'A')
        phase = self._field(phase, 'phase')
        if active is not None:
            return self._jacobian(A, phase, torch.as_tensor(active, dtype=torch.float32,
                                                            device=self.device).contiguous())
        jac = self._jacobian(A, phase, None)
        return jac * self.active_from_flux(self._tot)[None, :, None]

    def vjp(self, A, phase, seed, active=None):
        """Field-shaped sum_j seed[j] d slope_j / d phase_nm (zero outside the
        valid sub-apertures)."""
        A = self._field(A, 'A')
        phase = self._field(phase, 'phase')
        seed = torch.as_tensor(seed, dtype=torch.float32, device=self.device).contiguous()
        if seed.numel() != 2 * self.n_valid:
            raise ValueError(f'ShSlopesAdjoint.vjp: seed has {seed.numel()} entries, expected {2 * self.n_valid}')
        if active is None:
            active = self.active(A, phase)
        grad = torch.zeros((self.field, self.field), dtype=torch.float32, device=self.device)
        xw, yw, mw = self._weights()
        _lib.call('sb_sh_slopes_vjp', ctypes.byref(self.sh._plan), A.data_ptr(), phase.data_ptr(), self.n_valid,
                  self._lenslet.data_ptr(), xw, yw, mw, active.data_ptr(), seed.data_ptr(), grad.data_ptr(),
                  self._stream())
        return grad

    def pixel_to_column(self, dm, top=0, left=0):
        shape = tuple(dm.layer.phaseInNm.shape)
        return torch.as_tensor(pixel_to_column(dm._ifunc.idx_inf_func, shape, self.field, top, left),
                               device=self.device)

    def intmat(self, A, phase, dm, top=0, left=0, active=None, jac=None, pix2col=None):
        """Adjoint interaction matrix (n_modes x 2 n_valid) for the set-up
        mirror ``dm``: 2 * sign * J @ IF^T, the small-amplitude limit of the
        reference's push-pull matrix.  Two launches: the Jacobian (which also
        returns each sub-aperture's flux) and the contraction (which applies
        the CoG cut-off from that flux)."""
        tot = None
        if jac is None:
            A = self._field(A, 'A')
            phase = self._field(phase, 'phase')
            if active is None:
                jac = self._jacobian(A, phase, None)
                tot = self._tot
            else:
                jac = self.jacobian(A, phase, active)
        if pix2col is None:
            pix2col = self.pixel_to_column(dm, top, left)
        n_modes = dm._IF.shape[0]
        im = torch.empty((n_modes, 2 * self.n_valid), dtype=torch.float32, device=self.device)
        segs = self._segments(pix2col, dm)
        tot_ptr = 0 if tot is None else tot.data_ptr()
        if segs is not None:
            _lib.call('sb_intmat_contract_rows', jac.data_ptr(), tot_ptr, self.n_valid, self.np_sub, self.n_lenses,
                      self.field, self._slot.data_ptr(), pix2col.data_ptr(), segs[0].data_ptr(), segs[1],
                      dm._IF.data_ptr(), n_modes, dm._ld, float(2.0 * dm.sign), im.data_ptr(), self._stream())
        else:
            _lib.call('sb_intmat_contract', jac.data_ptr(), tot_ptr, self.n_valid, self.np_sub, self.n_lenses,
                      self.field, self._slot.data_ptr(), pix2col.data_ptr(), dm._IF.data_ptr(), n_modes, dm._ld,
                      float(2.0 * dm.sign), im.data_ptr(), self._stream())
        return im

    # TMA contraction limits: np_sub 4 or 8, at most 992 field columns,
    # influence-function rows of a multiple of 32 floats, a row segment of at
    # most 8192 floats (256 chunks of 32)
    TMA_NP_SUB = (4, 8)
    TMA_MAX_COLUMNS = 992
    TMA_MAX_SEGMENT = 8192

    def _segments(self, pix2col, dm):
        """(device table, largest count) of the row segments for the TMA
        contraction, or None when its limits are not met (then the
        gather kernel runs); cached per mirror column map."""
        if (self.np_sub not in self.TMA_NP_SUB or self.field > self.TMA_MAX_COLUMNS or dm._ld % 32 or
                dm._IF.data_ptr() % 16):
            return None
        key = (pix2col.data_ptr(), int(dm._ld))
        cache = getattr(self, '_seg_cache', None)
        if cache is None or cache[0] != key:
            seg, seg_max = row_segments(pix2col.cpu().numpy(), self._lenslet.cpu().numpy(), self.n_lenses,
                                        self.np_sub, self.field, dm._ld)
            val = None if seg_max > self.TMA_MAX_SEGMENT else (torch.as_tensor(seg, device=self.device), seg_max)
            cache = (key, val, pix2col)
            self._seg_cache = cache
        return cache[1]

    # -- push-pull on the same chain -----------------------------------------
    def pushpull_intmat(self, A, dm, amplitudes, graph=True):
        """The reference's push-pull matrix (s(+a_k) - s(-a_k)) / a_k from a
        flat wavefront, on the GPU chain: per step the mirror projects one
        mode's command (sb_dm_project on that influence function), then the
        SH forward and the CoG.  ``graph``: capture the 2 n_modes steps in
        one CUDA graph and replay it (returns (intmat, replay))."""
        A = self._field(A, 'A')
        n_modes = dm._IF.shape[0]
        amps = torch.as_tensor(np.asarray(amplitudes, dtype=np.float64), dtype=torch.float64)
        if amps.numel() == 1:
            amps = amps.repeat(n_modes)
        pm = torch.stack([amps, -amps], 1).reshape(-1).float().to(self.device)
        shape = tuple(dm.layer.phaseInNm.shape)
        if shape != (self.field, self.field):
            raise ValueError('pushpull_intmat: the mirror grid must be the SH field grid')
        phase = torch.zeros(shape, dtype=torch.float32, device=self.device)
        S = torch.empty((2 * n_modes, 2 * self.n_valid), dtype=torch.float32, device=self.device)
        sh = self.sh
        plan_sh = ctypes.byref(sh._plan)
        plan_sc = self._slopec_plan()
        mask_idx = dm._idx

        def run(st):
            for k in range(n_modes):
                row = dm._IF.data_ptr() + 4 * k * dm._ld
                for h in range(2):
                    j = 2 * k + h
                    _lib.call('sb_dm_project', row, 1, int(mask_idx.numel()), dm._ld, pm.data_ptr() + 4 * j, 1,
                              float(dm.sign), mask_idx.data_ptr(), phase.data_ptr(), st)
                    _lib.call('sb_sh_forward', plan_sh, A.data_ptr(), phase.data_ptr(), A.data_ptr(), A.numel(),
                              1.0, self._frame.data_ptr(), sh._scratch.data_ptr(), sh._scratch.numel(), st)
                    _lib.call('sb_slopec', ctypes.byref(plan_sc), self._frame.data_ptr(),
                              S[j].data_ptr(), self._flux.data_ptr(), self._sc_scratch.data_ptr(),
                              self._sc_scratch.numel(), st)

        def finish():
            return (S[0::2] - S[1::2]) / amps.float().to(self.device)[:, None]

        if not graph:
            run(self._stream())
            return finish(), None
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                run(s.cuda_stream)
        torch.cuda.current_stream(self.device).wait_stream(s)

        def replay():
            g.replay()
            return finish()

        # the graph writes and reads these buffers: keep them alive with it
        replay.graph = g
        replay.buffers = (A, phase, pm, S, amps)
        return replay(), replay


class ShSlopesFunction(torch.autograd.Function):
    """slopes = SH+CoG(phase) as a differentiable torch operation: forward
    through sb_sh_forward + sb_slopec, backward through sb_sh_slopes_vjp
    (the CoG cut-off is held at the forward point)."""

    @staticmethod
    def forward(ctx, phase, adj, A):
        phase = phase.detach().contiguous()
        slopes, flux = adj.slopes(A, phase)
        active = adj.active_from_flux(flux)
        ctx.adj, ctx.A = adj, A
        ctx.save_for_backward(phase, active)
        return slopes.clone()

    @staticmethod
    def backward(ctx, grad_slopes):
        phase, active = ctx.saved_tensors
        g = ctx.adj.vjp(ctx.A, phase, grad_slopes.contiguous(), active=active)
        return g, None, None


def sh_slopes(adj, A, phase):
    """Differentiable noise-free slopes of ``adj``'s SH + ShSlopec at
    (A, phase); ``phase`` may require grad."""
    return ShSlopesFunction.apply(phase, adj, A)
