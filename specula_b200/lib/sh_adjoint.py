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
import warnings

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


def resample_matrix(ext1, ext2, yy, xx, in_shape):
    """The SH's field resampling as a sparse float64 matrix (see
    _resample_matrix), built with torch's sparse index checks on."""
    with torch.sparse.check_sparse_tensor_invariants(enable=True):
        return _resample_matrix(ext1, ext2, yy, xx, in_shape)


def _resample_matrix(ext1, ext2, yy, xx, in_shape):
    """The SH's field resampling as a sparse float64 matrix (out pixels x in
    pixels): edge extrapolation of the input phase (extrapolate_edge_pixel.py:
    ext[k] = ph[k], ph[s1], or 2 ph[s1] - ph[s2]) followed by the bilinear
    interpolation at (yy, xx) on the input grid (interp2d.py:95-122, the
    weights of sb_interp2d_field).  Both steps are linear in the phase, so
    the resampled phase of any phase map is this matrix times it."""
    rows, cols = in_shape
    n_in = rows * cols
    s1 = torch.as_tensor(ext1, dtype=torch.int64).reshape(-1)
    s2 = torch.as_tensor(ext2, dtype=torch.int64).reshape(-1)
    k = torch.arange(n_in, dtype=torch.int64)
    own = s1 < 0
    one = (~own) & (s2 < 0)
    two = (~own) & (s2 >= 0)
    er = torch.cat([k[own], k[one], k[two], k[two]])
    ec = torch.cat([k[own], s1[one], s1[two], s2[two]])
    ev = torch.cat([torch.ones(int(own.sum()), dtype=torch.float64), torch.ones(int(one.sum()), dtype=torch.float64),
                    torch.full((int(two.sum()),), 2.0, dtype=torch.float64),
                    torch.full((int(two.sum()),), -1.0, dtype=torch.float64)])
    E = torch.sparse_coo_tensor(torch.stack([er, ec]), ev, (n_in, n_in), check_invariants=True).coalesce()
    y = torch.as_tensor(yy, dtype=torch.float64).reshape(-1)
    x = torch.as_tensor(xx, dtype=torch.float64).reshape(-1)
    y0 = torch.clamp(torch.floor(y), 0, rows - 2)
    x0 = torch.clamp(torch.floor(x), 0, cols - 2)
    fy, fx = y - y0, x - x0
    i00 = (y0 * cols + x0).long()
    n_out = y.numel()
    o = torch.arange(n_out, dtype=torch.int64)
    ir = torch.cat([o, o, o, o])
    ic = torch.cat([i00, i00 + 1, i00 + cols, i00 + cols + 1])
    iv = torch.cat([(1 - fy) * (1 - fx), (1 - fy) * fx, fy * (1 - fx), fy * fx])
    Ip = torch.sparse_coo_tensor(torch.stack([ir, ic]), iv, (n_out, n_in), check_invariants=True).coalesce()
    with warnings.catch_warnings():
        warnings.filterwarnings('ignore', message='Sparse CSR tensor support is in beta')
        return torch.sparse.mm(Ip, E).coalesce()


class ShSlopesAdjoint:
    """Jacobian / VJP of the slopes of a set-up ``SH`` + ``ShSlopec`` pair
    with respect to the SH input phase (nm), and the adjoint interaction
    matrix.  Noise-free detector, CoG threshold 0.

    Geometries that resample the field (fov_ovs != 1, sh.py:353-357,447-460):
    ``slopes``, ``vjp`` and ``intmat`` take the SH's input field (its grid)
    and run the SH's edge extrapolation and interpolation first; ``vjp``
    returns the gradient on the input grid through the transpose of that
    linear map, ``intmat`` contracts with the influence functions resampled
    by it; ``jacobian`` stays with respect to the resampled phase samples."""

    def __init__(self, sh, slopec):
        g = sh.geometry
        self.interp = bool(g.do_interpolation)
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
        if self.interp:
            self.in_shape = tuple(sh._in_ef.phaseInNm.shape)
            self._pext = torch.empty(self.in_shape, dtype=torch.float32, device=self.device)
            self._Ai = torch.empty((self.field, self.field), dtype=torch.float32, device=self.device)
            self._Pi = torch.empty((self.field, self.field), dtype=torch.float32, device=self.device)
            self._M = None
        else:
            self.in_shape = (self.field, self.field)

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
        if tuple(t.shape) != self.in_shape or not t.is_contiguous():
            raise ValueError(f'ShSlopesAdjoint: {name} must be a contiguous {self.in_shape[0]}x{self.in_shape[1]} '
                             'array')
        return t

    def resampled(self, A, phase, st=None):
        """The field the SH kernels see: (A, phase) itself, or with
        resampling the SH's extrapolated and interpolated field (the calls of
        SH.trigger_code; internal buffers)."""
        if not self.interp:
            return A, phase
        sh = self.sh
        st = self._stream() if st is None else st
        _lib.call('sb_edge_extrapolate', phase.data_ptr(), sh._ext1.data_ptr(), sh._ext2.data_ptr(), phase.numel(),
                  self._pext.data_ptr(), st)
        _lib.call('sb_interp2d_field', A.data_ptr(), self._pext.data_ptr(), self.in_shape[0], self.in_shape[1],
                  sh._yy.data_ptr(), sh._xx.data_ptr(), sh._yy.numel(), self._Ai.data_ptr(), self._Pi.data_ptr(), st)
        return self._Ai, self._Pi

    def resample_matrix(self):
        """The resampling as a sparse float64 matrix on the device (built once)."""
        if self._M is None:
            sh = self.sh
            self._M = resample_matrix(sh._ext1.cpu(), sh._ext2.cpu(), sh._yy.cpu(), sh._xx.cpu(),
                                      self.in_shape).to(self.device)
        return self._M

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
        Af, Pf = self.resampled(A, phase)
        _lib.call('sb_sh_forward', ctypes.byref(sh._plan), Af.data_ptr(), Pf.data_ptr(), A.data_ptr(), A.numel(),
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
        ``active`` when given); with resampling, with respect to the resampled
        phase samples."""
        A = self._field(A, 'A')
        phase = self._field(phase, 'phase')
        A, phase = self.resampled(A, phase)
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
        Af, Pf = self.resampled(A, phase)
        grad = torch.zeros((self.field, self.field), dtype=torch.float32, device=self.device)
        xw, yw, mw = self._weights()
        _lib.call('sb_sh_slopes_vjp', ctypes.byref(self.sh._plan), Af.data_ptr(), Pf.data_ptr(), self.n_valid,
                  self._lenslet.data_ptr(), xw, yw, mw, active.data_ptr(), seed.data_ptr(), grad.data_ptr(),
                  self._stream())
        if not self.interp:
            return grad
        # back through the resampling: its transpose, in float64
        g = torch.sparse.mm(self.resample_matrix().t(), grad.reshape(-1, 1).double())
        return g.reshape(self.in_shape).float()

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
                jac = self._jacobian(*self.resampled(A, phase), None)
                tot = self._tot
            else:
                jac = self.jacobian(A, phase, active)
        n_modes = dm._IF.shape[0]
        if self.interp:
            IF, ld, pix2col = self.resampled_ifunc(dm, top, left)
        else:
            IF, ld = dm._IF, dm._ld
            if pix2col is None:
                pix2col = self.pixel_to_column(dm, top, left)
        im = torch.empty((n_modes, 2 * self.n_valid), dtype=torch.float32, device=self.device)
        tot_ptr = 0 if tot is None else tot.data_ptr()
        ifl = self.lenslet_ifunc(IF, ld, pix2col) if self.contraction == 'lenslet' else None
        if ifl is not None:
            _lib.call('sb_intmat_contract_lenslets', jac.data_ptr(), tot_ptr, self.n_valid, self.np_sub,
                      ifl.data_ptr(), n_modes, float(2.0 * dm.sign), im.data_ptr(), self._stream())
            return im
        segs = self._segments(pix2col, IF, ld) if self.contraction in ('lenslet', 'rows') else None
        if segs is not None:
            _lib.call('sb_intmat_contract_rows', jac.data_ptr(), tot_ptr, self.n_valid, self.np_sub, self.n_lenses,
                      self.field, self._slot.data_ptr(), pix2col.data_ptr(), segs[0].data_ptr(), segs[1],
                      IF.data_ptr(), n_modes, ld, float(2.0 * dm.sign), im.data_ptr(), self._stream())
        else:
            _lib.call('sb_intmat_contract', jac.data_ptr(), tot_ptr, self.n_valid, self.np_sub, self.n_lenses,
                      self.field, self._slot.data_ptr(), pix2col.data_ptr(), IF.data_ptr(), n_modes, ld,
                      float(2.0 * dm.sign), im.data_ptr(), self._stream())
        return im

    def resampled_ifunc(self, dm, top=0, left=0):
        """The mirror's influence functions on the SH's resampled grid (one row
        per mode, a column per field pixel, rows padded to 32 floats) with the
        identity column map; cached per mirror and crop."""
        key = (id(dm), dm._IF.data_ptr(), top, left)
        cache = getattr(self, '_if_cache', None)
        if cache is not None and cache[0] == key:
            return cache[1]
        n_modes = dm._IF.shape[0]
        rows, cols = self.in_shape
        p2c = pixel_to_column(dm._ifunc.idx_inf_func, tuple(dm.layer.phaseInNm.shape), rows, top, left)
        if rows != cols:
            raise ValueError('ShSlopesAdjoint: square SH input fields only')
        p2c = torch.as_tensor(p2c, device=self.device).long()
        keep = p2c >= 0
        M = self.resample_matrix()
        n_out = self.field * self.field
        ld = (n_out + 31) // 32 * 32
        IF = torch.zeros((n_modes, ld), dtype=torch.float32, device=self.device)
        for m0 in range(0, n_modes, 64):
            m1 = min(n_modes, m0 + 64)
            src = torch.zeros((rows * cols, m1 - m0), dtype=torch.float64, device=self.device)
            src[keep] = dm._IF[m0:m1, p2c[keep]].t().double()
            IF[m0:m1, :n_out] = torch.sparse.mm(M, src).t().float()
        out = (IF, ld, torch.arange(n_out, dtype=torch.int32, device=self.device))
        self._if_cache = (key, out)
        return out

    # TMA contraction limits: np_sub 4 or 8, at most 992 field columns,
    # influence-function rows of a multiple of 32 floats, a row segment of at
    # most 7168 floats (two ring stages of four modes in one CTA's shared memory)
    # contraction form of ``intmat``: 'lenslet' (the influence functions
    # copied once per mirror into a lenslet-major layout, then streamed),
    # 'rows' (streamed by TMA from the mirror's own layout) or 'gather'; the
    # first two fall back to the next when their limits are not met, and all
    # three give the same matrix bit for bit
    contraction = 'lenslet'
    LENSLET_NP_SUB = (4, 8)
    LENSLET_MAX_BYTES = 16 << 30

    def lenslet_ifunc(self, IF, ld, pix2col):
        """The influence functions under the valid sub-apertures in the
        lenslet-major layout of sb_intmat_contract_lenslets (n_modes x n_valid
        x np_sub x np_sub floats, built by sb_intmat_lenslet_ifunc), or None
        when np_sub or its size is outside the limits; cached per mirror and
        column map (an influence-function tensor changed in place needs
        ``self._ifl_cache = None`` before the next matrix)."""
        n_modes = IF.shape[0]
        nbytes = 4 * n_modes * self.n_valid * self.np_sub ** 2
        if self.np_sub not in self.LENSLET_NP_SUB or nbytes > self.LENSLET_MAX_BYTES:
            return None
        key = (IF.data_ptr(), n_modes, int(ld), pix2col.data_ptr())
        cache = getattr(self, '_ifl_cache', None)
        if cache is None or cache[0] != key:
            self._ifl_cache = None
            ifl = torch.empty((n_modes, self.n_valid, self.np_sub, self.np_sub), dtype=torch.float32,
                              device=self.device)
            lens = self._lenslet.to(torch.int32)
            p2c = pix2col.to(torch.int32)
            _lib.call('sb_intmat_lenslet_ifunc', IF.data_ptr(), n_modes, int(ld), lens.data_ptr(), self.n_valid,
                      self.np_sub, self.n_lenses, self.field, p2c.data_ptr(), ifl.data_ptr(), self._stream())
            # the tables stay referenced until the copy has run
            cache = (key, ifl, IF, pix2col, lens, p2c)
            self._ifl_cache = cache
        return cache[1]

    TMA_NP_SUB = (4, 8)
    TMA_MAX_COLUMNS = 992
    TMA_MAX_SEGMENT = 7168

    def _segments(self, pix2col, IF, ld):
        """(device table, largest count) of the row segments for the TMA
        contraction, or None when its limits are not met (then the
        gather kernel runs); cached per mirror column map."""
        if (self.np_sub not in self.TMA_NP_SUB or self.field > self.TMA_MAX_COLUMNS or ld % 32 or
                IF.data_ptr() % 16):
            return None
        key = (pix2col.data_ptr(), int(ld))
        cache = getattr(self, '_seg_cache', None)
        if cache is None or cache[0] != key:
            seg, seg_max = row_segments(pix2col.cpu().numpy(), self._lenslet.cpu().numpy(), self.n_lenses,
                                        self.np_sub, self.field, ld)
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
        if shape != self.in_shape:
            raise ValueError('pushpull_intmat: the mirror grid must be the SH input grid')
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
                    Af, Pf = self.resampled(A, phase, st)
                    _lib.call('sb_sh_forward', plan_sh, Af.data_ptr(), Pf.data_ptr(), A.data_ptr(), A.numel(),
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
