"""Gradient of a closed-loop metric through the whole SCAO loop: reverse mode
with checkpointed recomputation.

Loop (noise-free detector, integer integrator delay d, the DM read one step
late as the reference's ``dm.out_layer:-1`` input):

    phi_t = atm_t + sign * IF^T y_{t-d-1}        (AtmoPropagation of the DM layer)
    s_t   = SH+CoG(A, phi_t)                      (sb_sh_forward + sb_slopec)
    m_t   = R s_t                                 (sb_modalrec)
    y_t   = ff * y_{t-1} + g * m_t                (iir_filter.py:171-197 with num=[0,g], den=[-ff,1])
    L     = (1/T) sum_t var_A(phi_t)              (residual wavefront variance over the pupil)

``LoopGradient.gradient(g, R)`` returns L, dL/dg (per-mode gains) and dL/dR
(the reconstructor).  The forward pass keeps only a checkpoint of the loop
state (atmosphere positions, the last d+1 integrator outputs) every
``checkpoint_every`` steps plus s_t and m_t (small); the reverse pass
restores each checkpoint, recomputes that segment's residual phases and
runs the adjoint backwards through it:

    lam_y_t = ff * lam_y_{t+1} + lam_c_{t+d+1}
    lam_m_t = g * lam_y_t              dL/dg += lam_y_t * m_t
    lam_s_t = R^T lam_m_t              dL/dR += lam_m_t s_t^T
    psi_t   = dv_t/dphi_t / T + VJP_SH(phi_t; lam_s_t)      (sb_sh_slopes_vjp)
    lam_c_t = sign * IF psi_t[mask]                           (sb_modalrec on the IF)

Every device step is one of the library's CUDA kernels or a cuBLAS product;
the short per-mode vectors are updated with torch element-wise operations.
"""
import torch

from specula_b200 import _lib
from specula_b200.lib.sh_adjoint import ShSlopesAdjoint


class LoopGradient:
    def __init__(self, loop, n_steps, checkpoint_every=50):
        """``loop``: a specula_b200.scao.ScaoLoop (its objects are used as
        kernels; its own integrator, DM state and CCD are not touched).
        The integrator delay must be an integer."""
        integ = loop.integ
        delay = integ.delay
        if delay != int(delay):
            raise NotImplementedError('LoopGradient: fractional integrator delays are not supported')
        if integ._n_num != 2 or integ._n_den != 2:
            raise NotImplementedError('LoopGradient: the loop filter must be a 2-tap integrator')
        self.loop = loop
        self.T = int(n_steps)
        self.K = int(checkpoint_every)
        if self.T < 1 or self.K < 1:
            raise ValueError('LoopGradient: n_steps and checkpoint_every must be positive')
        self.lag = int(delay) + 1                  # y_{t-lag} drives phi_t
        dev = loop.device
        self.device = dev
        loop.start()
        loop.step_eager()                          # sets every object's inputs and buffers up
        torch.cuda.synchronize(dev)
        self.adj = ShSlopesAdjoint(loop.sh, loop.slopec)
        self.ff = (-integ._den[:, 0]).to(torch.float32).contiguous()
        self.nm = int(integ._n)
        dm = loop.dm
        self.sign = float(dm.sign)
        self.IF, self.ld, self.idx = dm._IF, dm._ld, dm._idx
        self.nv = int(self.idx.numel())
        self.nsl = 2 * self.adj.n_valid
        self.dt = loop.atmo.t_to_seconds(loop.loop.dt)
        self.pos0 = torch.zeros_like(loop.atmo._positions)
        self.ef = loop.prop.outputs[next(iter(loop.prop.outputs))]
        self.dm_buf = torch.zeros_like(dm.layer.phaseInNm)

    # -- one forward step --------------------------------------------------
    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _residual(self, t, c):
        """Advance the atmosphere to step t and return (A, phi_t) with the DM
        driven by command vector c."""
        loop = self.loop
        _lib.call('sb_dm_project', self.IF.data_ptr(), self.nm, self.nv, self.ld, c.data_ptr(), self.nm,
                  self.sign, self.idx.data_ptr(), self.dm_buf.data_ptr(), self._stream())
        loop.atmo.delta_time = 0.0 if t == 0 else self.dt
        loop.atmo.trigger_code()
        loop.prop.trigger_code(phase_override={id(loop.dm.layer): self.dm_buf})
        return self.ef.A, self.ef.phaseInNm

    def _modes(self, R, s, out):
        _lib.call('sb_modalrec', R.data_ptr(), self.nm, self.nsl, R.stride(0), s.data_ptr(), out.data_ptr(),
                  self._stream())
        return out

    @staticmethod
    def _variance(A, phi):
        w = A.reshape(-1).double()
        p = phi.reshape(-1).double()
        sw = w.sum()
        mu = (w * p).sum() / sw
        return (w * (p - mu) ** 2).sum() / sw, mu, sw

    def _run(self, g, R, t0, t1, state, losses, record=None, seg=None):
        """Steps [t0, t1) from ``state`` = (positions, ring of the last `lag`
        integrator outputs, oldest first).  losses: (T,) float64 tensor that
        receives each step's residual variance; record: dict of (T, .)
        tensors s, m filled per step; seg: list receiving (phi_t, active_t)."""
        loop = self.loop
        pos, ring = state
        loop.atmo._positions.copy_(pos)
        ring = [r.clone() for r in ring]
        m = torch.empty(self.nm, dtype=torch.float32, device=self.device)
        for t in range(t0, t1):
            A, phi = self._residual(t, ring[0])
            s, flux = self.adj.slopes(A, phi)
            self._modes(R, s, m)
            y = torch.addcmul(self.ff * ring[-1], g, m)
            ring = ring[1:] + [y]
            v, _, _ = self._variance(A, phi)
            losses[t] = v
            if record is not None:
                record['s'][t].copy_(s)
                record['m'][t].copy_(m)
            if seg is not None:
                seg.append((phi.clone(), self.adj.active_from_flux(flux)))
        return loop.atmo._positions.clone(), ring

    def _initial_state(self):
        return (self.pos0.clone(), [torch.zeros(self.nm, dtype=torch.float32, device=self.device)
                                    for _ in range(self.lag)])

    def _params(self, g, R):
        g = torch.as_tensor(g, dtype=torch.float32, device=self.device).reshape(-1).contiguous()
        R = torch.as_tensor(R, dtype=torch.float32, device=self.device).contiguous()
        if g.numel() != self.nm or tuple(R.shape) != (self.nm, self.nsl):
            raise ValueError(f'LoopGradient: gains ({self.nm},) and reconstructor ({self.nm}, {self.nsl}) expected')
        return g, R

    def loss(self, g, R):
        """Mean residual variance over the T steps (float64)."""
        g, R = self._params(g, R)
        losses = torch.zeros(self.T, dtype=torch.float64, device=self.device)
        self._run(g, R, 0, self.T, self._initial_state(), losses)
        return float(losses.sum()) / self.T

    def trajectory(self, g, R):
        """(L, slopes (T, n_slopes), modes (T, n_modes)) of the forward loop."""
        g, R = self._params(g, R)
        rec = {'s': torch.empty((self.T, self.nsl), dtype=torch.float32, device=self.device),
               'm': torch.empty((self.T, self.nm), dtype=torch.float32, device=self.device)}
        losses = torch.zeros(self.T, dtype=torch.float64, device=self.device)
        self._run(g, R, 0, self.T, self._initial_state(), losses, record=rec)
        return float(losses.sum()) / self.T, rec['s'], rec['m']

    # -- gradient ---------------------------------------------------------
    def gradient(self, g, R):
        """(L, dL/dg, dL/dR) by reverse mode with checkpoints every K steps."""
        g, R = self._params(g, R)
        T, K, dev = self.T, self.K, self.device
        rec = {'s': torch.empty((T, self.nsl), dtype=torch.float32, device=dev),
               'm': torch.empty((T, self.nm), dtype=torch.float32, device=dev)}
        # forward: checkpoints at the segment starts
        ckpt = {}
        state = self._initial_state()
        losses = torch.zeros(T, dtype=torch.float64, device=dev)
        scratch = torch.zeros(T, dtype=torch.float64, device=dev)
        for t0 in range(0, T, K):
            ckpt[t0] = (state[0].clone(), [r.clone() for r in state[1]])
            state = self._run(g, R, t0, min(T, t0 + K), state, losses, record=rec)
        # reverse
        lam_m_all = torch.empty((T, self.nm), dtype=torch.float32, device=dev)
        dg = torch.zeros(self.nm, dtype=torch.float64, device=dev)
        lam_y_next = torch.zeros(self.nm, dtype=torch.float32, device=dev)
        lam_c = {}                                   # t -> sign * IF psi_t
        zero_nm = torch.zeros(self.nm, dtype=torch.float32, device=dev)
        gathered = torch.empty(self.nv, dtype=torch.float32, device=dev)
        for t0 in sorted(ckpt, reverse=True):
            t1 = min(T, t0 + K)
            seg = []
            self._run(g, R, t0, t1, ckpt[t0], scratch, seg=seg)
            A = self.ef.A
            for t in range(t1 - 1, t0 - 1, -1):
                phi, active = seg[t - t0]
                lam_y = torch.addcmul(lam_c.pop(t + self.lag, zero_nm), self.ff, lam_y_next)
                lam_m = g * lam_y
                dg += (lam_y.double() * rec['m'][t].double())
                lam_m_all[t].copy_(lam_m)
                lam_s = torch.mv(R.t(), lam_m).contiguous()
                _, mu, sw = self._variance(A, phi)
                psi = self.adj.vjp(A, phi, lam_s, active=active)
                psi += ((2.0 / (T * sw)) * A.double() * (phi.double() - mu)).float()
                torch.index_select(psi.reshape(-1), 0, self.idx.long(), out=gathered)
                lam_c[t] = self.sign * self._if_gemv(gathered)
                lam_y_next = lam_y
        dR = torch.matmul(lam_m_all.t(), rec['s'])
        return float(losses.sum()) / T, dg.float(), dR

    def _if_gemv(self, v):
        """IF (n_modes x n_valid, row stride ld) @ v with the library GEMV."""
        out = torch.empty(self.nm, dtype=torch.float32, device=self.device)
        _lib.call('sb_modalrec', self.IF.data_ptr(), self.nm, self.nv, self.ld, v.data_ptr(), out.data_ptr(),
                  self._stream())
        return out
