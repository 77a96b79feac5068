"""Oracle: the whole SCAO SH closed-loop step on the CPU (test
infrastructure and timed CPU baseline only).

Chains the restated reference functions in the trigger order of
main/scao/params_scao_sh.yml / simul.py:109-135: AtmoEvolution ->
AtmoPropagation (atmosphere, pupil stop, DM layer of the previous step) ->
SH -> CCD -> ShSlopec -> Modalrec -> Integrator -> DM.
"""
import numpy as np

from . import atmo as oatm, ccd as occd, control as octl, sh as osh, slopec as osl


class OracleScaoLoop:
    def __init__(self, cfg, ifunc, recmat, idxs, pupil, S0, strips=None, precision=1):
        """cfg: a specula_b200.scao.ScaoConfig-like object (plain attributes);
        ifunc (n_modes x n_valid), recmat (n_modes x n_slopes), idxs valid
        sub-aperture tables, pupil mask, S0 photon density; strips: per-layer
        screen strips (computed from the screen seed if None)."""
        c = cfg
        dt = np.float32 if precision == 1 else np.float64
        self.c = c
        self.dtype = dt
        self.pupil = pupil.astype(dt)
        self.ifunc = np.asarray(ifunc, dtype=dt)
        self.recmat = np.asarray(recmat, dtype=dt)
        self.idxs = idxs
        self.S0 = S0
        L = c.pixel_pupil
        if strips is None:
            per = c.pixel_phasescreens // L
            n_sq = -(-len(c.heights) // per)
            squares = [oatm.calc_phasescreen(np.array([c.L0])[0], c.pixel_phasescreens, c.pitch,
                                             seed=c.screen_seed + k, precision=precision) for k in range(n_sq)]
            strips = oatm.prepare_strips(squares, len(c.heights), L, c.cn2, precision=precision)
        self.evo = oatm.AtmoEvolutionOracle(strips, L, c.pitch, precision=precision)
        d_sub = c.diameter_m / c.n_lenses
        lamd = c.wavelength_nm * 1e-9 / d_sub * osh.RAD2ASEC
        pxs = c.pxscale_over_lamd * lamd
        g = osh.sh_geometry(c.wavelength_nm, c.subap_npx * pxs, pxs, c.n_lenses, c.subap_npx, L, c.pitch,
                            fov_ovs_coeff=c.fov_ovs_coeff)
        self.sh = osh.SHOracle(g, c.wavelength_nm, ef_A_for_tables=self.pupil, precision=precision)
        side = c.n_lenses * c.subap_npx
        self.ccd = occd.CCDOracle((side, side), c.time_step, c.time_step, 1.0, photon_noise=c.photon_noise,
                                  readout_noise=c.readout_noise > 0, readout_level=c.readout_noise,
                                  precision=precision)
        self.integ = octl.IntegratorOracle([c.gain] * c.n_modes, delay=c.delay, precision=precision)
        self.dm_phase = np.zeros((L, L), dtype=dt)
        self.mask_idx = np.where(self.pupil)
        self.t = 0
        self.slopes = None
        self.comm = None
        self.frame = None

    def step(self):
        c = self.c
        layers = self.evo.step(self.t, c.seeing, c.wind_speed, c.wind_direction)
        ones = np.ones_like(self.pupil)
        A, P = oatm.propagate_on_axis([ones] * len(layers) + [self.pupil, self.pupil],
                                      layers + [np.zeros_like(self.pupil), self.dm_phase], c.pixel_pupil,
                                      dtype=self.dtype)
        inten = self.sh.forward(A, P, self.S0, c.pitch)
        frame = self.ccd.step(inten)
        if frame is not None:
            self.frame = frame
        s, _ = osl.sh_slopes(self.frame, self.idxs)
        self.slopes = s
        modes = octl.modalrec(self.recmat, s)
        comm = self.integ.step(modes)
        self.comm = comm
        self.dm_phase = octl.dm_phase(self.ifunc, self.pupil, comm, idx=self.mask_idx)
        self.t += int(round(c.time_step * 1e9))
        return s
