"""Assemble and run the single-conjugate Shack-Hartmann closed loop.

``build_scao(cfg)`` wires the processing objects exactly as the reference's
SCAO SH configuration does (main/scao/params_scao_sh.yml; trigger order of
simul.py:109-135): AtmoEvolution -> AtmoPropagation (atmosphere + pupil stop
+ the DM layer of the previous step) -> SH -> CCD -> ShSlopec -> Modalrec ->
Integrator -> DM.  ``ScaoLoop`` runs it either object by object through
``LoopControl`` (the reference's scheduling) or as one CUDA graph holding
every object's ``trigger_code`` for a step; all loop state (layer positions,
CCD frame counter, integrator state, DM shape) lives on the device, so each
graph replay is a full new step.
"""
import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.ifunc import IFunc
from specula_b200.data_objects.pupilstop import Pupilstop
from specula_b200.data_objects.recmat import Recmat
from specula_b200.data_objects.simul_params import SimulParams
from specula_b200.data_objects.source import Source
from specula_b200.data_objects.subap_data import SubapData
from specula_b200.lib.make_mask import make_mask
from specula_b200.loop_control import LoopControl
from specula_b200.processing_objects.atmo_evolution import AtmoEvolution
from specula_b200.processing_objects.atmo_propagation import AtmoPropagation
from specula_b200.processing_objects.ccd import CCD
from specula_b200.processing_objects.dm import DM
from specula_b200.processing_objects.integrator import Integrator
from specula_b200.processing_objects.modalrec import Modalrec
from specula_b200.processing_objects.sh import SH
from specula_b200.processing_objects.sh_slopec import ShSlopec

RAD2ASEC = 180 * 3600 / math.pi


@dataclass
class ScaoConfig:
    """Synthetic SCAO SH system; defaults are the 8 m / 20x20 system."""
    pixel_pupil: int = 160
    diameter_m: float = 8.0
    obsratio: float = 0.14
    n_lenses: int = 20
    subap_npx: int = 8
    wavelength_nm: float = 750.0
    pxscale_over_lamd: float = 0.875       # detector pixel in lambda/d_sub
    fov_ovs_coeff: float = 1.0
    heights: list = field(default_factory=lambda: [0.0])
    cn2: list = field(default_factory=lambda: [1.0])
    wind_speed: list = field(default_factory=lambda: [10.0])
    wind_direction: list = field(default_factory=lambda: [0.0])
    r0: float = 0.15
    L0: float = 25.0
    pixel_phasescreens: int = 1024
    screen_seed: int = 1
    n_modes: int = 54
    gain: float = 0.5
    delay: float = 2
    photons_per_subap: float = 1e3
    readout_noise: float = 3.0
    photon_noise: bool = True
    time_step: float = 0.001
    seed: int = 1234
    subap_threshold: float = 0.5           # valid sub-apertures: illumination above this fraction (< 0: all)
    noise_seed: int = 1                    # detector seeds: photon noise_seed, read-out noise_seed + 1
    sh_dft: str = 'fp32'                   # SH DFTs: 'fp32' (CUDA cores) or 'split_bf16' (tensor cores)

    @property
    def pitch(self):
        return self.diameter_m / self.pixel_pupil

    @property
    def seeing(self):
        # r0 = 0.9759 * 0.5 / (seeing * 4.848) (atmo_evolution.py:265)
        return 0.9759 * 0.5 / (self.r0 * 4.848)


def elt_config(n_modes=500, layers=7, fft_pad=2, seed=1234):
    """39 m / 640 px / 80x80 SH / 6 px, 7-layer atmosphere with random winds
    5-30 m/s and random directions (seeded)."""
    rng = np.random.default_rng(seed)
    cn2 = [0.5, 0.15, 0.1, 0.1, 0.05, 0.05, 0.05][:layers]
    cn2 = list(np.array(cn2) / np.sum(cn2))
    heights = [0.0, 1000.0, 2000.0, 4000.0, 8000.0, 12000.0, 16000.0][:layers]
    return ScaoConfig(pixel_pupil=640, diameter_m=39.0, n_lenses=80, subap_npx=6,
                      pxscale_over_lamd=1.0 if fft_pad == 2 else 0.5, heights=heights, cn2=cn2,
                      wind_speed=list(rng.uniform(5, 30, layers)), wind_direction=list(rng.uniform(0, 360, layers)),
                      pixel_phasescreens=2048, n_modes=n_modes, seed=seed)


class ScaoLoop:
    def __init__(self, cfg: ScaoConfig, device_idx=0, ifunc=None, recmat=None):
        self.cfg = cfg
        dev = torch.device('cuda', device_idx)
        self.device = dev
        c = cfg
        sp = SimulParams(pixel_pupil=c.pixel_pupil, pixel_pitch=c.pitch, time_step=c.time_step)
        self.simul_params = sp
        rng = np.random.default_rng(c.seed)
        pupil = make_mask(c.pixel_pupil, c.obsratio, 1.0)
        self.pupil = pupil
        nv = int(pupil.sum())
        d_sub = c.diameter_m / c.n_lenses
        lamd = c.wavelength_nm * 1e-9 / d_sub * RAD2ASEC
        pxs = c.pxscale_over_lamd * lamd
        # photon flux: photons_per_subap per valid (fully lit) sub-aperture per frame
        n_valid_est = max(1, int(round(pupil.sum() / (c.pixel_pupil / c.n_lenses) ** 2)))
        phot_total = c.photons_per_subap * n_valid_est
        S0 = phot_total / (pupil.sum() * c.pitch ** 2 * c.time_step * 1.0)

        # per-step inputs: float64 device vectors, read in place by AtmoEvolution
        nl = len(c.heights)
        self.n_inputs = 1 + 2 * nl
        self._inputs = torch.tensor([c.seeing] + list(c.wind_speed) + list(c.wind_direction), dtype=torch.float64,
                                    device=dev)
        self.seeing = BaseValue(value=self._inputs[0:1], target_device_idx=device_idx)
        self.wind_speed = BaseValue(value=self._inputs[1:1 + nl], target_device_idx=device_idx)
        self.wind_direction = BaseValue(value=self._inputs[1 + nl:], target_device_idx=device_idx)
        self.atmo = AtmoEvolution(sp, L0=c.L0, heights=c.heights, Cn2=c.cn2, data_dir='',
                                  pixel_phasescreens=c.pixel_phasescreens, seed=c.screen_seed,
                                  target_device_idx=device_idx)
        self.atmo.inputs['seeing'].set(self.seeing)
        self.atmo.inputs['wind_speed'].set(self.wind_speed)
        self.atmo.inputs['wind_direction'].set(self.wind_direction)
        self.pupilstop = Pupilstop(sp, obs_diam=c.obsratio, target_device_idx=device_idx)
        if ifunc is None:
            g = torch.Generator(device=dev).manual_seed(c.seed)
            ifunc = torch.randn((c.n_modes, nv), device=dev, generator=g) * 10.0
        self.dm = DM(sp, 0, ifunc=IFunc(ifunc=ifunc, mask=pupil, target_device_idx=device_idx),
                     target_device_idx=device_idx)
        src = Source([0.0, 0.0], 8, c.wavelength_nm, phot_density_value=S0)
        self.prop = AtmoPropagation(sp, {'on_axis_source': src}, target_device_idx=device_idx)
        self.prop.inputs['atmo_layer_list'].set(self.atmo.layer_list)
        self.prop.inputs['common_layer_list'].set([self.pupilstop, self.dm.layer])
        self.sh = SH(wavelengthInNm=c.wavelength_nm, subap_wanted_fov=c.subap_npx * pxs, sensor_pxscale=pxs,
                     subap_on_diameter=c.n_lenses, subap_npx=c.subap_npx, fov_ovs_coeff=c.fov_ovs_coeff,
                     dft=c.sh_dft, target_device_idx=device_idx)
        self.sh.inputs['in_ef'].set(self.prop.outputs['out_on_axis_source_ef'])
        side = c.n_lenses * c.subap_npx
        self.ccd = CCD(sp, size=[side, side], dt=c.time_step, bandw=1.0, photon_noise=c.photon_noise,
                       readout_noise=c.readout_noise > 0, readout_level=c.readout_noise, quantum_eff=1.0,
                       photon_seed=c.noise_seed, readout_seed=c.noise_seed + 1, target_device_idx=device_idx)
        self.ccd.inputs['in_i'].set(self.sh.outputs['out_i'])
        idxs, dmap = valid_subaps(pupil, c.n_lenses, c.subap_npx, c.subap_threshold)
        self.subapdata = SubapData(idxs=idxs, display_map=dmap, nx=c.n_lenses, ny=c.n_lenses,
                                   target_device_idx=device_idx)
        self.slopec = ShSlopec(self.subapdata, target_device_idx=device_idx)
        self.slopec.inputs['in_pixels'].set(self.ccd.outputs['out_pixels'])
        nsl = 2 * len(idxs)
        if recmat is None:
            g = torch.Generator(device=dev).manual_seed(c.seed + 1)
            recmat = torch.randn((c.n_modes, nsl), device=dev, generator=g) * (1.0 / math.sqrt(nsl))
        self.rec = Modalrec(recmat=Recmat(recmat, target_device_idx=device_idx), target_device_idx=device_idx)
        self.rec.inputs['in_slopes'].set(self.slopec.outputs['out_slopes'])
        self.integ = Integrator(sp, int_gain=[c.gain] * c.n_modes, delay=c.delay, target_device_idx=device_idx)
        self.integ.inputs['delta_comm'].set(self.rec.outputs['out_modes'])
        self.dm.inputs['in_command'].set(self.integ.outputs['out_comm'])
        self.objects = [self.atmo, self.prop, self.sh, self.ccd, self.slopec, self.rec, self.integ, self.dm]
        self.loop = LoopControl()
        for k, o in enumerate(self.objects):
            self.loop.add(o, k)
        self.graph = None
        self.pipelined = False
        self.steps_per_replay = 1
        self.io_inputs = None
        self.io_outputs = None
        self.n_valid_subaps = len(idxs)
        self.n_valid_pixels = nv

    def start(self):
        for v in (self.seeing, self.wind_speed, self.wind_direction):
            v.generation_time = 0
        self.loop.start(1e9, self.cfg.time_step)

    def step_eager(self):
        """One step object by object (check_ready / trigger / post_trigger)."""
        t = self.loop.t
        for v in (self.seeing, self.wind_speed, self.wind_direction):
            v.generation_time = t
        self.loop.iter()

    def _point_inputs(self, vec):
        """Make the seeing / wind BaseValues views of a float64 device vector
        laid out as [seeing, wind_speed (n), wind_direction (n)]."""
        nl = len(self.cfg.heights)
        self.seeing.value = vec[0:1]
        self.wind_speed.value = vec[1:1 + nl]
        self.wind_direction.value = vec[1 + nl:]

    def capture(self, pipelined=True, io=False, fuse_atmo=None, fuse_chain=None, early_atmo=False, io_slots=1):
        """Capture whole steps in a CUDA graph.  Call after at least one eager
        step, so the time step used by AtmoEvolution is the loop's (the first
        step has delta_time = 0).

        Sequential form: one step, every object's trigger_code in trigger order.

        Pipelined form (integer integrator delay >= 1): the DM command of step
        t is the integrator output computed at step t-delay, known when step t
        starts, so the DM projection of step t (HBM-bound) runs on a second
        stream concurrently with AtmoEvolution..Integrator of step t
        (latency-bound).  The DM phase is double-buffered: step t writes
        buffer t%2 while the propagation of step t reads buffer (t-1)%2,
        which is the reference's ``dm.out_layer:-1`` input; only that
        propagation waits for DM(t-1), so AtmoEvolution of step t overlaps
        the end of DM(t-1).  The graph holds two steps so the buffers
        alternate statically; after each replay the DM layer tensor holds the
        latest DM phase, as in the sequential form.

        ``fuse_atmo`` (pipelined form): AtmoEvolution and AtmoPropagation as
        one launch (sb_atmo_propagate_batched with one system; the same
        bits), which then waits for DM(t-1) as the propagation does; its
        smaller HBM traffic leaves more to the DM projection (ELT step 110.5
        against 113 us).  None: fused whenever the layers allow it.

        ``fuse_chain`` (both forms): SH, CCD and ShSlopec as two launches
        (sb_sh_ccd_slopec: the SH forward, then normalisation, detector and
        CoG on each lenslet's pixels in shared memory) instead of five; the
        same bits.  None: fused whenever the objects allow it.

        ``io_slots`` (with ``io``): that many graphs of the same two steps,
        each with its own input / output slots (``io_inputs_slots[k]``,
        ``io_outputs_slots[k]``, run by ``replay(k)``), so a caller can copy
        the next replay's inputs and the last replay's results while a
        replay runs; ``io_inputs`` / ``io_outputs`` are slot 0's.

        ``early_atmo`` (pipelined form with both fusions and the FP32 SH):
        the mirror term of the propagation moves into the SH's field read
        (sb_sh_ccd_slopec with the mirror arguments, which also writes the
        propagated field), so the atmosphere of a step no longer waits for
        the previous mirror: both steps' atmospheres run on a third stream
        from the start of the replay, into per-step buffers, and only the
        SH waits for DM(t-1).  The chain that must end before the next DM
        projection is then SH, detector/CoG and reconstructor.  The same
        bits.  Off by default: on the ELT step it measured 117.9 us against
        109.7 us for the fused form, the two atmospheres competing with the
        replay's first DM projection for HBM and SMs.
        """
        self.step_eager()
        torch.cuda.synchronize(self.device)
        self.atmo.delta_time = self.atmo.t_to_seconds(self.loop.dt)
        g = torch.cuda.CUDAGraph()
        self.pipelined = bool(pipelined and self.integ.next_output_available)
        if fuse_atmo is None:
            fuse_atmo = self._can_fuse_atmo()
        fuse_atmo = bool(fuse_atmo and self.pipelined)
        self.fused_atmo = fuse_atmo
        if fuse_chain is None:
            fuse_chain = self._can_fuse_chain()
        self.fused_chain = bool(fuse_chain)
        if self.fused_chain:
            self._setup_chain()
        # measured slower on the ELT step (117.9 against 109.7 us: both atmospheres then compete with the
        # first DM projection of the replay), so it is chosen only when asked for
        early_atmo = bool(early_atmo)
        self.early_atmo = bool(early_atmo and self.pipelined and self.fused_atmo and self.fused_chain)
        if early_atmo and not self.early_atmo:
            raise NotImplementedError('ScaoLoop.capture: the early atmosphere needs the pipelined form with the '
                                      'fused atmosphere and the fused SH / detector / slope chain')
        if io and not self.pipelined:
            raise ValueError('ScaoLoop.capture: io slots need the pipelined form (integer integrator delay >= 1)')
        if not self.pipelined:
            with torch.cuda.graph(g):
                self.atmo.trigger_code()
                self.prop.trigger_code()
                self._chain()
                self._rec_integ()
                self.dm.trigger_code()
            self.steps_per_replay = 1
        else:
            dm_buf = [self.dm.layer.phaseInNm, torch.empty_like(self.dm.layer.phaseInNm)]
            dm_buf[1].copy_(dm_buf[0])
            nxt = [torch.empty_like(self.integ.out_comm.value) for _ in range(2)]
            # after the eager step t0 (even), step t0+1 will emit state[:, delay-1]
            nxt[1].copy_(self.integ.next_output())
            # in steady state the DM projection (HBM-bound, one CTA per SM)
            # is the critical path: DM(t+1) follows DM(t), and the chain of
            # step t, which must end before DM(t+1), has slack once DM(t-1)
            # is done.  The DM's side stream gets the high priority, so the
            # chain's CTAs fill in around it (measured 111-113 us per ELT
            # step against 113.5-115 us the other way round)
            side = torch.cuda.Stream(self.device, priority=-1)
            cap = torch.cuda.Stream(self.device, priority=0)
            self._side = side
            self._cap = cap
            self._bufs = (dm_buf, nxt)
            n_slots = max(1, int(io_slots)) if io else 1
            if io:
                nsl = self.slopec.slopes.slopes.numel()
                nm = self.integ.out_comm.value.numel()
                self.io_inputs_slots = [self._inputs.repeat(2, 1).contiguous() for _ in range(n_slots)]
                self.io_outputs_slots = [torch.zeros((2, nsl + nm), dtype=torch.float32, device=self.device)
                                         for _ in range(n_slots)]
            self.graphs = []
            for k in range(n_slots):
                gk = g if k == 0 else torch.cuda.CUDAGraph()
                if io:
                    self.io_inputs, self.io_outputs = self.io_inputs_slots[k], self.io_outputs_slots[k]
                if self.early_atmo:
                    self._capture_early(gk, side, cap, dm_buf, nxt, io)
                else:
                    self._capture_pipelined(gk, side, cap, dm_buf, nxt, io, fuse_atmo)
                self.graphs.append(gk)
            if io:
                self.io_inputs, self.io_outputs = self.io_inputs_slots[0], self.io_outputs_slots[0]
                self._point_inputs(self._inputs)
            self.steps_per_replay = 2
        torch.cuda.synchronize(self.device)
        self.graph = g
        return g

    def _capture_pipelined(self, g, side, cap, dm_buf, nxt, io, fuse_atmo):
        """The pipelined two-step graph (see capture())."""
        if io:
            nsl = self.slopec.slopes.slopes.numel()
        with torch.cuda.graph(g, stream=cap):
            main = torch.cuda.current_stream(self.device)
            dm_done = None
            for step, par in enumerate((1, 0)):    # odd step, then even step
                # DM(t) needs the integrator output of step t-1
                side.wait_stream(main)
                with torch.cuda.stream(side):
                    self.dm.project(nxt[par], dm_buf[par])
                    ev = torch.cuda.Event()
                    ev.record(side)
                # AtmoEvolution(t) does not depend on the mirror
                if io:
                    self._point_inputs(self.io_inputs[step])
                if fuse_atmo:
                    if dm_done is not None:
                        main.wait_event(dm_done)
                    self._atmo_propagate(dm_buf[1 - par])
                else:
                    self.atmo.trigger_code()
                    # the propagation of step t reads DM(t-1): the previous
                    # replay (already complete) for the first step of the graph
                    if dm_done is not None:
                        main.wait_event(dm_done)
                    self.prop.trigger_code(phase_override={id(self.dm.layer): dm_buf[1 - par]})
                self._chain()
                self._rec_integ(out_next=nxt[1 - par])
                if io:
                    self.io_outputs[step, :nsl].copy_(self.slopec.slopes.slopes)
                    self.io_outputs[step, nsl:].copy_(self.integ.out_comm.value)
                dm_done = ev
            main.wait_stream(side)

    def _capture_early(self, g, side, cap, dm_buf, nxt, io):
        """The pipelined two-step graph with the atmosphere of both steps on
        a stream of its own (see capture(early_atmo=...))."""
        L = self.cfg.pixel_pupil
        # per-step product / sum of the turbulence and the stop (the mirror is applied by the SH)
        self._early = [(torch.empty((L, L), dtype=torch.float32, device=self.device),
                        torch.empty((L, L), dtype=torch.float32, device=self.device)) for _ in range(2)]
        atm = torch.cuda.Stream(self.device, priority=0)
        self._atm = atm
        if io:
            nsl = self.slopec.slopes.slopes.numel()
        with torch.cuda.graph(g, stream=cap):
            main = torch.cuda.current_stream(self.device)
            atm.wait_stream(main)
            atmo_done = []
            for step, par in enumerate((1, 0)):        # odd step, then even step
                with torch.cuda.stream(atm):
                    if io:
                        self._point_inputs(self.io_inputs[step])
                    self._atmo_propagate(None, out=self._early[par])
                    ev = torch.cuda.Event()
                    ev.record(atm)
                atmo_done.append(ev)
            dm_done = None
            for step, par in enumerate((1, 0)):
                # DM(t) needs the integrator output of step t-1
                side.wait_stream(main)
                with torch.cuda.stream(side):
                    self.dm.project(nxt[par], dm_buf[par])
                    ev = torch.cuda.Event()
                    ev.record(side)
                main.wait_event(atmo_done[step])
                # the SH applies DM(t-1): the previous replay (already complete) for the first step
                if dm_done is not None:
                    main.wait_event(dm_done)
                self._sh_ccd_slopec(mirror=dm_buf[1 - par], partial=self._early[par])
                self._rec_integ(out_next=nxt[1 - par])
                if io:
                    self.io_outputs[step, :nsl].copy_(self.slopec.slopes.slopes)
                    self.io_outputs[step, nsl:].copy_(self.integ.out_comm.value)
                dm_done = ev
            main.wait_stream(side)
            main.wait_stream(atm)

    def _can_early_atmo(self):
        """True when the mirror term can move into the SH's field read: the
        fused atmosphere and chain apply, the SH runs its FP32 DFTs on the
        pupil grid itself (one phase sample per lenslet pixel)."""
        sh = self.sh
        g = sh.geometry
        return (self._can_fuse_atmo() and self._can_fuse_chain() and sh._forward == 'sb_sh_forward' and
                not g.do_interpolation and int(sh._plan.field_ld) == self.cfg.pixel_pupil and
                int(sh._plan.n_lenses) * int(sh._plan.np_sub) == self.cfg.pixel_pupil)

    def _chain(self):
        """SH, CCD and ShSlopec of one step: two launches when fused, else
        the three objects' trigger_code."""
        if self.fused_chain:
            self._sh_ccd_slopec()
        else:
            self.sh.trigger_code()
            self.ccd.trigger_code()
            self.slopec.trigger_code()

    def lenslet_subap_map(self):
        """Valid sub-aperture index of every lenslet (row-major n x n, -1 when
        not valid), when every row of the sub-aperture table is one lenslet's
        npx x npx detector box listed row-major; else None."""
        n, npx = self.cfg.n_lenses, self.cfg.subap_npx
        side = n * npx
        idxs = np.asarray(self.subapdata.idxs)
        if idxs.ndim != 2 or idxs.shape[1] != npx * npx:
            return None
        rr, cc = np.meshgrid(np.arange(npx), np.arange(npx), indexing='ij')
        box = (rr * side + cc).ravel()
        r0, c0 = idxs[:, 0] // side, idxs[:, 0] % side
        if np.any(r0 % npx) or np.any(c0 % npx) or np.any(r0 >= side) or np.any(c0 >= side):
            return None
        if not np.array_equal(idxs, idxs[:, :1] + box[np.newaxis, :]):
            return None
        lens = (r0 // npx) * n + c0 // npx
        if len(np.unique(lens)) != len(lens):
            return None
        out = np.full(n * n, -1, dtype=np.int32)
        out[lens] = np.arange(len(lens), dtype=np.int32)
        return out

    def _can_fuse_chain(self):
        """True when sb_sh_ccd_slopec computes exactly what SH + CCD + ShSlopec
        do: plain (not interpolated, not LGS) SH with the FP32 or split-BF16
        DFTs, a detector of the SH frame size reading out every step without
        binning, the slope computer reading that detector's pixels with no
        option beyond thr_value, and a sub-aperture table of row-major lenslet
        boxes."""
        sh, ccd, sl = self.sh, self.ccd, self.slopec
        return (not sh.geometry.do_interpolation and sh._kernelobj is None and
                sh._forward in ('sb_sh_forward', 'sb_sh_forward_split_bf16') and
                ccd._bin_scratch is None and ccd._cte is None and int(ccd._frames_per_read) == 1 and
                ccd._in_i.i.data_ptr() == sh._out_i.i.data_ptr() and
                sl._pix.pixels.data_ptr() == ccd._pixels.pixels.data_ptr() and sl.options_plain() and
                int(sh._plan.subap_npx) <= 16 and self.lenslet_subap_map() is not None)

    def _setup_chain(self):
        if not self._can_fuse_chain():
            raise NotImplementedError('ScaoLoop: the fused SH / CCD / slope chain needs a plain SH, a detector read '
                                      'every step without binning and lenslet-box sub-apertures')
        self._lenslet_subap = torch.as_tensor(self.lenslet_subap_map(), device=self.device)
        nb = _lib.load().sb_sh_ccd_slopec_scratch_bytes(ctypes.byref(self.sh._plan), self.slopec._plan.n_subaps)
        self._chain_scratch = torch.zeros(nb, dtype=torch.uint8, device=self.device)

    def _sh_ccd_slopec(self, mirror=None, partial=None):
        """The fused chain on the propagated field; with ``mirror`` (a DM
        phase buffer) and ``partial`` ((A, phase) of turbulence and stop) the
        SH applies the mirror itself and writes the propagated field."""
        sh, ccd, sl = self.sh, self.ccd, self.slopec
        ef = sh._in_ef
        st = sh.stream_handle()
        mode = 0 if sh._forward == 'sb_sh_forward' else 1
        if mirror is None:
            A, P, mA, mP, fA, fP = ef.A, ef.phaseInNm, None, None, None, None
        else:
            A, P = partial
            mA, mP, fA, fP = self.dm.layer.A.data_ptr(), mirror.data_ptr(), ef.A.data_ptr(), ef.phaseInNm.data_ptr()
        _lib.call('sb_sh_ccd_slopec', ctypes.byref(sh._plan), mode, A.data_ptr(), P.data_ptr(),
                  A.data_ptr(), A.numel(), mA, mP, fA, fP, sh._photon_scale, sh._out_i.i.data_ptr(),
                  ctypes.byref(ccd._params),
                  ccd._integrated_i.i.data_ptr(), ccd._pixels.pixels.data_ptr(), ctypes.byref(sl._plan),
                  self._lenslet_subap.data_ptr(), sl._target.data_ptr(), sl._flux.data_ptr(),
                  self._chain_scratch.data_ptr(), self._chain_scratch.numel(), st)
        sl._apply_products(st)

    def _can_fuse_atmo(self):
        """True when the fused atmosphere kernel reads every input in its
        layout: pupil-sized dense layers in the SCAO order, and the stop's
        and the mirror's amplitude and phase as dense L x L arrays."""
        prop = self.prop
        L = self.cfg.pixel_pupil

        def dense(t):
            return t is not None and tuple(t.shape) == (L, L) and t.is_contiguous() and t.dtype == torch.float32

        return (not prop._interpolated and len(prop._layers) >= 2 and prop._layers[-1] is self.dm.layer and
                prop._layers[-2] is self.pupilstop and
                all(dense(ly.phaseInNm) for ly in prop._layers) and
                dense(self.pupilstop.A) and dense(self.dm.layer.A) and
                len(prop._layers) - 2 == len(self.atmo.layer_list) and
                all(a is b for a, b in zip(prop._layers[:-2], self.atmo.layer_list)))

    def _atmo_propagate(self, dm_phase, out=None):
        """AtmoEvolution.trigger_code + AtmoPropagation.trigger_code in one
        launch: pupil-sized turbulence layers, then the pupil stop and the
        mirror (phase read from ``dm_phase``; None: no mirror term).  The
        field goes to the propagation output, or to ``out`` = (A, phase)."""
        atmo, prop = self.atmo, self.prop
        nl = atmo.n_phasescreens
        if not self._can_fuse_atmo():
            raise NotImplementedError('ScaoLoop: the fused atmosphere needs pupil-sized layers in the SCAO order')
        consts = atmo.inputs_struct(atmo.delta_time)
        ins = (_lib.AtmoLayerInputs * nl)()
        for k in range(nl):
            ins[k].seeing = consts.seeing
            ins[k].wind_speed = consts.wind_speed + (8 * k if consts.n_wind_speed > 1 else 0)
            ins[k].wind_direction = consts.wind_direction + (8 * k if consts.n_wind_direction > 1 else 0)
            ins[k].position = atmo._positions.data_ptr() + 8 * k
        ef = prop.outputs['out_on_axis_source_ef']
        L = self.cfg.pixel_pupil
        stop = self.pupilstop
        oA, oP = (ef.A, ef.phaseInNm) if out is None else out
        _lib.call('sb_atmo_propagate_batched', atmo._layers, ins, nl, 1, L, ctypes.byref(consts),
                  atmo._work.data_ptr(), atmo._work.numel(), stop.A.data_ptr(), stop.phaseInNm.data_ptr(),
                  self.dm.layer.A.data_ptr(), None if dm_phase is None else dm_phase.data_ptr(), L * L,
                  oA.data_ptr(), oP.data_ptr(), L * L, atmo.stream_handle())

    def _rec_integ(self, out_next=None):
        """Modalrec + Integrator of this loop as one launch
        (sb_modalrec_integrator), falling back to the two objects when the
        reconstructor output is sliced."""
        rec, integ = self.rec, self.integ
        full = rec.output_slice == slice(None, None, None) and integ._n == rec._R.shape[0]
        if not full:
            rec.trigger_code()
            integ.trigger_code(out_next=out_next)
            return
        s = rec.local_inputs['in_slopes'].slopes
        integ._plan.out_next = None if out_next is None else out_next.data_ptr()
        try:
            _lib.call('sb_modalrec_integrator', rec._R.data_ptr(), rec._R.shape[0], rec._R.shape[1],
                      rec._R.stride(0), s.data_ptr(), rec._all_modes.data_ptr(), ctypes.byref(integ._plan),
                      integ.out_comm.value.data_ptr(), rec.stream_handle())
        finally:
            integ._plan.out_next = None

    def replay(self, slot=0):
        """Run the captured graph (of input / output slot ``slot``):
        ``steps_per_replay`` loop steps."""
        (self.graph if slot == 0 else self.graphs[slot]).replay()

    # kernels launched by one captured step (for the launch count): atmo
    # advance + evolve, propagate, SH forward + normalise, CCD, slopes (2),
    # reconstructor with the integrator, DM projection
    KERNELS_PER_STEP = 10

    @property
    def kernels_per_step(self):
        """Kernels of one captured step: one fewer with the atmosphere and
        the propagation fused, three fewer with the SH / CCD / slope chain
        fused (five launches become two)."""
        return (self.KERNELS_PER_STEP - (1 if getattr(self, 'fused_atmo', False) else 0) -
                (3 if getattr(self, 'fused_chain', False) else 0))


def valid_subaps(pupil, n_lenses, npx, threshold=0.5):
    """Sub-apertures whose pupil illumination exceeds `threshold` of the
    brightest, with their detector pixel tables in the ShSubapCalibrator
    layout (sh_subap_calibrator.py:46-92: boxes scanned lenslet-column first,
    row-major pixels, display_map = j*n + i)."""
    pix = pupil.shape[0]
    ps = pix // n_lenses
    illum = pupil[:n_lenses * ps, :n_lenses * ps].reshape(n_lenses, ps, n_lenses, ps).sum(axis=(1, 3))
    side = n_lenses * npx
    idxs, dmap = [], []
    for i in range(n_lenses):
        for j in range(n_lenses):
            # box rows come from lenslet column j, box columns from row i
            if threshold < 0 or illum[j, i] > threshold * illum.max():
                r0, c0 = j * npx, i * npx
                rr, cc = np.meshgrid(np.arange(r0, r0 + npx), np.arange(c0, c0 + npx), indexing='ij')
                idxs.append((rr * side + cc).ravel())
                dmap.append(j * n_lenses + i)
    return np.array(idxs, dtype=np.int64), np.array(dmap, dtype=np.int64)
