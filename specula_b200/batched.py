"""Batched Monte-Carlo of uneven SCAO SH systems on one B200.

Realisations come in geometry groups (same pupil, sub-aperture grid,
wavelength, mirror and reconstructor; their own atmosphere (r0, seed) and
detector noise seeds).  Each realisation is one ``ScaoLoop``'s objects, and
within a group its turbulence layers, field, detector frames, slopes and DM
layer are rows of group stacks.  Per step every group makes one launch per
stage for all its realisations: the atmosphere (``sb_atmo_evolve_batched``,
every layer of every realisation), the propagation
(``sb_propagate_batched``), the SH forward (``sb_sh_forward_batched``, or
``sb_sh_forward_split_bf16_batched`` with ``dft='split_bf16'``), the CCD
(``sb_ccd_step_batched``, per-realisation seeds), the slopes
(``sb_slopec_batched``), the reconstructor (``sb_modalrec_batched``: R read
once for up to 16 realisations), the integrators (one ``sb_integrator`` call)
and the mirror (``sb_dm_project_batched``: the influence functions read once
for up to 16 realisations).  ``capture()`` puts the step of every group into
one CUDA graph, each group on a stream of its own.

``BatchedScao.capture_mc()`` puts the step of every group into the
Monte-Carlo step of the C ABI instead (``sb_mc_step``): six launches per
step, each stage one launch over every realisation of every group, the same
bits as the group-by-group graph.

``BatchedScao.replay_plain()`` runs the same realisations the plain way (each
``ScaoLoop``'s own captured step with the FP32 SH, its own reconstructor and
mirror), for comparison.
"""
import ctypes
import math
from dataclasses import replace

import numpy as np
import torch

from specula_b200 import _lib
from specula_b200.base_value import BaseValue
from specula_b200.processing_objects.integrator import Integrator
from specula_b200.lib.make_mask import make_mask
from specula_b200.scao import ScaoConfig, ScaoLoop, elt_config, valid_subaps


def graph_kernel_count(graph):
    """Kernel nodes of a captured torch CUDA graph (made with keep_graph=True)."""
    from cuda.bindings import runtime as rt
    h = rt.cudaGraph_t(init_value=graph.raw_cuda_graph())
    err, _, n = rt.cudaGraphGetNodes(h, 0)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f'cudaGraphGetNodes: {err}')
    err, nodes, n = rt.cudaGraphGetNodes(h, n)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f'cudaGraphGetNodes: {err}')
    count = 0
    for node in nodes[:n]:
        err, kind = rt.cudaGraphNodeGetType(node)
        if err != rt.cudaError_t.cudaSuccess:
            raise RuntimeError(f'cudaGraphNodeGetType: {err}')
        count += kind == rt.cudaGraphNodeType.cudaGraphNodeTypeKernel
    return count


def seeing_from_r0(r0):
    """Seeing [arcsec] giving r0 [m] at 500 nm (atmo_evolution.py:265)."""
    return 0.9759 * 0.5 / (r0 * 4.848)


def mc_groups(seed=7, n_real=(55, 27, 14), wavelengths=(589.0, 750.0)):
    """The Monte-Carlo mix: 20x20 sub-apertures on 160 px (8 m, 1 layer, 54
    modes), 40x40 on 320 px (8 m, 3 layers, 300 modes) and 74x74 on 592 px
    (39 m, 7 layers, 500 modes) in the given counts, each split between the
    two wavelengths; r0 uniform in [0.08, 0.20] m and the screen / noise seeds
    per realisation.  Returns [(ScaoConfig template, [per-realisation
    ScaoConfig])]."""
    rng = np.random.default_rng(seed)
    e = elt_config()
    sizes = [
        ScaoConfig(pixel_pupil=160, diameter_m=8.0, n_lenses=20, subap_npx=8, n_modes=54),
        ScaoConfig(pixel_pupil=320, diameter_m=8.0, n_lenses=40, subap_npx=6, pxscale_over_lamd=1.0, n_modes=300,
                   heights=[0.0, 4000.0, 10000.0], cn2=[0.6, 0.25, 0.15], wind_speed=[8.0, 15.0, 25.0],
                   wind_direction=[10.0, 130.3, 250.6], pixel_phasescreens=1024),
        ScaoConfig(pixel_pupil=592, diameter_m=39.0, n_lenses=74, subap_npx=6, pxscale_over_lamd=1.0, n_modes=500,
                   heights=e.heights, cn2=e.cn2, wind_speed=e.wind_speed, wind_direction=e.wind_direction,
                   pixel_phasescreens=2048),
    ]
    groups = []
    k = 0
    for cfg, n in zip(sizes, n_real):
        for w, lam in enumerate(wavelengths):
            cnt = (n + 1 - w) // 2
            reals = []
            for _ in range(cnt):
                r0 = float(rng.uniform(0.08, 0.20))
                reals.append(replace(cfg, wavelength_nm=lam, r0=r0, screen_seed=100 + k, noise_seed=1000 + 17 * k))
                k += 1
            if reals:
                groups.append((replace(cfg, wavelength_nm=lam), reals))
    return groups


SH_FORWARD = {'fp32': 'sb_sh_forward_batched', 'split_bf16': 'sb_sh_forward_split_bf16_batched'}


class _Group:
    def __init__(self, template, reals, device_idx, dft='fp32'):
        if dft not in SH_FORWARD:
            raise ValueError(f"dft must be one of {sorted(SH_FORWARD)}, not {dft!r}")
        self.sh_forward = SH_FORWARD[dft]
        # True: atmosphere and propagation as one launch
        # (sb_atmo_propagate_batched, the same bits); the default two launches
        # (sb_atmo_evolve_batched, sb_propagate_batched) measured faster
        self.fuse_atmo = False
        dev = torch.device('cuda', device_idx)
        self.device = dev
        self.n = len(reals)
        c0 = template
        # shared mirror and reconstructor of the group (random, as ScaoLoop's defaults)
        pupil = make_mask(c0.pixel_pupil, c0.obsratio, 1.0)
        nv, nm = int(pupil.sum()), c0.n_modes
        nsl = 2 * len(valid_subaps(pupil, c0.n_lenses, c0.subap_npx, c0.subap_threshold)[0])
        g = torch.Generator(device=dev).manual_seed(c0.seed)
        self.ifunc = torch.randn((nm, nv), device=dev, generator=g) * 10.0
        g = torch.Generator(device=dev).manual_seed(c0.seed + 1)
        self.recmat = torch.randn((nm, nsl), device=dev, generator=g) * (1.0 / math.sqrt(nsl))
        self.loops = [ScaoLoop(c, device_idx=device_idx, ifunc=self.ifunc, recmat=self.recmat) for c in reals]
        L = c0.pixel_pupil
        self.nm, self.nsl, self.L = nm, nsl, L
        # group matrices: rows are the realisations
        self.S = torch.zeros((self.n, nsl), dtype=torch.float32, device=dev)
        self.M = torch.zeros((self.n, nm), dtype=torch.float32, device=dev)
        self.dm_phase = torch.zeros((self.n, L, L), dtype=torch.float32, device=dev)
        side = c0.n_lenses * c0.subap_npx
        self.side = side
        # per-realisation buffers as rows of group stacks, so the SH, CCD and
        # slope computer run as one batched launch each for the group
        self.EA = torch.zeros((self.n, L, L), dtype=torch.float32, device=dev)
        self.EP = torch.zeros((self.n, L, L), dtype=torch.float32, device=dev)
        self.I = torch.zeros((self.n, side, side), dtype=torch.float32, device=dev)
        self.INT = torch.zeros((self.n, side, side), dtype=torch.float32, device=dev)
        self.PIX = torch.zeros((self.n, side, side), dtype=torch.float32, device=dev)
        self.FLUX = torch.zeros((self.n, nsl // 2), dtype=torch.float32, device=dev)
        self.n_atm = len(c0.heights)
        self.ATM = torch.zeros((self.n, self.n_atm, L, L), dtype=torch.float32, device=dev)
        for b, lp in enumerate(self.loops):
            for k, layer in enumerate(lp.atmo.layer_list):
                layer.phaseInNm = self.ATM[b, k]
            lp.slopec.slopes.slopes = self.S[b]
            lp.dm.layer.phaseInNm = self.dm_phase[b]
            ef = lp.prop.outputs['out_on_axis_source_ef']
            ef.A = self.EA[b]
            ef.phaseInNm = self.EP[b]
            lp.sh._out_i.i = self.I[b]
            lp.ccd._integrated_i.i = self.INT[b]
            lp.ccd._pixels.pixels = self.PIX[b]
        self.integ = Integrator(self.loops[0].simul_params, int_gain=[c0.gain] * (nm * self.n), delay=c0.delay,
                                target_device_idx=device_idx)
        self.integ.inputs['delta_comm'].set(BaseValue(value=self.M.view(-1), target_device_idx=device_idx))

    def start(self):
        for b, lp in enumerate(self.loops):
            lp.start()
            lp.slopec._flux = self.FLUX[b]
            lp.slopec.flux_per_subaperture_vector.value = self.FLUX[b]
            lp.step_eager()
        self.integ.setup()
        self.dm = self.loops[0].dm        # its padded IF copy and mask index serve the group
        lp0 = self.loops[0]
        if lp0.sh.geometry.do_interpolation:
            raise NotImplementedError('BatchedScao: SH geometries that resample the field are not batched')
        if any(lp.sh._photon_scale != lp0.sh._photon_scale for lp in self.loops):
            raise ValueError('BatchedScao: the realisations of a group must share the photon flux')
        dev = self.device
        self.pseeds = torch.tensor([lp.ccd._photon_seed for lp in self.loops], dtype=torch.int64, device=dev)
        self.rseeds = torch.tensor([lp.ccd._readout_seed for lp in self.loops], dtype=torch.int64, device=dev)
        lib = _lib.load()
        if self.sh_forward != SH_FORWARD['fp32'] and not lib.sb_sh_split_bf16_supported(ctypes.byref(lp0.sh._plan)):
            g = lp0.sh.geometry
            raise ValueError(f'BatchedScao: no split-BF16 SH kernel for np_sub={g.ovs_np_sub}, cutsize={g.cutsize}, '
                             f'subap_npx={g.subap_npx}')
        self.sh_scratch = torch.empty(self.n * lib.sb_sh_scratch_bytes(ctypes.byref(lp0.sh._plan)),
                                      dtype=torch.uint8, device=dev)
        self.sc_scratch = torch.empty(self.n * lib.sb_slopec_scratch_bytes(ctypes.byref(lp0.slopec._plan)),
                                      dtype=torch.uint8, device=dev)
        # every turbulence layer of every realisation in one atmosphere launch:
        # per layer its strip, output row, position and its realisation's inputs
        nl = self.n_atm
        n_all = self.n * nl
        self.atmo_layers = (_lib.AtmoLayer * n_all)()
        self.atmo_inputs = (_lib.AtmoLayerInputs * n_all)()
        for b, lp in enumerate(self.loops):
            if lp.prop._layers[-1] is not lp.dm.layer or any(
                    ly.phaseInNm.shape != (self.L, self.L) for ly in lp.prop._layers):
                raise NotImplementedError('BatchedScao: pupil-sized layers in the SCAO order are batched only')
            base = lp._inputs.data_ptr()
            for k in range(nl):
                i = b * nl + k
                ctypes.memmove(ctypes.byref(self.atmo_layers[i]), ctypes.byref(lp.atmo._layers[k]),
                               ctypes.sizeof(_lib.AtmoLayer))
                self.atmo_inputs[i].seeing = base
                self.atmo_inputs[i].wind_speed = base + 8 * (1 + k)
                self.atmo_inputs[i].wind_direction = base + 8 * (1 + nl + k)
                self.atmo_inputs[i].position = lp.atmo._positions.data_ptr() + 8 * k
        self.atmo_work = torch.empty(n_all * 128, dtype=torch.uint8, device=dev)
        self.stop = lp0.pupilstop
        self.sync_from_loops()

    def sync_from_loops(self):
        """Group integrator state <- the realisations' own integrators."""
        nm = self.nm
        for b, lp in enumerate(self.loops):
            self.integ.state[b * nm:(b + 1) * nm].copy_(lp.integ.state)
            self.integ._ist[b * nm:(b + 1) * nm].copy_(lp.integ._ist)
            self.integ._ost[b * nm:(b + 1) * nm].copy_(lp.integ._ost)
            self.integ.out_comm.value[b * nm:(b + 1) * nm].copy_(lp.integ.out_comm.value)

    def mc_group(self, pipelined=False):
        """This group as an sb_mc_group: the same buffers, plans and seeds the
        group-by-group launches use (keeps the ctypes arrays it points to).
        pipelined: with a second mirror-phase buffer and the integrators'
        next output, for sb_mc_stage's overlapped mirror."""
        lp = self.loops[0]
        if not lp._can_fuse_chain():
            raise NotImplementedError('BatchedScao: the Monte-Carlo step needs the fused detector / slope chain '
                                      '(plain SH, a detector read every step, slopes with thr_value only)')
        dm = self.dm
        L2, F2 = self.L * self.L, self.side * self.side
        self._lenslet_subap = torch.as_tensor(lp.lenslet_subap_map(), device=self.device)
        m = _lib.McGroup()
        m.n_batch, m.n_atm, m.L = self.n, self.n_atm, self.L
        m.layers = ctypes.cast(self.atmo_layers, ctypes.POINTER(_lib.AtmoLayer))
        m.inputs = ctypes.cast(self.atmo_inputs, ctypes.POINTER(_lib.AtmoLayerInputs))
        m.constants = lp.atmo.inputs_struct(lp.atmo.delta_time)
        m.atm, m.atm_real_stride = self.ATM.data_ptr(), self.n_atm * L2
        m.stop_A, m.stop_phase = self.stop.A.data_ptr(), self.stop.phaseInNm.data_ptr()
        m.dm_A = lp.dm.layer.A.data_ptr()
        m.dm_phase, m.dm_stride = self.dm_phase.data_ptr(), L2
        m.field_A, m.field_phase, m.field_stride = self.EA.data_ptr(), self.EP.data_ptr(), L2
        m.sh = lp.sh._plan
        m.dft_mode = 0 if self.sh_forward == SH_FORWARD['fp32'] else 1
        m.photon_scale = lp.sh._photon_scale
        m.intensity, m.integrated, m.pixels = self.I.data_ptr(), self.INT.data_ptr(), self.PIX.data_ptr()
        m.frame_stride = F2
        m.ccd = lp.ccd._params
        m.photon_seeds, m.readout_seeds = self.pseeds.data_ptr(), self.rseeds.data_ptr()
        m.slopec = lp.slopec._plan
        m.lenslet_subap = self._lenslet_subap.data_ptr()
        m.slopes, m.slopes_stride = self.S.data_ptr(), self.nsl
        m.flux, m.flux_stride = self.FLUX.data_ptr(), self.nsl // 2
        R = lp.rec._R
        m.R, m.n_modes, m.n_slopes, m.ldr = R.data_ptr(), self.nm, self.nsl, R.stride(0)
        m.modes = self.M.data_ptr()
        m.iir = self.integ._plan
        m.commands = self.integ.out_comm.value.data_ptr()
        if pipelined:
            self.dm_phase_alt = torch.zeros_like(self.dm_phase)
            self.commands_next = torch.zeros_like(self.integ.out_comm.value)
            m.dm_phase_alt = self.dm_phase_alt.data_ptr()
            m.commands_next = self.commands_next.data_ptr()
            m.iir.out_next = m.commands_next         # on the group's copy of the plan only
        m.ifunc, m.n_valid, m.ld_if = dm._IF.data_ptr(), int(dm._idx.numel()), dm._ld
        m.mask_idx, m.dm_sign = dm._idx.data_ptr(), float(dm.sign)
        return m

    def group_ops(self):
        """The whole step of every realisation of the group, one launch each:
        atmosphere (every layer), propagation, SH, CCD, slopes, the shared
        reconstructor, the integrators and the shared mirror."""
        st = torch.cuda.current_stream(self.device).cuda_stream
        lp = self.loops[0]
        L2 = self.L * self.L
        consts = lp.atmo.inputs_struct(lp.atmo.delta_time)
        if self.fuse_atmo and self.n_atm > 0:
            # layers and field in one launch (the same bits as the two calls below)
            _lib.call('sb_atmo_propagate_batched', self.atmo_layers, self.atmo_inputs, self.n_atm, self.n, self.L,
                      ctypes.byref(consts), self.atmo_work.data_ptr(), self.atmo_work.numel(),
                      self.stop.A.data_ptr(), self.stop.phaseInNm.data_ptr(), lp.dm.layer.A.data_ptr(),
                      self.dm_phase.data_ptr(), L2, self.EA.data_ptr(), self.EP.data_ptr(), L2, st)
        else:
            _lib.call('sb_atmo_evolve_batched', self.atmo_layers, self.atmo_inputs, self.n * self.n_atm, self.L,
                      ctypes.byref(consts), self.atmo_work.data_ptr(), self.atmo_work.numel(), st)
            _lib.call('sb_propagate_batched', self.ATM.data_ptr(), self.n_atm, L2, self.n_atm * L2,
                      self.stop.A.data_ptr(), self.stop.phaseInNm.data_ptr(), lp.dm.layer.A.data_ptr(),
                      self.dm_phase.data_ptr(), L2, self.n, self.L, self.EA.data_ptr(), self.EP.data_ptr(), L2, st)
        lp = self.loops[0]
        L2, F2 = self.L * self.L, self.side * self.side
        _lib.call(self.sh_forward, ctypes.byref(lp.sh._plan), self.EA.data_ptr(), L2, self.EP.data_ptr(), L2,
                  self.EA.data_ptr(), L2, L2, lp.sh._photon_scale, self.I.data_ptr(), F2, self.n,
                  self.sh_scratch.data_ptr(), self.sh_scratch.numel(), st)
        _lib.call('sb_ccd_step_batched', ctypes.byref(lp.ccd._params), self.pseeds.data_ptr(), self.rseeds.data_ptr(),
                  self.n, self.I.data_ptr(), self.INT.data_ptr(), self.PIX.data_ptr(), st)
        _lib.call('sb_slopec_batched', ctypes.byref(lp.slopec._plan), self.PIX.data_ptr(), F2, self.S.data_ptr(),
                  self.nsl, self.FLUX.data_ptr(), self.nsl // 2, self.n, self.sc_scratch.data_ptr(),
                  self.sc_scratch.numel(), st)
        R = lp.rec._R
        _lib.call('sb_modalrec_batched', R.data_ptr(), self.nm, self.nsl, R.stride(0), self.S.data_ptr(),
                  self.nsl, self.n, self.M.data_ptr(), self.nm, st)
        _lib.call('sb_integrator', ctypes.byref(self.integ._plan), self.M.data_ptr(),
                  self.integ.out_comm.value.data_ptr(), st)
        dm = self.dm
        _lib.call('sb_dm_project_batched', dm._IF.data_ptr(), self.nm, int(dm._idx.numel()), dm._ld,
                  self.integ.out_comm.value.data_ptr(), self.nm, self.n, float(dm.sign), dm._idx.data_ptr(),
                  self.dm_phase.data_ptr(), self.L * self.L, st)


class BatchedScao:
    def __init__(self, groups, device_idx=0, dft='fp32'):
        self.device = torch.device('cuda', device_idx)
        self.dft = dft
        self.groups = [_Group(t, reals, device_idx, dft=dft) for t, reals in groups]
        self.graph = None
        self.plain_graphs = None
        self._launches = None
        self.steps_per_replay = 1

    def set_dft(self, dft):
        """Switch the groups' SH forward between 'fp32' and 'split_bf16'; the
        step graph must be captured again."""
        if dft not in SH_FORWARD:
            raise ValueError(f"dft must be one of {sorted(SH_FORWARD)}, not {dft!r}")
        lib = _lib.load()
        for g in self.groups:
            sh = g.loops[0].sh
            plan = getattr(sh, '_plan', None)      # set up by start(); checked there otherwise
            if dft != 'fp32' and plan is not None and not lib.sb_sh_split_bf16_supported(ctypes.byref(plan)):
                raise ValueError(f'BatchedScao: no split-BF16 SH kernel for cutsize={sh.geometry.cutsize}, '
                                 f'subap_npx={sh.geometry.subap_npx}')
        for g in self.groups:
            g.sh_forward = SH_FORWARD[dft]
        self.dft = dft
        self.graph = None

    def autotune(self, tuner=None):
        """Tune the tile shapes of every group's batched mirror projection and
        reconstructor (and of its SH forward, in the FP32 form) on the group's
        own buffers with a
        specula_b200.autotune.Autotuner; the launches are idempotent, so the
        simulation state is unchanged.  Capture the step graph afterwards.
        Returns the tuner's records."""
        from specula_b200.autotune import Autotuner
        tuner = tuner or Autotuner(self.device)
        torch.cuda.synchronize(self.device)
        for g in self.groups:
            lp = g.loops[0]
            dm = g.dm
            tuner.tune_dm_batched(dm._IF, g.nm, int(dm._idx.numel()), dm._ld, g.integ.out_comm.value, g.nm, g.n,
                                  float(dm.sign), dm._idx, g.dm_phase, g.L * g.L)
            R = lp.rec._R
            tuner.tune_modalrec_batched(R, g.nm, g.nsl, R.stride(0), g.S, g.nsl, g.n, g.M, g.nm)
            if g.sh_forward == SH_FORWARD['fp32']:
                L2, F2 = g.L * g.L, g.side * g.side
                tuner.tune_sh_fp32(lp.sh._plan, g.EA, L2, g.EP, L2, g.EA, L2, L2, lp.sh._photon_scale, g.I, F2, g.n,
                                   g.sh_scratch)
        self.graph = None
        return tuner.results

    @property
    def n_realisations(self):
        return sum(g.n for g in self.groups)

    def start(self):
        for g in self.groups:
            g.start()
        for g in self.groups:
            for lp in g.loops:
                lp.atmo.delta_time = lp.atmo.t_to_seconds(lp.loop.dt)
        torch.cuda.synchronize(self.device)

    def step_eager(self):
        """One batched step without a graph (every group's launches in turn)."""
        for g in self.groups:
            g.group_ops()

    def capture(self):
        """The batched step of every group in one CUDA graph, each group's
        launches on a stream of its own so the groups overlap one another."""
        self.step_eager()
        torch.cuda.synchronize(self.device)
        gstreams = [torch.cuda.Stream(self.device) for _ in self.groups]
        cap = torch.cuda.Stream(self.device)
        g = torch.cuda.CUDAGraph(keep_graph=True)
        with torch.cuda.graph(g, stream=cap):
            main = torch.cuda.current_stream(self.device)
            for grp, gs in zip(self.groups, gstreams):
                gs.wait_stream(main)
                with torch.cuda.stream(gs):
                    grp.group_ops()
            for gs in gstreams:
                main.wait_stream(gs)
        torch.cuda.synchronize(self.device)
        self.graph = g
        self._launches = graph_kernel_count(g)
        self.steps_per_replay = 1
        return g

    def replay(self):
        self.graph.replay()

    @property
    def launches_per_step(self):
        """Kernel launches of one captured step, counted in the graph."""
        return self._launches

    def capture_mc(self, pipelined=False):
        """The batched step of every group as one sb_mc_step (six launches,
        each over every realisation of every group) captured in a CUDA graph.
        pipelined: two steps per replay, each step's mirror projection on a
        second (high-priority) stream overlapping the step's atmosphere, SH
        and detector stages (sb_mc_stage); the same results."""
        lib = _lib.load()
        self.release_mc()
        groups = (_lib.McGroup * len(self.groups))(*[g.mc_group(pipelined) for g in self.groups])
        nbytes = lib.sb_mc_workspace_bytes(groups, len(self.groups))
        if nbytes == 0:
            raise ValueError('BatchedScao: ' + (lib.sb_last_error() or b'').decode())
        self.mc_workspace = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        handle = ctypes.c_void_p()
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.call('sb_mc_create', groups, len(self.groups), self.mc_workspace.data_ptr(), nbytes, ctypes.byref(handle),
                  st)
        self._mc_groups = groups
        self.mc_handle = handle
        # one eager step, as capture() takes; with pipelining it also fills
        # the integrators' next output and the mirror phase of step t = 0
        _lib.call('sb_mc_step', handle, st)
        torch.cuda.synchronize(self.device)
        cap = torch.cuda.Stream(self.device)
        g = torch.cuda.CUDAGraph(keep_graph=True)
        if not pipelined:
            with torch.cuda.graph(g, stream=cap):
                _lib.call('sb_mc_step', handle, torch.cuda.current_stream(self.device).cuda_stream)
            self.steps_per_replay = 1
        else:
            side = torch.cuda.Stream(self.device, priority=-1)

            def stage(k, p, stream):
                _lib.call('sb_mc_stage', handle, k, p, stream.cuda_stream)

            with torch.cuda.graph(g, stream=cap):
                main = torch.cuda.current_stream(self.device)
                for p in (1, 0):
                    side.wait_stream(main)            # the commands of step t: after REC(t-1)
                    stage(_lib.SB_MC_DM, p, side)
                    for k in (_lib.SB_MC_ATMO, _lib.SB_MC_SH, _lib.SB_MC_CHAIN):
                        stage(k, p, main)
                    main.wait_stream(side)            # REC(t) rewrites the next commands
                    stage(_lib.SB_MC_REC, p, main)
            self.steps_per_replay = 2
        torch.cuda.synchronize(self.device)
        self.graph = g
        self._launches = graph_kernel_count(g) // self.steps_per_replay
        return g

    def step_mc(self):
        """One Monte-Carlo step without a graph (after capture_mc)."""
        _lib.call('sb_mc_step', self.mc_handle, torch.cuda.current_stream(self.device).cuda_stream)

    def release_mc(self):
        """Free the Monte-Carlo step's handle (the graph that replays it goes too)."""
        h = getattr(self, 'mc_handle', None)
        if h is not None and h.value:
            if self.graph is not None:
                torch.cuda.synchronize(self.device)
                self.graph = None
            _lib.load().sb_mc_destroy(h)
        self.mc_handle = None

    def __del__(self):
        try:
            self.release_mc()
        except Exception:
            pass

    def capture_plain(self):
        """Every realisation's own sequential step graph (its own
        reconstructor, integrator and mirror: the plain form)."""
        for grp in self.groups:
            for lp in grp.loops:
                lp.capture(pipelined=False)
        torch.cuda.synchronize(self.device)

    def replay_plain(self):
        for grp in self.groups:
            for lp in grp.loops:
                lp.replay()

    def slopes(self):
        return [grp.S.clone() for grp in self.groups]
