"""Benchmark: closed-loop SCAO Shack-Hartmann steps per second on B200.

Workload (one step = one pass of the whole loop over one frame): 39 m pupil
on 640 px, 80x80 sub-apertures of 8x8 phase px, 16x16 FFT (cut 4) onto 6x6
detector px, complex64 field, 7-layer atmosphere (Cn2 0.5/0.15/0.1/0.1/
0.05/0.05/0.05, 0-16 km, winds 5-30 m/s in random directions), r0 0.15 m,
L0 25 m, photon noise (1e3 ph / sub-aperture / frame) and 3 e- read-out,
500-mode DM, modal reconstructor, integrator gain 0.5 with 2-frame delay.
Synthetic seeded inputs (screens from the von Karman synthesis, random
influence functions and reconstructor of the right shapes).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  ``value``: whole-job steps/s of the captured
CUDA-graph step with everything resident in HBM; ``e2e``: steps/s through
the public object API (LoopControl.iter) with the per-step inputs copied
host->device and the slopes + DM commands read back device->host.
``--impl reference`` times the CPU oracle (NumPy restatement of the
reference's CPU path) on the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'SH loop steps/s at 80x80 subaps'
# Stored, not measured by this run: dram__bytes_read.sum (632 241 664) +
# dram__bytes_write.sum (3 805 440) of one dm_project_tma_kernel launch of
# this workload, captured 2026-12-04 with
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none \
#       --profile-from-start off -k regex:dm_project_tma -c 1 python bench.py --profile-loop 1
# (one pass; the step graph's mirror launch)
DM_TRAFFIC_BYTES = 636_047_104
UNIT = 'steps/s'
WORKLOAD = 'elt_80x80_fft16_7layers_500modes'


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=4000)
    p.add_argument('--warmup', type=int, default=10)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--cpu-baseline-seconds', type=float, default=20.0)
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-adjoint', action='store_true', help='skip the adjoint interaction-matrix leg')
    p.add_argument('--no-gradient', action='store_true',
                   help='skip the checkpointed loop-gradient leg (1000 ELT steps, finite-difference check)')
    p.add_argument('--gradient-only', action='store_true', help='run only the loop-gradient leg (one GPU)')
    p.add_argument('--no-batched', action='store_true', help='skip the batched Monte-Carlo leg')
    p.add_argument('--profile-batched', action='store_true',
                   help='set up the batched Monte-Carlo graph (split-BF16 SH, autotuned), then run one replay '
                        'between cudaProfilerStart/Stop (for ncu --profile-from-start off) and exit')
    p.add_argument('--profile-loop', type=int, default=0, metavar='R',
                   help='set up the ELT step graph, then run R replays between cudaProfilerStart/Stop '
                        '(for ncu --profile-from-start off) and exit')
    p.add_argument('--profile-mc', action='store_true',
                   help='as --profile-batched, for the Monte-Carlo step (sb_mc_step) instead of the group graph')
    p.add_argument('--batched-only', action='store_true',
                   help='run only the 96-realisation batched Monte-Carlo leg (one GPU)')
    p.add_argument('--psf-only', action='store_true', help='run only the PSF leg (one GPU)')
    p.add_argument('--adjoint-only', action='store_true',
                   help='run only the adjoint interaction-matrix leg (one GPU) and print its JSON object')
    return p.parse_args()


def config_dict(cfg, n_gpus):
    return {'workload': WORKLOAD, 'pupil_px': cfg.pixel_pupil, 'diameter_m': cfg.diameter_m,
            'subaps': f'{cfg.n_lenses}x{cfg.n_lenses}', 'phase_px_per_subap': cfg.pixel_pupil // cfg.n_lenses,
            'fft': 16, 'detector_px_per_subap': cfg.subap_npx, 'layers': len(cfg.heights), 'modes': cfg.n_modes,
            'parallelism': f'replicas{n_gpus}',
            'l2': 'inputs larger than L2 (influence functions 631 MB streamed every step)'}


class ClockSampler:
    """SM clock and clock-event reasons of one GPU, polled every millisecond
    by a background thread through NVML (read-only queries) while the timed
    region runs; nvidia-smi at 50 ms when NVML cannot be loaded.  The timed
    region of a short run lasts a few milliseconds, so the 1 ms poll is what
    gives it samples of its own."""
    REASONS = (('hw_slowdown', 'nvmlClocksEventReasonHwSlowdown'),
               ('hw_thermal_slowdown', 'nvmlClocksEventReasonHwThermalSlowdown'),
               ('sw_thermal_slowdown', 'nvmlClocksEventReasonSwThermalSlowdown'),
               ('sw_power_cap', 'nvmlClocksEventReasonSwPowerCap'))
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = int(gpu_index)
        self.proc = None
        self.nvml = None
        self.lines = []
        self.sm = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(getattr(torch.cuda.get_device_properties(self.gpu), 'uuid', '') or '')
        if uuid:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith('GPU-') else 'GPU-' + uuid)
            except Exception:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
        except Exception:
            self.nvml = None
        if self.nvml is not None:
            nv, h = self.nvml
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _poll(self):
        nv, h = self.nvml
        masks = [(name, getattr(nv, attr, 0)) for name, attr in self.REASONS]
        while not self._stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, m in masks:
                    if m and r & m:
                        self.reasons.add(name)
            except Exception:
                break
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            if not self.sm:
                return None
            return {'sm_mhz': statistics.median(self.sm), 'sm_max_mhz': self.max_mhz,
                    'reasons': sorted(self.reasons), 'samples': len(self.sm), 'source': 'nvml, 1 ms poll'}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = [n for n, _ in self.REASONS]
        for l in self.lines:
            f = [x.strip() for x in l.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() in ('active', '1', 'yes'):
                    reasons.add(n)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': mx, 'reasons': sorted(reasons), 'samples': len(sm),
                'source': 'nvidia-smi, 50 ms'}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            return float(json.load(f)['hbm_gbs']), 'measured'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback'


def cpu_oracle_loop(cfg, loop=None):
    """Oracle chain on the bench workload; uses the GPU loop's IF / R / tables
    when given so both arms run the same system."""
    from oracle.loop import OracleScaoLoop
    from specula_b200.scao import ScaoLoop, valid_subaps
    from specula_b200.lib.make_mask import make_mask
    import math
    pupil = make_mask(cfg.pixel_pupil, cfg.obsratio, 1.0)
    idxs, _ = valid_subaps(pupil, cfg.n_lenses, cfg.subap_npx)
    nv = int(pupil.sum())
    rng = np.random.default_rng(cfg.seed)
    if loop is not None:
        ifunc = loop.dm._ifunc.influence_function.cpu().numpy()
        recmat = loop.rec.recmat.recmat.cpu().numpy()
        S0 = loop.prop.outputs['out_on_axis_source_ef'].S0
    else:
        ifunc = rng.standard_normal((cfg.n_modes, nv), dtype=np.float32) * 10.0
        recmat = rng.standard_normal((cfg.n_modes, 2 * len(idxs)), dtype=np.float32) / math.sqrt(2 * len(idxs))
        n_valid_est = max(1, int(round(pupil.sum() / (cfg.pixel_pupil / cfg.n_lenses) ** 2)))
        S0 = cfg.photons_per_subap * n_valid_est / (pupil.sum() * cfg.pitch ** 2 * cfg.time_step)
    return OracleScaoLoop(cfg, ifunc, recmat, idxs, pupil, S0)


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get('num_threads', 1) for i in threadpool_info() if i.get('user_api') == 'blas']
        return max(n) if n else 1
    except Exception:
        return os.cpu_count() or 1


def time_cpu_oracle(cfg, budget_s, max_steps, loop=None):
    """Steps/s of the CPU oracle: one untimed step, then steps until the
    budget is spent (at most max_steps)."""
    ol = cpu_oracle_loop(cfg, loop)
    ol.step()
    n = 0
    t0 = time.perf_counter()
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        ol.step()
        n += 1
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args):
    from specula_b200.scao import elt_config
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    cfg = elt_config()
    steps = max(1, min(args.steps, 50))
    value, n, dt = time_cpu_oracle(cfg, budget_s=120.0, max_steps=steps)
    cores = blas_threads()
    sample = f'{n} oracle loop steps of the workload after 1 untimed step ({dt:.1f} s)'
    line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'impl': 'reference', 'n_gpus': args.gpus,
            'steps': n, 'warmup': 1, 'ms_per_step': 1e3 / value, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic', 'config': config_dict(cfg, 1),
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': cores, 'kind': 'port', 'sample': sample},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def bench_adjoint_im(dev, reps, cpu_budget_s):
    """Adjoint interaction matrix against push-pull on the 40x40 / 320 px /
    FFT 16 calibration system with 500 KL modes (one B200).  Each timed call is
    bracketed by CUDA events on the launching stream with an L2 flush
    (256 MB written, then 256 MB read) between calls."""
    import torch
    from specula_b200.calibration import ShCalibrationSystem
    t0 = time.perf_counter()
    cal = ShCalibrationSystem(modes='kl', device_idx=dev.index)
    torch.cuda.synchronize(dev)
    setup_s = time.perf_counter() - t0
    st = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    clean = torch.ones(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    amp = 10.0

    def timed(fn, n):
        ms = []
        out = None
        for _ in range(n):
            # evict L2 by writing 256 MB, then read another 256 MB so the
            # dirty lines are written back before the timed call
            flush.fill_(1.0)
            clean.sum()
            # keep the device busy (~0.5 ms) while the host prepares the timed
            # call, so the start event does not count host-side launch work
            torch.cuda._sleep(1_000_000)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            out = fn()
            e1.record(st)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        return statistics.median(ms), out

    for _ in range(3):
        cal.adjoint_intmat()
        cal.pushpull_intmat(amp)
    torch.cuda.synchronize(dev)
    adj_ms, im_a = timed(cal.adjoint_intmat, reps)
    pp_ms, im_p = timed(lambda: cal.pushpull_intmat(amp), max(2, reps // 2))
    adj = cal.adjoint
    active = adj.active(cal.A, cal._flat)
    jac_ms, jac = timed(lambda: adj.jacobian(cal.A, cal._flat, active), reps)
    con_ms, _ = timed(lambda: adj.intmat(cal.A, cal._flat, cal.dm, jac=jac, pix2col=cal._pix2col), reps)
    # set-up of the contraction's lenslet-major copy of the influence functions
    # (once per mirror and column map; cached by the adjoint)
    def relayout():
        adj._ifl_cache = None
        return adj.lenslet_ifunc(cal.dm._IF, cal.dm._ld, cal._pix2col)
    layout_ms, _ = timed(relayout, 3)
    n_in = cal.pixels_under_valid_subaps()
    con_bytes = cal.contract_bytes(cal.n_modes, n_in, cal.n_valid, adj.np_sub ** 2)
    peak, peak_kind = measured_peak_hbm()
    con_gbs = con_bytes / (con_ms / 1e3) / 1e9
    err = float((im_a - im_p).abs().max() / im_p.abs().max())
    out = {'workload': 'calib_40x40_320px_fft16_500kl', 'n_modes': cal.n_modes, 'n_slopes': 2 * cal.n_valid,
           'modes': 'KL (von Karman r0 0.15 m, L0 25 m) of 547 zonal thin-plate-spline functions, unit RMS',
           'setup_s': setup_s,
           'adjoint_ms': adj_ms, 'pushpull_ms': pp_ms, 'speedup_vs_gpu_pushpull': pp_ms / adj_ms,
           'pushpull_amplitude': amp, 'pushpull_steps': 2 * cal.n_modes,
           'pushpull_form': 'same CUDA chain, one influence function projected per step, whole sequence in one '
                            'CUDA graph',
           'rel_diff_vs_gpu_pushpull': err,
           'jacobian_kernel_us': jac_ms * 1e3, 'contract_kernel_us': con_ms * 1e3,
           'contract_form': adj.contraction, 'contract_layout_us': layout_ms * 1e3,
           'contract_roofline': {'bound': 'hbm', 'achieved': con_gbs, 'peak': peak, 'peak_kind': peak_kind,
                                 'unit': 'GB/s', 'frac': con_gbs / peak, 'algorithmic_bytes': con_bytes},
           'l2': 'flushed before every timed call (256 MB written, then 256 MB read)'}
    if cpu_budget_s > 0:
        out['cpu_baseline'] = cpu_pushpull(cal, amp, cpu_budget_s)
    return out


def cpu_pushpull(cal, amp, budget_s):
    """The reference's push-pull on the host cores (CPU oracle, float32):
    as many modes as fit in the budget, scaled to all modes."""
    from oracle import sh as osh, slopec as osl, control as octl
    g = cal.sh.geometry
    geom = osh.sh_geometry(cal.sh._wavelengthInNm, cal.sh._subap_wanted_fov_arcsec, cal.sh._sensor_pxscale_arcsec,
                           g.n_lenses, g.subap_npx, cal.pupil.shape[0], cal.simul_params.pixel_pitch,
                           fov_ovs_coeff=1.0)
    o = osh.SHOracle(geom, cal.sh._wavelengthInNm, precision=1)
    A = cal.pupil.astype(np.float32)
    IF = cal.dm._ifunc.influence_function.cpu().numpy()
    idxs = cal.subapdata.idxs
    pitch = cal.simul_params.pixel_pitch

    def slopes_fn(k, a):
        cmd = np.zeros(IF.shape[0], np.float32)
        cmd[k] = a
        ph = octl.dm_phase(IF, cal.pupil, cmd, sign=cal.dm.sign)
        return osl.sh_slopes(o.forward(A, ph, 1.0, pitch), idxs)[0]

    slopes_fn(0, amp)                     # untimed: first call
    t0 = time.perf_counter()
    k = 0
    while k < IF.shape[0] and time.perf_counter() - t0 < budget_s:
        octl.pushpull_intmat(lambda _, a: slopes_fn(k, a), 1, [amp])
        k += 1
    dt = time.perf_counter() - t0
    return {'value': dt / k * IF.shape[0], 'unit': 's per interaction matrix', 'cores': blas_threads(),
            'kind': 'port', 'sample': f'{k} of {IF.shape[0]} modes pushed and pulled in {dt:.1f} s, scaled'}


def bench_loop_gradient(dev, n_steps=1000, checkpoint_every=50, n_dirs=8, fd_eps=2e-2):
    """Gradient of the mean residual wavefront variance of the ELT loop
    (noise-free detector, every one of the 80x80 sub-apertures valid, 500
    Zernike modes, reconstructor = pseudo-inverse of the adjoint interaction
    matrix calibrated with DM sign +1, gains 0.5) with respect to the 500 integrator gains and the
    reconstructor, checkpoints every 50 steps, against central finite
    differences on seeded random gain directions."""
    import torch
    from specula_b200.data_objects.intmat import Intmat
    from specula_b200.lib.loop_gradient import LoopGradient
    from specula_b200.lib.sh_adjoint import ShSlopesAdjoint
    from specula_b200.lib.zernike import compute_zern_ifunc
    from specula_b200.scao import ScaoLoop, elt_config
    cfg = elt_config()
    cfg.photon_noise = False
    cfg.readout_noise = 0.0
    cfg.subap_threshold = -1.0
    t0 = time.perf_counter()
    from specula_b200.lib.make_mask import make_mask
    pupil = make_mask(cfg.pixel_pupil, cfg.obsratio, 1.0)
    ifunc, _ = compute_zern_ifunc(cfg.pixel_pupil, cfg.n_modes, mask=pupil)
    loop = ScaoLoop(cfg, device_idx=dev.index, ifunc=torch.as_tensor(ifunc, device=dev))
    lg = LoopGradient(loop, n_steps, checkpoint_every=checkpoint_every)
    adj = ShSlopesAdjoint(loop.sh, loop.slopec)
    flat = torch.zeros_like(loop.dm.layer.phaseInNm)
    # calibrated with the DM sign flipped (+1), as the reference's calibration
    # configuration does, so the loop (DM sign -1) has negative feedback
    im = adj.intmat(lg.ef.A, flat, loop.dm) * (-1.0)
    R = Intmat(im, target_device_idx=dev.index).pseudo_invert(im).t().contiguous().float()
    setup_s = time.perf_counter() - t0
    g = torch.full((lg.nm,), 0.5, dtype=torch.float32, device=dev)
    lg.gradient(g, R)                      # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    L, dg, dR = lg.gradient(g, R)
    torch.cuda.synchronize(dev)
    grad_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    L_fwd = lg.loss(g, R)
    fwd_s = time.perf_counter() - t0
    gen = torch.Generator(device=dev).manual_seed(7)
    rel = []
    t0 = time.perf_counter()
    for _ in range(n_dirs):
        d = torch.randn(lg.nm, device=dev, generator=gen)
        d /= d.norm()
        fd = (lg.loss(g + fd_eps * d, R) - lg.loss(g - fd_eps * d, R)) / (2 * fd_eps)
        ad = float((dg.double() * d.double()).sum())
        rel.append(abs(ad - fd) / max(abs(fd), 1e-300))
    fd_s = time.perf_counter() - t0
    return {'workload': 'elt_80x80_all_subaps_7layers_500zernike_1000steps', 'steps': n_steps,
            'checkpoint_every': checkpoint_every, 'n_slopes': lg.nsl, 'loss_nm2': L, 'loss_forward_only_nm2': L_fwd,
            'gradient_s': grad_s, 'forward_s': fwd_s, 'gradient_over_forward': grad_s / fwd_s,
            'fd_directions': n_dirs, 'fd_eps': fd_eps, 'fd_seconds': fd_s,
            'fd_rel_err_max': max(rel), 'fd_rel_err': rel, 'setup_s': setup_s,
            'dR_shape': list(dR.shape), 'reconstructor': 'pinv of the adjoint interaction matrix'}


def bench_batched(dev, steps, cpu_budget_s):
    """The 96-realisation Monte-Carlo mix (55 x 20x20 / 160 px, 27 x 40x40 /
    320 px, 14 x 74x74 / 592 px, two wavelengths, r0 ~ U(0.08, 0.20) m):
    realisation-steps/s of the batched graph against the plain form (every
    realisation its own step graph, reconstructor and mirror), CUDA events
    around `steps` steps of each after warm-up."""
    import torch
    from specula_b200 import replicas
    from specula_b200.batched import BatchedScao, mc_groups
    t0 = time.perf_counter()
    all_groups = mc_groups()
    rank, ws = replicas.world()
    # N > 1: every rank steps its share of every geometry group (no data-path collective)
    groups = replicas.shard_groups(all_groups, ws, rank)
    sys_b = BatchedScao(groups, device_idx=dev.index)
    sys_b.start()
    sys_b.capture_plain()
    sys_b.capture()
    setup_s = time.perf_counter() - t0
    n_local = sys_b.n_realisations
    n_real = int(replicas.sum_over_ranks(n_local, device=dev))
    st = torch.cuda.current_stream(dev)

    def timed(fn, n):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return replicas.max_over_ranks(e0.elapsed_time(e1) / n, device=dev)

    plain_ms = timed(sys_b.replay_plain, steps)
    untuned_ms = timed(sys_b.replay, steps)
    # tile shapes from the autotuner (timed on each group's own buffers), graph captured again
    from specula_b200.autotune import Autotuner
    tuner = Autotuner(dev)
    t_tune = time.perf_counter()
    sys_b.autotune(tuner)
    sys_b.capture()
    batched_ms = timed(sys_b.replay, steps)
    # the same batched graph with the split-BF16 tensor-core SH
    sys_b.set_dft('split_bf16')
    sys_b.autotune(tuner)
    sys_b.capture()
    tune_s = time.perf_counter() - t_tune
    bf16_ms = timed(sys_b.replay, steps)
    group_launches = sys_b.launches_per_step
    # the Monte-Carlo step of the C ABI: one launch per stage over every group
    mc = {}
    for dft, pipe in (('fp32', False), ('split_bf16', False), ('split_bf16', True)):
        sys_b.set_dft(dft)
        sys_b.capture_mc(pipelined=pipe)
        spr = sys_b.steps_per_replay
        mc[(dft, pipe)] = (timed(sys_b.replay, max(1, steps // spr)) / spr, sys_b.launches_per_step)
    sys_b.release_mc()
    _lib_status()
    by_size = {}
    for (tmpl, reals) in all_groups:
        key = f'{tmpl.n_lenses}x{tmpl.n_lenses}/{tmpl.pixel_pupil}px'
        by_size[key] = by_size.get(key, 0) + len(reals)
    out = {'workload': 'mc96_20x20_40x40_74x74_2wavelengths', 'realisations': n_real, 'split': by_size,
           'groups': len(all_groups), 'steps_timed': steps, 'n_gpus': ws,
           'scaling': 'strong (the 96 realisations split across the GPUs)',
           'batched_ms_per_step': batched_ms, 'batched_untuned_ms_per_step': untuned_ms,
           'plain_ms_per_step': plain_ms,
           'batched_realisation_steps_per_s': n_real / (batched_ms / 1e3),
           'plain_realisation_steps_per_s': n_real / (plain_ms / 1e3),
           'speedup_batched_vs_plain': plain_ms / batched_ms,
           'batched_split_bf16_ms_per_step': bf16_ms,
           'batched_split_bf16_realisation_steps_per_s': n_real / (bf16_ms / 1e3),
           'speedup_batched_split_bf16_vs_plain': plain_ms / bf16_ms, 'setup_s': setup_s,
           'group_graph_launches_per_step': group_launches,
           'mc_step_ms_per_step': mc[('fp32', False)][0],
           'mc_step_split_bf16_ms_per_step': mc[('split_bf16', False)][0],
           'mc_step_pipelined_split_bf16_ms_per_step': mc[('split_bf16', True)][0],
           'mc_step_launches_per_step': mc[('split_bf16', True)][1],
           'mc_step_realisation_steps_per_s': n_real / (min(v[0] for v in mc.values()) / 1e3),
           'mc_step': 'sb_mc_step: six launches per step (layer parameters, layers + on-axis field, SH, '
                      'normalisation + detector + slopes, reconstructor + integrators, mirror), each over every '
                      'realisation of every group, captured in one graph; pipelined: the mirror of each step on a '
                      'second stream beside its other stages',
           'autotune_s': tune_s,
           'autotune': [{k: r[k] for k in ('family', 'shape', 'variant', 'name', 'times_us', 'speedup_vs_variant0',
                                           'cached')} for r in tuner.results],
           'graph': 'one CUDA graph per step for all 96 realisations: each geometry group on a stream of its own, '
                    'one batched launch per stage (atmosphere, propagation, SH, CCD, slopes, reconstructor, '
                    'integrator, mirror)'}
    if cpu_budget_s > 0 and ws == 1:
        # the reference has no batched mode: the sum of per-realisation CPU runs,
        # sampled per geometry (steps/s of each size, weighted by its count)
        per = {}
        total_s = 0.0
        for tmpl, reals in all_groups:
            key = f'{tmpl.n_lenses}x{tmpl.n_lenses}'
            if key not in per:
                v, n, dt = time_cpu_oracle(reals[0], budget_s=cpu_budget_s / 3, max_steps=50)
                per[key] = v
            total_s += len(reals) / per[key]
        out['cpu_baseline'] = {'value': n_real / total_s, 'unit': 'realisation-steps/s', 'cores': blas_threads(),
                               'kind': 'port', 'sample': 'CPU-oracle steps of one realisation per geometry, '
                               'weighted by the realisation counts: ' + json.dumps({k: round(v, 3) for k, v in per.items()})}
    return out


def bench_sh_forms(dev, reps=200):
    """Device time of one SH forward (FP32 CUDA-core DFTs against split-BF16
    tensor-core DFTs) on the 80x80 ELT field (FFT 16 and FFT 32) and on a
    batch of 7 fields of 74x74 sub-apertures, CUDA events over `reps`
    launches after warm-up."""
    import ctypes
    import torch
    from specula_b200 import _lib
    from specula_b200.scao import ScaoLoop, elt_config
    from specula_b200.batched import mc_groups
    out = {}
    cfgs = [('elt_80x80_640px', elt_config(), 1),
            # the 4x-padded ELT variant: FFT 32, 0.5 lambda/d pixels (the mirror size does not enter the SH)
            ('elt_80x80_640px_fft32', elt_config(n_modes=10, fft_pad=4), 1),
            ('mc_74x74_592px_x7', mc_groups()[-1][0], 7)]
    for name, cfg, nb in cfgs:
        loop = ScaoLoop(cfg, device_idx=dev.index)
        loop.start()
        loop.step_eager()
        sh = loop.sh
        ef = sh._in_ef
        L2 = ef.A.numel()
        side = cfg.n_lenses * cfg.subap_npx
        A = ef.A.reshape(1, -1).repeat(nb, 1).contiguous()
        P = ef.phaseInNm.reshape(1, -1).repeat(nb, 1).contiguous()
        I = torch.empty((nb, side * side), device=dev)
        scratch = torch.zeros(nb * _lib.load().sb_sh_scratch_bytes(ctypes.byref(sh._plan)), dtype=torch.uint8,
                              device=dev)
        st = torch.cuda.current_stream(dev)
        res = {}
        for form, fn in (('fp32', 'sb_sh_forward_batched'), ('split_bf16', 'sb_sh_forward_split_bf16_batched')):
            def call():
                _lib.call(fn, ctypes.byref(sh._plan), A.data_ptr(), L2, P.data_ptr(), L2, A.data_ptr(), L2, L2,
                          sh._photon_scale, I.data_ptr(), side * side, nb, scratch.data_ptr(), scratch.numel(),
                          st.cuda_stream)
            for _ in range(5):
                call()
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(reps):
                call()
            e1.record(st)
            torch.cuda.synchronize(dev)
            res[form + '_us'] = e0.elapsed_time(e1) / reps * 1e3
        res['speedup_split_bf16_vs_fp32'] = res['fp32_us'] / res['split_bf16_us']
        res['fields'] = nb
        res['sub_apertures_per_field'] = cfg.n_lenses ** 2
        res['fft'] = int(sh.geometry.fft_size)
        res['cutsize'] = int(sh._plan.cutsize)
        if name == 'elt_80x80_640px':
            res['lgs_us'] = _time_lgs(dev, cfg, loop, reps)
        out[name] = res
        del loop
    _lib_status()
    return out


def _time_lgs(dev, cfg, loop, reps):
    """Device time of the laser-guide-star SH (sb_sh_forward_lgs, Gaussian 1 arcsec spot) on the loop's field."""
    import ctypes
    import torch
    from specula_b200 import _lib
    from specula_b200.processing_objects.sh import SH
    from specula_b200.data_objects.laser_launch_telescope import LaserLaunchTelescope
    s0 = loop.sh
    ef = s0._in_ef
    sh = SH(wavelengthInNm=s0._wavelengthInNm, subap_wanted_fov=s0._subap_wanted_fov_arcsec,
            sensor_pxscale=s0._sensor_pxscale_arcsec, subap_on_diameter=cfg.n_lenses, subap_npx=cfg.subap_npx,
            fov_ovs_coeff=cfg.fov_ovs_coeff, laser_launch_tel=LaserLaunchTelescope(spot_size=1.0),
            target_device_idx=dev.index)
    sh.inputs['in_ef'].set(ef)
    sh.setup()
    st = torch.cuda.current_stream(dev)

    def call():
        _lib.call('sb_sh_forward_lgs', ctypes.byref(sh._plan), ctypes.byref(sh._lgs), ef.A.data_ptr(),
                  ef.phaseInNm.data_ptr(), ef.A.data_ptr(), ef.A.numel(), sh._photon_scale,
                  sh._out_i.i.data_ptr(), sh._scratch.data_ptr(), sh._scratch.numel(), st.cuda_stream)
    for _ in range(5):
        call()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        call()
    e1.record(st)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / reps * 1e3


def accuracy_vs_fp64(loop, A, phase):
    """Error of the headline step's float32 kernels against float64 on one
    noise-free frame: the loop's SH (sb_sh_forward) on the turbulent field
    (A, phase) against the float64 oracle SH, and the loop's slope computer
    (sb_slopec) on that frame against float64 CoG slopes of the float64
    frame; max |d| / max |ref| over the frame and over the slopes."""
    import torch
    from oracle import sh as osh, slopec as osl
    cfg = loop.cfg
    ef = loop.sh._in_ef
    ef.A.copy_(A)
    ef.phaseInNm.copy_(phase)
    loop.sh.trigger_code()
    pix = loop.ccd.outputs['out_pixels'].pixels
    pix.copy_(loop.sh.outputs['out_i'].i)
    loop.slopec.trigger_code()
    torch.cuda.synchronize(loop.device)
    got_i = loop.sh.outputs['out_i'].i.cpu().numpy().astype(np.float64)
    got_s = loop.slopec.slopes.slopes.cpu().numpy().astype(np.float64)
    s = loop.sh
    g = osh.sh_geometry(s._wavelengthInNm, s._subap_wanted_fov_arcsec, s._sensor_pxscale_arcsec, cfg.n_lenses,
                        cfg.subap_npx, cfg.pixel_pupil, cfg.pitch, fov_ovs_coeff=cfg.fov_ovs_coeff)
    ref_i = osh.SHOracle(g, s._wavelengthInNm, precision=0).forward(
        A.cpu().numpy().astype(np.float64), phase.cpu().numpy().astype(np.float64), ef.S0, cfg.pitch)
    ref_s, _ = osl.sh_slopes(ref_i, loop.subapdata.idxs, precision=0)

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
    return {'intensity_rel_err_vs_fp64': rel(got_i, ref_i), 'slopes_rel_err_vs_fp64': rel(got_s, ref_s),
            'frame': 'the first step of the bench loop (7 turbulent layers, flat mirror), noise-free',
            'metric': 'max |float32 - float64| / max |float64|',
            'targets': {'intensity': 1e-5, 'slopes': 1e-4}}


def bench_psf(dev, reps=20):
    """The PSF object's image on the ELT field (640 px, nd 8: 5120 x 5120)
    through sb_psf_tc (split-BF16 tcgen05 GEMMs), CUDA events over `reps`
    calls after warm-up, beside the same two complex products as complex64
    GEMMs through the library (torch.matmul) for reference."""
    import torch
    from specula_b200.processing_objects.psf import PSF
    from specula_b200.data_objects.electric_field import ElectricField
    from specula_b200.lib.make_mask import make_mask
    pix, nd, lam = 640, 8, 1650.0
    A = torch.as_tensor(make_mask(pix, 0.14, 1.0).astype(np.float32), device=dev)
    ef = ElectricField(pix, pix, 39.0 / pix, S0=1.0, target_device_idx=dev.index)
    ef.A.copy_(A)
    g = torch.Generator(device=dev).manual_seed(5)
    ef.phaseInNm.copy_(torch.randn((pix, pix), device=dev, generator=g) * 120.0 * A)
    p = PSF(wavelengthInNm=lam, nd=nd, target_device_idx=dev.index)
    p.inputs['in_ef'].set(ef)
    p.setup()
    n = p._n
    st = torch.cuda.current_stream(dev)

    def timeit(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    tc_ms = timeit(p.trigger_code)
    _lib_status()
    # the library form of the same two products (complex64), for comparison
    k = (np.arange(n) - n // 2) % n
    W = torch.polar(torch.ones((n, pix), dtype=torch.float64),
                    torch.as_tensor((-2.0 * np.pi / n) * (np.outer(k, np.arange(pix)) % n))).to(torch.complex64).to(dev)
    WT = W.t().contiguous()
    u = torch.polar(A, ef.phaseInNm * p._k).to(torch.complex64)
    G = torch.empty((pix, n), dtype=torch.complex64, device=dev)
    F = torch.empty((n, n), dtype=torch.complex64, device=dev)

    def lib_products():
        torch.matmul(u, WT, out=G)
        torch.matmul(W, G, out=F)
    lib_ms = timeit(lib_products)
    mp, np_ = (pix + 127) // 128 * 128, (n + 127) // 128 * 128
    bf16_flop = 3 * 2 * (np_ * (2 * mp) * (2 * mp) + np_ * (2 * np_) * (2 * mp))
    return {'workload': 'psf_640px_nd8_5120x5120', 'psf_ms': tc_ms, 'library_complex64_products_ms': lib_ms,
            'speedup_vs_library_products': lib_ms / tc_ms,
            'split_bf16_tflops': bf16_flop / (tc_ms / 1e3) / 1e12,
            'form': 'Strehl reduction + field + two tcgen05 split-BF16 GEMMs (3 launches); the library figure is '
                    'the two complex64 products alone'}


def _lib_status():
    from specula_b200 import _lib
    _lib.call('sb_device_status')


def run_b200(args):
    import torch
    import torch.distributed as dist
    from specula_b200.scao import ScaoLoop, elt_config
    from specula_b200 import _lib
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120), device_id=dev)

    cfg = elt_config()
    loop = ScaoLoop(cfg, device_idx=local)
    loop.start()
    loop.step_eager()                     # t = 0 (no screen motion yet)
    # the turbulent field of that step (the mirror is still flat), kept for the accuracy check
    ef0 = loop.sh._in_ef
    acc_field = (ef0.A.clone(), ef0.phaseInNm.clone())
    loop.capture()
    for _ in range(max(3, args.warmup)):
        loop.replay()
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    st = torch.cuda.current_stream(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    spr = loop.steps_per_replay
    n_rep = max(1, args.steps // spr)
    steps = n_rep * spr
    e0.record(st)
    for _ in range(n_rep):
        loop.replay()
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    _lib.call('sb_device_status')         # raises if a bounded in-kernel wait gave up
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * steps / (ms_max / 1e3)

    # dominant kernel: DM influence-function projection, timed alone on the
    # launching stream (IF = 631 MB > L2, so no launch reuses cached lines)
    dm = loop.dm
    n_rep = max(20, min(args.steps, 200))
    dm.trigger_code()
    torch.cuda.synchronize(dev)
    d0 = torch.cuda.Event(enable_timing=True)
    d1 = torch.cuda.Event(enable_timing=True)
    d0.record(st)
    for _ in range(n_rep):
        dm.trigger_code()
    d1.record(st)
    torch.cuda.synchronize(dev)
    dm_ms = d0.elapsed_time(d1) / n_rep
    nm, nv = dm._IF.shape[0], loop.n_valid_pixels
    dm_bytes = nm * nv * 4 + nm * 4 + nv * 4 + nv * 4   # IF + commands + index table + phase writes
    peak, peak_kind = measured_peak_hbm()
    achieved = dm_bytes / (dm_ms / 1e3) / 1e9

    # algorithmic bytes of one whole step (screens, pupil, IF, R, DM phase,
    # detector frame, slopes, modes): the step's own roofline position
    L = cfg.pixel_pupil
    nsl = 2 * loop.n_valid_subaps
    step_bytes = (len(cfg.heights) * L * (L + 1) * 4 + L * L * 4 + nm * nv * 4 + nm * nsl * 4 + L * L * 4 +
                  (cfg.n_lenses * cfg.subap_npx) ** 2 * 4 + nsl * 4 + nm * 4)

    # end to end through the public loop API with host buffers: the captured
    # two-step graph (ScaoLoop.capture(io=True) / replay), each step's seeing
    # and wind values copied host->device from pinned memory before the
    # replay and each step's slopes + DM commands read back device->host
    # after it.  Two forms: the host waits for each replay's results before
    # launching the next (synchronous), or reads them one replay behind into
    # two alternating pinned buffers, so the device never waits for the host
    # (overlapped; the reported e2e)
    nl = len(cfg.heights)
    loop.capture(io=True, io_slots=2)
    h_in = torch.empty(tuple(loop.io_inputs.shape), dtype=torch.float64).pin_memory()
    h_in.copy_(loop.io_inputs.cpu())
    h_out = [torch.empty(tuple(loop.io_outputs.shape), dtype=torch.float32).pin_memory() for _ in range(2)]
    e2e_reps = max(10, min(args.steps, 2000)) // loop.steps_per_replay
    cur = torch.cuda.current_stream(dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    done = [torch.cuda.Event(), torch.cuda.Event()]
    ran = [torch.cuda.Event(), torch.cuda.Event()]
    fed = [torch.cuda.Event(), torch.cuda.Event()]

    def e2e_round(k, overlapped):
        if not overlapped:
            loop.io_inputs.copy_(h_in, non_blocking=True)
            loop.replay()
            h_out[0].copy_(loop.io_outputs, non_blocking=True)
            done[0].record(cur)
            done[0].synchronize()
            return
        # slot k % 2: its inputs go in on one copy stream once the replay that
        # last read them (k - 2) is done, its results come out on another
        # while the next replay runs; the host takes replay k-1's results
        j = k % 2
        if k >= 2:
            s_in.wait_event(ran[j])
        with torch.cuda.stream(s_in):
            loop.io_inputs_slots[j].copy_(h_in, non_blocking=True)
            fed[j].record(s_in)
        cur.wait_event(fed[j])
        loop.replay(j)
        ran[j].record(cur)
        s_out.wait_event(ran[j])
        with torch.cuda.stream(s_out):
            h_out[j].copy_(loop.io_outputs_slots[j], non_blocking=True)
            done[j].record(s_out)
        if k >= 1:
            done[1 - j].synchronize()           # the previous replay's results are on the host

    def e2e_run(overlapped):
        for k in range(3):
            e2e_round(k, overlapped)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for k in range(e2e_reps):
            e2e_round(k, overlapped)
        done[(e2e_reps - 1) % 2 if overlapped else 0].synchronize()
        dt = time.perf_counter() - t0
        t = torch.tensor([dt], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return world * e2e_reps * loop.steps_per_replay / float(t.item())

    e2e_sync_value = e2e_run(False)
    e2e_value = e2e_run(True)
    e2e_steps = e2e_reps * loop.steps_per_replay

    # the same through the object API (LoopControl.iter: every object's
    # check_ready / trigger / post_trigger in Python, one step at a time)
    obj_steps = max(10, min(args.steps, 100))
    for _ in range(3):
        loop.step_eager()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(obj_steps):
        loop._inputs.copy_(h_in[0], non_blocking=True)
        loop.step_eager()
        h_out[0][0, :nsl].copy_(loop.slopec.slopes.slopes, non_blocking=True)
        h_out[0][0, nsl:].copy_(loop.integ.out_comm.value, non_blocking=True)
        torch.cuda.synchronize(dev)
    obj_dt = time.perf_counter() - t0
    t_obj = torch.tensor([obj_dt], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t_obj, op=dist.ReduceOp.MAX)
    obj_value = world * obj_steps / float(t_obj.item())

    pieces = step_pieces(loop) if loop.fused_atmo else None
    accuracy = accuracy_vs_fp64(loop, *acc_field) if rank == 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, n, dt = time_cpu_oracle(cfg, budget_s=args.cpu_baseline_seconds, max_steps=200, loop=loop)
        cpu = {'value': v, 'unit': UNIT, 'cores': blas_threads(), 'kind': 'port',
               'sample': f'{n} CPU-oracle loop steps of the same system after 1 untimed step ({dt:.1f} s)'}

    loop_grad = None
    if world == 1 and not args.no_gradient:
        loop_grad = bench_loop_gradient(dev)

    adjoint_im = None
    if world == 1 and not args.no_adjoint:
        adjoint_im = bench_adjoint_im(dev, reps=max(3, min(args.steps, 10)),
                                      cpu_budget_s=0 if args.no_cpu_baseline else 10.0)

    sh_forms = None
    psf = None
    if world == 1 and not args.no_batched:
        sh_forms = bench_sh_forms(dev)
        psf = bench_psf(dev)

    batched_mc = None
    if not args.no_batched:
        batched_mc = bench_batched(dev, steps=50, cpu_budget_s=0 if args.no_cpu_baseline or world > 1 else 15.0)

    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': steps,
                'warmup': max(3, args.warmup), 'ms_per_step': ms_max / steps, 'higher_is_better': True,
                'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
                'config': config_dict(cfg, world),
                'e2e': {'value': e2e_value, 'unit': UNIT, 'h2d_bytes_per_step': int(loop.n_inputs * 8),
                        'd2h_bytes_per_step': int((nsl + nm) * 4),
                        'api': 'ScaoLoop.replay (captured 2-step graphs of two input / output slots); every step '
                               'inputs host->device and results device->host on copy streams beside the replays, '
                               'the host reading each replay\'s results one replay behind',
                        'steps': e2e_steps},
                'e2e_synchronous': {'value': e2e_sync_value, 'unit': UNIT,
                                    'api': 'the same, the host waiting for each replay\'s results before the next',
                                    'steps': e2e_steps},
                'e2e_object_api': {'value': obj_value, 'unit': UNIT, 'api': 'LoopControl.iter (object by object)',
                                   'steps': obj_steps},
                'gpu_launches': loop.kernels_per_step * steps,
                'step_graph': ('pipelined (DM projection concurrent with the SH chain' +
                               (', atmosphere early on a third stream)' if loop.early_atmo else ')'))
                if loop.pipelined else 'sequential',
                'roofline': {'bound': 'hbm', 'kernel': 'dm_project_tma_kernel', 'achieved': achieved, 'peak': peak,
                             'peak_kind': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak, 'traffic': DM_TRAFFIC_BYTES,
                             'traffic_source': 'stored ncu capture of this kernel and workload (bench.py comment)',
                             'traffic_over_algorithmic': DM_TRAFFIC_BYTES / dm_bytes,
                             'algorithmic_bytes_per_launch': dm_bytes, 'avg_launch_us': dm_ms * 1e3},
                'step_roofline': {'algorithmic_bytes': step_bytes,
                                  'achieved_gbs': step_bytes / (ms_max / steps / 1e3) / 1e9,
                                  'frac': step_bytes / (ms_max / steps / 1e3) / 1e9 / peak},
                'accuracy': accuracy, 'step_pieces': pieces, 'clocks': clk, 'cpu_baseline': cpu, 'adjoint_im': adjoint_im, 'loop_gradient': loop_grad,
                'sh_forms': sh_forms, 'psf': psf, 'batched_mc': batched_mc}
        print(json.dumps(line), flush=True)
    del loop
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def step_pieces(loop, reps=200):
    """Device time of the captured step and of its pieces, each captured in a
    graph of its own (CUDA events over ``reps`` replays after warm-up): the
    chain (atmosphere, SH, detector/CoG, reconstructor) of two steps without
    the DM projection, the DM projection alone, and the chain's parts."""
    import torch
    st = torch.cuda.current_stream(loop.device)

    def timeit(fn):
        for _ in range(10):
            fn()
        torch.cuda.synchronize(loop.device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(loop.device)
        return e0.elapsed_time(e1) / reps * 1e3

    dm_buf, nxt = loop._bufs
    graphs = []

    def graph_of(fn):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        graphs.append(g)
        return g.replay

    early = getattr(loop, 'early_atmo', False)

    def atmosphere(par):
        if early:
            loop._atmo_propagate(None, out=loop._early[par])
        else:
            loop._atmo_propagate(dm_buf[1 - par])

    def sh_chain(par):
        if early:
            loop._sh_ccd_slopec(mirror=dm_buf[1 - par], partial=loop._early[par])
        else:
            loop._chain()

    def chain_two_steps():
        for par in (1, 0):
            atmosphere(par)
            sh_chain(par)
            loop._rec_integ(out_next=nxt[1 - par])

    out = {'step_us': timeit(loop.replay) / loop.steps_per_replay,
           'chain_alone_us_per_step': timeit(graph_of(chain_two_steps)) / 2,
           'dm_alone_us': timeit(graph_of(lambda: loop.dm.project(nxt[1], dm_buf[1]))),
           'atmosphere_propagation_us': timeit(graph_of(lambda: atmosphere(0))),
           'sh_detector_slopes_us': timeit(graph_of(lambda: sh_chain(0))),
           'reconstructor_integrator_us': timeit(graph_of(lambda: loop._rec_integ(out_next=nxt[0]))),
           'early_atmosphere': early}
    del graphs
    _lib_status()
    return out


def profile_loop(dev, replays):
    """The headline step graph (ELT workload) set up and warmed, then
    ``replays`` replays (two steps each) between cudaProfilerStart/Stop, for
    ncu --profile-from-start off."""
    import torch
    from specula_b200.scao import ScaoLoop, elt_config
    loop = ScaoLoop(elt_config(), device_idx=dev.index)
    loop.start()
    loop.step_eager()
    loop.capture()
    for _ in range(3):
        loop.replay()
    torch.cuda.synchronize(dev)
    torch.cuda.cudart().cudaProfilerStart()
    for _ in range(replays):
        loop.replay()
    torch.cuda.synchronize(dev)
    torch.cuda.cudart().cudaProfilerStop()
    _lib_status()
    print(json.dumps({'profiled_replays': replays, 'steps_per_replay': loop.steps_per_replay,
                      'kernels_per_step': loop.kernels_per_step}), flush=True)


def profile_batched(dev, mc=False):
    """One replay of the batched graph (mc: the pipelined Monte-Carlo step,
    two steps) bracketed for a profiler."""
    import torch
    from specula_b200.batched import BatchedScao, mc_groups
    sys_b = BatchedScao(mc_groups(), device_idx=dev.index, dft='split_bf16')
    sys_b.start()
    if mc:
        sys_b.capture_mc(pipelined=True)
    else:
        sys_b.autotune()
        sys_b.capture()
    for _ in range(3):
        sys_b.replay()
    torch.cuda.synchronize(dev)
    torch.cuda.cudart().cudaProfilerStart()
    sys_b.replay()
    torch.cuda.synchronize(dev)
    torch.cuda.cudart().cudaProfilerStop()
    _lib_status()


def main():
    args = parse()
    if args.profile_loop:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        profile_loop(dev, args.profile_loop)
        return
    if args.profile_batched or args.profile_mc:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        profile_batched(dev, mc=args.profile_mc)
        return
    if args.batched_only:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        out = bench_batched(dev, steps=max(5, min(args.steps, 200)),
                            cpu_budget_s=0 if args.no_cpu_baseline else 15.0)
        print(json.dumps({'sh_forms': bench_sh_forms(dev), 'batched_mc': out}), flush=True)
        return
    if args.gradient_only:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({'loop_gradient': bench_loop_gradient(dev)}), flush=True)
        return
    if args.psf_only:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({'psf': bench_psf(dev)}), flush=True)
        return
    if args.adjoint_only:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        out = bench_adjoint_im(dev, reps=max(3, min(args.steps, 10)),
                               cpu_budget_s=0 if args.no_cpu_baseline else 10.0)
        print(json.dumps({'adjoint_im': out}), flush=True)
        return
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
