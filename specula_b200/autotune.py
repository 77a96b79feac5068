"""Autotuner of the library's tile shapes (an addition: the reference has no
tuned kernels).

Each tunable kernel family of the C library (``SB_TUNE_*`` in
specula_b200.h) has several compiled tile shapes.  ``Autotuner.tune`` runs
one launch per variant on the caller's own buffers and checks its output
against variant 0.  It then times every variant that agrees: CUDA events on
the current stream, the median of ``reps`` batches of ``launches`` launches
after warm-up.  It registers the fastest for that shape with
``sb_tune_set``; later launches of that shape (captured graphs included)
use it.

Results are kept per (device name, family, shape) and, when ``cache_path``
is given, in a JSON file, so a second process skips the timing.

Families wired here:

* ``dm_batched``: ``sb_dm_project_batched``, realisations per pass x mode-row
  groups (6 variants), and the register-blocked form (4 columns x 8 or 16
  realisations per thread) with 1024-, 512- or 256-column tiles (6 variants);
* ``sh_fp32``: ``sb_sh_forward_batched`` (FP32 form), sub-apertures per CTA
  (8, 4, 2);
* ``modalrec_batched``: ``sb_modalrec_batched``, reconstructor rows per CTA
  (2, 1, 4).
"""
import ctypes
import json
import os
import statistics

import torch

from specula_b200 import _lib

FAMILIES = {'dm_batched': _lib.SB_TUNE_DM_BATCHED, 'sh_fp32': _lib.SB_TUNE_SH_FP32,
            'modalrec_batched': _lib.SB_TUNE_MODALREC_BATCHED}


class Autotuner:
    def __init__(self, device, cache_path=None, reps=5, launches=10, rtol=1e-5):
        self.device = torch.device(device)
        self.cache_path = cache_path
        self.reps = int(reps)
        self.launches = int(launches)
        self.rtol = float(rtol)
        self.device_name = torch.cuda.get_device_name(self.device)
        self.results = []
        self._cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self._cache = json.load(f)

    def _cache_key(self, family, shape):
        return f'{self.device_name}|{family}|{",".join(str(int(v)) for v in shape)}'

    def _save(self):
        if not self.cache_path:
            return
        d = os.path.dirname(os.path.abspath(self.cache_path))
        os.makedirs(d, exist_ok=True)
        tmp = self.cache_path + '.tmp'
        with open(tmp, 'w') as f:
            json.dump(self._cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def tune(self, family, shape, launch, output):
        """Tune ``family`` (a key of FAMILIES) for ``shape`` (the three
        ints of its sb_tune_key).  ``launch()`` makes one launch of the kernel
        on the current stream; it must be idempotent (same inputs, same output
        tensor).  ``output`` is the tensor it writes, compared across variants."""
        lib = _lib.load()
        fam = FAMILIES[family]
        key = lib.sb_tune_key(*[int(v) for v in shape])
        ck = self._cache_key(family, shape)
        if ck in self._cache:
            v = int(self._cache[ck]['variant'])
            _lib.call('sb_tune_set', fam, key, v)
            rec = dict(self._cache[ck], family=family, shape=list(shape), cached=True)
            self.results.append(rec)
            return rec
        n = lib.sb_tune_variants(fam)
        st = torch.cuda.current_stream(self.device)
        ref = None
        times, agree = [], []
        for v in range(n):
            _lib.call('sb_tune_set', fam, key, v)
            launch()
            torch.cuda.synchronize(self.device)
            out = output.detach().clone()
            if ref is None:
                ref = out
                ok = True
            else:
                scale = float(ref.abs().max())
                ok = bool(torch.isfinite(out).all()) and float((out - ref).abs().max()) <= self.rtol * max(scale, 1e-30)
            agree.append(ok)
            if not ok:
                times.append(None)
                continue
            for _ in range(3):
                launch()
            samples = []
            for _ in range(self.reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(self.launches):
                    launch()
                e1.record(st)
                torch.cuda.synchronize(self.device)
                samples.append(e0.elapsed_time(e1) / self.launches * 1e3)
            times.append(statistics.median(samples))
        _lib.call('sb_device_status')
        best = min((t, v) for v, t in enumerate(times) if t is not None)[1]
        _lib.call('sb_tune_set', fam, key, best)
        rec = {'variant': best, 'name': lib.sb_tune_variant_name(fam, best).decode(),
               'times_us': [None if t is None else round(t, 3) for t in times],
               'agrees_with_variant0': agree, 'speedup_vs_variant0': times[0] / times[best]}
        self._cache[ck] = rec
        self._save()
        rec = dict(rec, family=family, shape=list(shape), cached=False)
        self.results.append(rec)
        return rec

    # -- the library's tunable launches ---------------------------------------
    def tune_dm_batched(self, ifunc, n_modes, n_valid, ld_if, cmd, ld_cmd, n_batch, sign, mask_idx, phase,
                        phase_stride):
        def launch():
            _lib.call('sb_dm_project_batched', ifunc.data_ptr(), n_modes, n_valid, ld_if, cmd.data_ptr(), ld_cmd,
                      n_batch, float(sign), mask_idx.data_ptr(), phase.data_ptr(), phase_stride,
                      torch.cuda.current_stream(self.device).cuda_stream)
        return self.tune('dm_batched', (n_modes, n_valid, n_batch), launch, phase)

    def tune_sh_fp32(self, plan, A, A_stride, phase, phase_stride, A_norm, A_norm_stride, n_norm, photon_scale,
                     intensity, intensity_stride, n_batch, scratch):
        def launch():
            _lib.call('sb_sh_forward_batched', ctypes.byref(plan), A.data_ptr(), A_stride, phase.data_ptr(),
                      phase_stride, A_norm.data_ptr(), A_norm_stride, n_norm, photon_scale, intensity.data_ptr(),
                      intensity_stride, n_batch, scratch.data_ptr(), scratch.numel(),
                      torch.cuda.current_stream(self.device).cuda_stream)
        return self.tune('sh_fp32', (plan.n_lenses, plan.cutsize, n_batch), launch, intensity)

    def tune_modalrec_batched(self, R, n_modes, n_slopes, ldr, slopes, lds, n_batch, modes, ldm):
        def launch():
            _lib.call('sb_modalrec_batched', R.data_ptr(), n_modes, n_slopes, ldr, slopes.data_ptr(), lds, n_batch,
                      modes.data_ptr(), ldm, torch.cuda.current_stream(self.device).cuda_stream)
        return self.tune('modalrec_batched', (n_modes, n_slopes, n_batch), launch, modes)
