"""Turbulence evolution on the B200 (mirrors
specula/processing_objects/atmo_evolution.py:14-323).

Screens are synthesised once at construction (float64 on the device,
specula_b200.lib.phasescreen; read from / written to the reference's FITS
cache in ``data_dir`` when one is given, or read from
``user_defined_phasescreen``) and cut into per-layer strips exactly as
atmo_evolution.py:164-226 does (sqrt(Cn2), de-mean, nm, odd layers
flipped), then stored in float32.  Each step is one sb_atmo_evolve_inputs
call: the seeing and wind inputs are read on the device (float64 CUDA
tensors are used in place, anything else is staged into device buffers),
the per-layer shift, rot90, fractional-degree rotation and r0 scale are
computed there, the layer positions (float64, on the device) advance by
wind_speed * dt / pitch with the reference's cycling rule, and every layer
gets the column lerp, rot90, rotation and r0 scaling.  A captured CUDA
graph of trigger_code() therefore follows new input values.
"""
import ctypes
import math

import numpy as np
import torch

from specula_b200 import ASEC2RAD, _lib, cpuArray
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputValue
from specula_b200.data_objects.layer import Layer
from specula_b200.lib import fits_io
from specula_b200.lib.phasescreen import calc_phasescreen
from specula_b200.lib.phasescreen_manager import phasescreens_manager


def _cosdg_sindg(angle):
    """cos/sin of an angle in degrees, exact at multiples of 90 (scipy.special.cosdg/sindg)."""
    from scipy.special import cosdg, sindg
    return float(cosdg(angle)), float(sindg(angle))


class AtmoEvolution(BaseProcessingObj):
    def __init__(self, simul_params, L0: list, heights: list, Cn2: list, data_dir: str,
                 wavelengthInNm: float = 500.0, fov: float = 0.0, pixel_phasescreens: int = 8192, seed: int = 1,
                 verbose: bool = False, user_defined_phasescreen: str = '', make_cycle: bool = False,
                 fov_in_m: float = None, pupil_position: list = (0, 0), target_device_idx: int = None,
                 precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if make_cycle:
            raise NotImplementedError('make_cycle is not implemented')
        self.user_defined_phasescreen = user_defined_phasescreen
        npdt = np.float32 if self.precision == 1 else np.float64
        self.simul_params = simul_params
        self.pixel_pupil = simul_params.pixel_pupil
        self.pixel_pitch = simul_params.pixel_pitch
        self.zenithAngleInDeg = simul_params.zenithAngleInDeg
        self.n_phasescreens = len(heights)
        self.airmass = 1.0 / np.cos(np.radians(self.zenithAngleInDeg or 0.0), dtype=npdt)
        heights = np.array(heights, dtype=npdt)
        fov_rad = fov * ASEC2RAD
        self.pixel_layer = np.ceil((self.pixel_pupil + 2 * np.sqrt(np.sum(np.array(pupil_position, dtype=npdt) * 2))
                                    / self.pixel_pitch + abs(heights) / self.pixel_pitch * fov_rad) / 2.0) * 2.0
        if fov_in_m is not None:
            self.pixel_layer = np.full_like(heights, int(fov_in_m / self.pixel_pitch / 2.0) * 2)
        self.L0 = L0
        self.heights = heights
        self.Cn2 = np.array(Cn2, dtype=npdt)
        self.data_dir = data_dir
        self.wavelengthInNm = wavelengthInNm
        self.pixel_square_phasescreens = pixel_phasescreens
        if self.pixel_square_phasescreens < max(self.pixel_layer):
            raise ValueError('Error: phase-screens dimension must be greater than layer dimension!')
        if len(set(int(x) for x in self.pixel_layer)) != 1:
            raise NotImplementedError('AtmoEvolution: layers of different sizes are not on the specula_b200 path')
        if not np.isclose(np.sum(self.Cn2), 1.0, atol=1e-6):
            raise ValueError(f' Cn2 total must be 1. Instead is: {np.sum(self.Cn2)}.')
        if seed <= 0:
            raise ValueError('seed must be >0')
        self.verbose = verbose
        L = int(self.pixel_layer[0])
        self.layer_list = [Layer(L, L, self.pixel_pitch, float(h), precision=self.precision,
                                 target_device_idx=self.target_device_idx) for h in heights]
        for layer in self.layer_list:
            layer._unit_amplitude = True      # amplitude stays 1 (atmo_evolution.py never changes it)
        self.outputs['layer_list'] = self.layer_list
        self.inputs['seeing'] = InputValue(type=BaseValue)
        self.inputs['wind_speed'] = InputValue(type=BaseValue)
        self.inputs['wind_direction'] = InputValue(type=BaseValue)
        self.last_t = 0
        self.extra_delta_time = 0
        self.delta_time = 1
        self._seed = seed
        self.compute()

    @property
    def seed(self):
        return self._seed

    @seed.setter
    def seed(self, value):
        self._seed = value
        self.compute()

    def compute(self):
        """Square screens -> per-layer strips (atmo_evolution.py:142-252).
        With a non-empty ``data_dir`` the square screens go through the FITS
        cache of specula_b200.lib.phasescreen_manager (the reference's file
        names); an empty ``data_dir`` keeps them in memory only."""
        L = int(self.pixel_layer[0])
        if self.user_defined_phasescreen:
            self._user_defined_screen(L)
            return
        if len(np.unique(np.atleast_1d(self.L0))) != 1:
            raise NotImplementedError('AtmoEvolution: per-layer L0 is not on the specula_b200 path')
        L0 = float(np.atleast_1d(self.L0)[0])
        per_square = self.pixel_square_phasescreens // L
        n_sq = int(math.ceil(self.n_phasescreens / per_square))
        if self.data_dir:
            squares = phasescreens_manager([L0], self.pixel_square_phasescreens, self.pixel_pitch, self.data_dir,
                                           precision=self.precision, seed=np.arange(self._seed, self._seed + n_sq),
                                           device=self.device)
        else:
            squares = [calc_phasescreen(L0, self.pixel_square_phasescreens, self.pixel_pitch, seed=self._seed + k,
                                        device=self.device) for k in range(n_sq)]
        strips = []
        for i in range(self.n_phasescreens):
            sq, k = divmod(i, per_square)
            s = squares[sq][L * k:L * (k + 1), :].clone()
            s *= float(np.sqrt(self.Cn2[i]))
            s -= torch.mean(s)
            s *= self.wavelengthInNm / (2 * np.pi)
            if i % 2 != 0:
                s = torch.flip(s, dims=(1,))
            strips.append(s.to(self.dtype).contiguous())
        del squares
        self.phasescreens = strips
        self.phasescreens_sizes = [s.shape[1] for s in strips]
        self._positions = torch.zeros(self.n_phasescreens, dtype=torch.float64, device=self.device)

    def _user_defined_screen(self, L):
        """One layer from a FITS screen (atmo_evolution.py:150-165): made at
        least as tall as wide, de-meaned and converted to nm in the file's
        precision, then stored as float32."""
        if len(self.Cn2) > 1:
            raise ValueError('The user-defined phasescreen works only if the total phasescreens are 1.')
        scr = np.array(fits_io.getdata(self.user_defined_phasescreen))
        if scr.ndim != 2:
            raise ValueError('AtmoEvolution: the user-defined phasescreen must be a 2-D image')
        if scr.shape[0] < scr.shape[1]:
            scr = scr.T
        if scr.shape[0] < L or scr.shape[1] < L + 1:
            raise ValueError(f'AtmoEvolution: the user-defined phasescreen {scr.shape} is smaller than the '
                             f'{L} x {L + 1} pixels a layer reads')
        scr = scr - np.mean(scr)
        scr = scr * (self.wavelengthInNm / (2 * np.pi))
        strip = torch.as_tensor(np.ascontiguousarray(scr), device=self.device).to(self.dtype).contiguous()
        self.phasescreens = [strip]
        self.phasescreens_sizes = [strip.shape[1]]
        self._positions = torch.zeros(self.n_phasescreens, dtype=torch.float64, device=self.device)

    def set_last_position(self, last_position):
        lp = np.broadcast_to(np.asarray(last_position, dtype=np.float64), (self.n_phasescreens,))
        L = int(self.pixel_layer[0])
        for p, s in zip(lp, self.phasescreens_sizes):
            # the kernel reads columns [pos, pos + L]; keep the window inside the strip
            if not (0 <= p < s - L):
                raise ValueError(f'AtmoEvolution: position {p} outside [0, {s - L}) for a {s}-column strip')
        self._positions.copy_(torch.as_tensor(np.array(lp)))

    @property
    def last_position(self):
        return self._positions.detach().cpu().numpy()

    def set_last_t(self, last_t):
        self.last_t = last_t

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        for s in self.phasescreens:
            if s.dtype != torch.float32 or s.device != self.device or not s.is_contiguous():
                raise ValueError('AtmoEvolution: phase screens must be contiguous float32 on the device')
        n = self.n_phasescreens
        L = int(self.pixel_layer[0])
        arr = (_lib.AtmoLayer * n)()
        for k, (p, out) in enumerate(zip(self.phasescreens, self.layer_list)):
            arr[k].screen = p.data_ptr()
            arr[k].screen_ld = p.stride(0)
            arr[k].screen_cols = p.shape[1]
            arr[k].out = out.phaseInNm.data_ptr()
        self._layers = arr
        self._stage = {name: torch.zeros(1 if name == 'seeing' else n, dtype=torch.float64, device=self.device)
                       for name in ('seeing', 'wind_speed', 'wind_direction')}
        nb = _lib.load().sb_atmo_work_bytes(n)
        self._work = torch.empty(max(nb, 1), dtype=torch.uint8, device=self.device)
        # float32 constants of the r0 scale, with NumPy's promotion rules
        # (atmo_evolution.py:265-267: Python floats meet the float32 airmass)
        self._airmass_pow = float(self.airmass ** (-3. / 5.))
        self._lambda_factor = float(np.float32((self.wavelengthInNm / 500.0) ** (6. / 5.)))
        self._pitch_f = float(np.float32(self.pixel_pitch))
        del L

    def prepare_trigger(self, t):
        super().prepare_trigger(t)
        self.delta_time = self.t_to_seconds(self.current_time - self.last_t) + self.extra_delta_time

    def _device_input(self, name):
        """(pointer, count) of a float64 device vector holding input `name`:
        the input tensor itself when it already is one, else a staged copy."""
        v = self.local_inputs[name].value
        n_max = 1 if name == 'seeing' else self.n_phasescreens
        if (isinstance(v, torch.Tensor) and v.device == self.device and v.dtype == torch.float64
                and v.is_contiguous() and v.numel() in (1, n_max)):
            return v.data_ptr(), v.numel()
        dst = self._stage[name]
        src = torch.as_tensor(np.asarray(cpuArray(v), dtype=np.float64) if not isinstance(v, torch.Tensor) else v)
        src = src.to(device=self.device, dtype=torch.float64).reshape(-1)
        if src.numel() not in (1, n_max):
            raise ValueError(f'AtmoEvolution: {name} has {src.numel()} values for {n_max} layers')
        dst.copy_(src.expand(dst.numel()) if src.numel() == 1 else src)
        return dst.data_ptr(), dst.numel()

    def inputs_struct(self, delta_time):
        """sb_atmo_inputs for this step (device pointers to the inputs)."""
        ps, _ = self._device_input('seeing')
        pw, nw = self._device_input('wind_speed')
        pd, nd = self._device_input('wind_direction')
        return _lib.AtmoInputs(seeing=ps, wind_speed=pw, wind_direction=pd, n_wind_speed=nw, n_wind_direction=nd,
                               delta_time=float(delta_time), pixel_pitch=float(self.pixel_pitch),
                               pixel_pitch_f=self._pitch_f, airmass_pow=self._airmass_pow,
                               lambda_factor=self._lambda_factor)

    def layer_params(self, delta_time):
        """Per-layer kernel descriptors computed on the host
        (atmo_evolution.py:262-294), for sb_atmo_evolve."""
        seeing = float(cpuArray(self.local_inputs['seeing'].value))
        ws = np.broadcast_to(np.asarray(cpuArray(self.local_inputs['wind_speed'].value), dtype=np.float64),
                             (self.n_phasescreens,))
        wd = np.broadcast_to(np.asarray(cpuArray(self.local_inputs['wind_direction'].value), dtype=np.float64),
                             (self.n_phasescreens,))
        r0 = 0.9759 * 0.5 / (seeing * 4.848) * self.airmass ** (-3. / 5.)
        r0l = r0 * (self.wavelengthInNm / 500.0) ** (6. / 5.)
        scale = (self.pixel_pitch / r0l) ** (5. / 6.)
        delta = ws * delta_time / self.pixel_pitch
        _, wdi = np.modf(wd / 90.0)
        wdf_full, _ = np.modf(wd)
        L = int(self.pixel_layer[0])
        arr = (_lib.AtmoLayer * len(self.phasescreens))()
        for k, (p, out) in enumerate(zip(self.phasescreens, self.layer_list)):
            d = arr[k]
            d.screen = p.data_ptr()
            d.screen_ld = p.stride(0)
            d.screen_cols = p.shape[1]
            d.delta = float(delta[k])
            d.rot90 = int(wdi[k]) % 4
            d.rotate = int(wdf_full[k] != 0)
            if d.rotate:
                # scipy.ndimage.rotate(reshape=False): input = M @ output + offset
                c, s = _cosdg_sindg(wdf_full[k])
                ctr = (L - 1) / 2.0
                d.m00, d.m01, d.m10, d.m11 = c, s, -s, c
                d.off0 = ctr - (c * ctr + s * ctr)
                d.off1 = ctr - (-s * ctr + c * ctr)
            d.scale = float(scale)
            d.out = out.phaseInNm.data_ptr()
        return arr

    def trigger_code(self):
        L = int(self.pixel_layer[0])
        inp = self.inputs_struct(self.delta_time)
        _lib.call('sb_atmo_evolve_inputs', self._layers, self.n_phasescreens, L, self._positions.data_ptr(),
                  ctypes.byref(inp), self._work.data_ptr(), self._work.numel(), self.stream_handle())

    def post_trigger(self):
        for layer in self.layer_list:
            layer.generation_time = self.current_time
        self.last_t = self.current_time
