"""CCD detector on the B200 (mirrors specula/processing_objects/ccd.py:22-305).

Same constructor, inputs (``in_i``) and outputs (``out_pixels``,
``integrated_i``).  ``trigger_code()`` is one sb_ccd_step call: integrate the
intensity, and on the steps that close a frame apply QE, background/dark,
Poisson and read-out noise and the ADU quantisation (ccd.py:198-262).

Noise uses Philox4x32-10 keyed by (photon_seed | readout_seed, frame,
pixel) instead of NumPy's PCG64 / CuPy's XORWOW, so draws are deterministic
and independent of launch shape; the reference's own CPU and GPU streams
already differ from each other, so only the distributions are shared.  The
frame counter lives on the device, so the object can be replayed from a CUDA
graph.  EMCCD excess noise (a Gamma draw of shape excess_delta * n and scale
emccd_gain, Marsaglia-Tsang), clock-induced charge (a Bernoulli electron),
charge-transfer inefficiency (sb_ccd_step_cte: cte0 * frame * cte1 before the
noise), pixel gains (constructor or setQuadrantGains) and a per-pixel QE map
(the reference's notUniformQe attributes) follow ccd.py:218-262 in its order.
start_time > 0 (ccd.py:199-207): nothing is integrated or read out before
start_time, and frames close every dt from there; the gate is evaluated on
the host at each trigger (a graph captured before start_time would replay
the capture-time decision), and start_time must be a multiple of the time
step.  Not on this path (raises NotImplementedError): 'auto' noise levels (a
table of vendor detector figures).  Binning (b x b)
runs as sb_ccd_step_binned: block sums scaled as the reference does
(ccd.py:262-280), then the same QE / noise / ADU model on the binned pixels.
"""
import torch

from specula_b200 import _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.connections import InputValue
from specula_b200.data_objects.intensity import Intensity
from specula_b200.data_objects.pixels import Pixels


class CCD(BaseProcessingObj):
    def __init__(self,
                 simul_params,
                 size,
                 dt: float,
                 bandw: float,
                 name: str = '',
                 binning: int = 1,
                 photon_noise: bool = False,
                 readout_noise: bool = False,
                 excess_noise: bool = False,
                 darkcurrent_noise: bool = False,
                 background_noise: bool = False,
                 cic_noise: bool = False,
                 cte_noise: bool = False,
                 readout_level='',
                 darkcurrent_level='',
                 background_level='',
                 cic_level: float = 0,
                 cte_mat=None,
                 quantum_eff: float = 1.0,
                 pixelGains=None,
                 photon_seed: int = 1,
                 readout_seed: int = 2,
                 excess_seed: int = 3,
                 excess_delta: float = 1.0,
                 start_time: int = 0,
                 ADU_gain: int = 8,
                 ADU_bias: int = 400,
                 emccd_gain: int = 1,
                 target_device_idx: int = None,
                 precision: int = None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if dt <= 0:
            raise ValueError(f'dt (integration time) is {dt} and must be greater than zero')
        self.loop_dt = self.seconds_to_t(simul_params.time_step)
        self._dt = self.seconds_to_t(dt)
        if self._dt % self.loop_dt != 0:
            raise ValueError(f'integration time dt={dt} must be a multiple of the basic simulation '
                             f'time_step={simul_params.time_step}')
        if 'auto' in (readout_level, darkcurrent_level, background_level):
            raise NotImplementedError("CCD: 'auto' levels are not on the specula_b200 path")
        self._start_time = self.seconds_to_t(start_time)
        if self._start_time < 0:
            raise ValueError(f'start_time is {start_time} and must not be negative')
        if self._start_time % self.loop_dt != 0:
            raise NotImplementedError(f'CCD: start_time={start_time} must be a multiple of the time step '
                                      f'{simul_params.time_step} on the specula_b200 path')
        if excess_noise:
            # the reference sets the EMCCD and ADU gains itself when excess noise is on (ccd.py:100-103)
            emccd_gain = 400
            ADU_gain = 1 / 20
        self._excess_noise = bool(excess_noise)
        self._excess_seed = int(excess_seed)
        self._excess_delta = float(excess_delta)
        self._emccd_gain = float(emccd_gain)
        self._cic_noise = bool(cic_noise)
        self._cic_level = float(cic_level)
        self._cte_noise = bool(cte_noise)
        self._cte_mat = cte_mat
        self._pixelGains = pixelGains
        # per-pixel QE (the reference's notUniformQe attributes, set by the user)
        self._notUniformQe = False
        self._notUniformQeMatrix = None
        self._normNotUniformQe = False
        self._photon_noise = bool(photon_noise)
        self._readout_noise = bool(readout_noise)
        self._darkcurrent_noise = bool(darkcurrent_noise)
        self._background_noise = bool(background_noise)
        self._readout_level = float(readout_level) if readout_level != '' else 0.0
        self._darkcurrent_level = float(darkcurrent_level) if darkcurrent_level != '' else 0.0
        self._background_level = float(background_level) if background_level != '' else 0.0
        self._qe = quantum_eff
        self._binning = binning
        self._bandw = bandw
        self._ADU_gain = ADU_gain
        self._ADU_bias = ADU_bias
        self._photon_seed = int(photon_seed)
        self._readout_seed = int(readout_seed)
        self._pixels = Pixels(size[0] // binning, size[1] // binning, target_device_idx=target_device_idx,
                              precision=precision)
        self._integrated_i = Intensity(size[0], size[1], target_device_idx=target_device_idx, precision=precision)
        self._frames_per_read = self._dt // self.loop_dt
        self._n_integrated = 0
        self.inputs['in_i'] = InputValue(type=Intensity)
        self.outputs['out_pixels'] = self._pixels
        self.outputs['integrated_i'] = self._integrated_i

    @property
    def dt(self):
        return self._dt

    def setQuadrantGains(self, quadrantsGains):
        """Pixel gains constant over the four quadrants of the frame, in the
        reference's quadrant order (ccd.py:289-296)."""
        import numpy as np
        rows, cols = self._pixels.size
        g = np.zeros((rows, cols), dtype=np.float32)
        for i in range(2):
            for j in range(2):
                g[(rows // self._binning // 2) * i:(rows // self._binning // 2) * (i + 1),
                  (cols // self._binning // 2) * j:(cols // self._binning // 2) * (j + 1)] = quadrantsGains[j * 2 + i]
        self._pixelGains = g

    @property
    def size(self):
        return self._pixels.size

    @property
    def bandw(self):
        return self._bandw

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        in_i = self.inputs['in_i'].get(self.target_device_idx)
        if in_i is None:
            raise ValueError('Input intensity object has not been set')
        if in_i.size != self._integrated_i.size:
            raise ValueError(f'CCD: intensity {in_i.size} does not match detector {self._integrated_i.size}')
        # sb_ccd_state: uint64 frame_index, int n_integrated, uint blocks_done
        self._state = torch.zeros(2, dtype=torch.int64, device=self.device)
        bg = self._background_level + self._darkcurrent_level \
            if (self._background_noise or self._darkcurrent_noise) else 0.0
        self._params = _lib.CcdParams(
            n_pixels=self._integrated_i.i.numel(), frames_per_read=int(self._frames_per_read),
            rate=float(self.t_to_seconds(self.loop_dt) * self._bandw), qe=float(self._qe), bg_plus_dark=float(bg),
            photon_noise=int(self._photon_noise), readout_noise=int(self._readout_noise),
            readout_level=self._readout_level, adu_gain=float(self._ADU_gain), adu_bias=float(self._ADU_bias),
            dark_level=self._darkcurrent_level, dark_noise=int(self._darkcurrent_noise),
            photon_seed=self._photon_seed, readout_seed=self._readout_seed, state=self._state.data_ptr(),
            cic_noise=int(self._cic_noise), cic_level=self._cic_level, excess_noise=int(self._excess_noise),
            excess_delta=self._excess_delta, emccd_gain=self._emccd_gain, excess_seed=self._excess_seed)
        rows, cols = self._pixels.size
        int_frame = self._photon_noise and not self._excess_noise
        self._gains_t = None
        if self._pixelGains is not None:
            if int_frame:
                raise ValueError('CCD: pixel gains multiply a float frame; with photon noise and no excess noise '
                                 "the reference's frame is an integer array (ccd.py:239-240)")
            self._gains_t = self._device_map(self._pixelGains, rows, cols, 'pixelGains')
            self._params.pixel_gains = self._gains_t.data_ptr()
        self._qe_t = None
        if self._notUniformQe:
            if self._normNotUniformQe and int_frame:
                raise ValueError('CCD: the QE-map normalisation multiplies a float frame; with photon noise and no '
                                 "excess noise the reference's frame is an integer array (ccd.py:242-245)")
            self._qe_t = self._device_map(self._notUniformQeMatrix, rows, cols, 'notUniformQeMatrix')
            self._params.qe_map = self._qe_t.data_ptr()
            self._params.qe_map_normalise = int(bool(self._normNotUniformQe))
        self._cte = None
        if self._cte_noise:
            if self._binning != 1 or rows != cols:
                raise NotImplementedError('CCD: CTE noise needs a square frame without binning (ccd.py:223-224)')
            import numpy as np
            m = np.zeros((rows, cols, 2), dtype=np.float32) if self._cte_mat is None else np.asarray(self._cte_mat)
            if m.shape != (rows, cols, 2):
                raise ValueError(f'CCD: cte_mat of shape {m.shape} for a {rows} x {cols} frame')
            self._cte = (self._tensor(np.ascontiguousarray(m[:, :, 0])).contiguous(),
                         self._tensor(np.ascontiguousarray(m[:, :, 1])).contiguous())
            nb = _lib.load().sb_ccd_cte_scratch_bytes(rows)
            self._cte_scratch = torch.zeros(nb, dtype=torch.uint8, device=self.device)
        self._in_i = in_i
        self._bin_scratch = None
        if self._binning > 1:
            rows, cols = self._integrated_i.size
            nb = _lib.load().sb_ccd_binned_scratch_bytes(rows, cols, self._binning)
            if nb == 0:
                raise ValueError('Warning: binning requested not applied')
            self._bin_scratch = torch.zeros(nb, dtype=torch.uint8, device=self.device)

    def _device_map(self, a, rows, cols, name):
        t = self._tensor(a).reshape(-1).contiguous()
        if t.numel() != rows * cols:
            raise ValueError(f'CCD: {name} must hold {rows} x {cols} values')
        return t

    def _before_start(self):
        # ccd.py:199: no integration (and no frame) before start_time
        return self._start_time > 0 and self.current_time < self._start_time

    def trigger_code(self):
        if self._before_start():
            return
        if self._cte is not None:
            rows = self._pixels.size[0]
            _lib.call('sb_ccd_step_cte', _byref(self._params), rows, self._cte[0].data_ptr(), self._cte[1].data_ptr(),
                      self._in_i.i.data_ptr(), self._integrated_i.i.data_ptr(), self._pixels.pixels.data_ptr(),
                      self._cte_scratch.data_ptr(), self._cte_scratch.numel(), self.stream_handle())
            return
        if self._bin_scratch is not None:
            rows, cols = self._integrated_i.size
            _lib.call('sb_ccd_step_binned', _byref(self._params), rows, cols, self._binning, self._in_i.i.data_ptr(),
                      self._integrated_i.i.data_ptr(), self._pixels.pixels.data_ptr(), self._bin_scratch.data_ptr(),
                      self._bin_scratch.numel(), self.stream_handle())
            return
        _lib.call('sb_ccd_step', _byref(self._params), self._in_i.i.data_ptr(), self._integrated_i.i.data_ptr(),
                  self._pixels.pixels.data_ptr(), self.stream_handle())

    def post_trigger(self):
        if self._before_start():
            return
        # host mirror of the device frame counter, for the time stamps
        self._n_integrated += 1
        if self._n_integrated >= self._frames_per_read:
            self._n_integrated = 0
            self._pixels.generation_time = self.current_time
        self._integrated_i.generation_time = self.current_time


def _byref(s):
    import ctypes
    return ctypes.byref(s)
