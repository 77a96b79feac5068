"""Shack-Hartmann wavefront sensor on the B200 (mirrors
specula/processing_objects/sh.py:30-477).

Same constructor, inputs (``in_ef``: ElectricField) and outputs (``out_i``:
Intensity) as the reference.  ``setup()`` solves the geometry on the host
(sh.py:112-323), uploads the pruned-DFT / field-stop / rebin tables and
captures ``trigger_code()`` in a CUDA graph (as the reference's
build_stream).  ``trigger_code()`` makes one C-ABI call, sb_sh_forward
(preceded by sb_edge_extrapolate + sb_interp2d_field when the geometry
oversamples the field), which also applies the photon normalisation of
sh.py:422-428 on the device.

With ``laser_launch_tel`` the laser-guide-star form runs (sh.py:289-321,
382-394): the sub-aperture images are correlated with the sodium-spot
kernels of a GaussianConvolutionKernel (no launcher position) or a
ConvolutionKernel (launcher position, ``sodium_altitude`` /
``sodium_intensity`` inputs), one sb_sh_forward_lgs call per step.

``dft='split_bf16'`` (an addition; the reference has one FFT path) runs the
two small DFT products on the tcgen05 tensor cores in split-BF16
(sb_sh_forward_split_bf16); geometries without such a kernel raise
ValueError at setup.
"""
import ctypes
import math

import numpy as np
import torch

from specula_b200 import RAD2ASEC, _lib
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.connections import InputValue
from specula_b200.data_objects.electric_field import ElectricField
from specula_b200.data_objects.intensity import Intensity
from specula_b200.data_objects.lenslet import Lenslet
from specula_b200.lib import sh_geometry as shg
from specula_b200.lib.lgs import lgs_tables
from specula_b200.base_value import BaseValue
from specula_b200.data_objects.convolution_kernel import ConvolutionKernel, GaussianConvolutionKernel
from specula_b200.lib.edge_extrapolation import extrapolation_tables, per_pixel_tables
from specula_b200.lib.interp2d import interp_coords


class SH(BaseProcessingObj):
    def __init__(self,
                 wavelengthInNm: float,
                 subap_wanted_fov: float,
                 sensor_pxscale: float,
                 subap_on_diameter: int,
                 subap_npx: int,
                 FoVres30mas: bool = False,
                 squaremask: bool = True,
                 fov_ovs_coeff: float = 0,
                 xShiftPhInPixel: float = 0,
                 yShiftPhInPixel: float = 0,
                 aXShiftPhInPixel: float = 0,
                 aYShiftPhInPixel: float = 0,
                 rotAnglePhInDeg: float = 0,
                 aRotAnglePhInDeg: float = 0,
                 do_not_double_fov_ovs: bool = False,
                 set_fov_res_to_turbpxsc: bool = False,
                 laser_launch_tel=None,
                 target_device_idx: int = None,
                 precision: int = None,
                 dft: str = 'fp32'):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        if dft not in ('fp32', 'split_bf16'):
            raise ValueError(f"SH: dft must be 'fp32' or 'split_bf16', not {dft!r}")
        if laser_launch_tel is not None and dft != 'fp32':
            raise ValueError("SH: the laser-guide-star form runs with dft='fp32'")
        self._dft = dft
        self._laser_launch_tel = laser_launch_tel
        self._kernelobj = None
        self._wavelengthInNm = wavelengthInNm
        self._lenslet = Lenslet(subap_on_diameter)
        self._subap_wanted_fov_arcsec = subap_wanted_fov
        self._sensor_pxscale_arcsec = sensor_pxscale
        self._subap_npx = subap_npx
        self._opts = dict(FoVres30mas=FoVres30mas, squaremask=squaremask, fov_ovs_coeff=fov_ovs_coeff,
                          xShiftPhInPixel=xShiftPhInPixel, yShiftPhInPixel=yShiftPhInPixel,
                          aXShiftPhInPixel=aXShiftPhInPixel, aYShiftPhInPixel=aYShiftPhInPixel,
                          rotAnglePhInDeg=rotAnglePhInDeg, aRotAnglePhInDeg=aRotAnglePhInDeg,
                          do_not_double_fov_ovs=do_not_double_fov_ovs,
                          set_fov_res_to_turbpxsc=set_fov_res_to_turbpxsc)
        self._ccd_side = subap_npx * self._lenslet.n_lenses
        self._out_i = Intensity(self._ccd_side, self._ccd_side, precision=self.precision,
                                target_device_idx=self.target_device_idx)
        self.geometry = None
        if laser_launch_tel is not None:
            # sodium profile of the elongated kernel (sh.py:105-107)
            self.inputs['sodium_altitude'] = InputValue(type=BaseValue, optional=True)
            self.inputs['sodium_intensity'] = InputValue(type=BaseValue, optional=True)
        self.inputs['in_ef'] = InputValue(type=ElectricField)
        self.outputs['out_i'] = self._out_i
        self._photon_scale = None

    # geometry accessors with the reference's attribute names
    @property
    def _np_sub(self):
        return self.geometry.np_sub

    @property
    def _fft_size(self):
        return self.geometry.fft_size

    @property
    def _cutpixels(self):
        return self.geometry.cutpixels

    @property
    def _cutsize(self):
        return self.geometry.cutsize

    @property
    def _fov_ovs(self):
        return self.geometry.fov_ovs

    @property
    def _ovs_np_sub(self):
        return self.geometry.ovs_np_sub

    @property
    def subap_npx(self):
        return self._subap_npx

    @property
    def subap_on_diameter(self):
        return self._lenslet.n_lenses

    def setup(self):
        super().setup()
        self._require_gpu_fp32()
        _lib.load()
        in_ef = self.inputs['in_ef'].get(self.target_device_idx)
        ef_size = in_ef.size[0]
        g = shg.solve(self._wavelengthInNm, self._subap_wanted_fov_arcsec, self._sensor_pxscale_arcsec,
                      self._lenslet.n_lenses, self._subap_npx, ef_size, in_ef.pixel_pitch, **self._opts)
        self.geometry = g
        p = g.ovs_np_sub
        n = g.n_lenses
        field = int(ef_size * g.fov_ovs) if g.do_interpolation else ef_size
        if field != n * p:
            raise ValueError(f'SH: sampled field of {field} px is not {n} sub-apertures of {p} px')
        dev = self.device
        tw = shg.twiddle_table(p, g.fft_size, g.cutpixels)
        tilt = shg.tilt_table(p, g.fft_size)
        self._tw = torch.as_tensor(np.ascontiguousarray(tw).view(np.float32).reshape(-1), device=dev)
        self._tilt = torch.as_tensor(np.ascontiguousarray(tilt).view(np.float32).reshape(-1), device=dev)
        self._mask = torch.as_tensor(shg.field_stop_cut(g).reshape(-1), device=dev)
        self._rebin = torch.as_tensor(shg.rebin_table(g.cutsize, g.subap_npx).reshape(-1), device=dev)
        self._plan = _lib.ShPlan(n_lenses=n, np_sub=p, cutsize=g.cutsize, subap_npx=g.subap_npx,
                                 field_ld=field, phase_to_rad=float(np.float32((2 * math.pi) / self._wavelengthInNm)),
                                 twiddle=self._tw.data_ptr(), tilt=self._tilt.data_ptr(),
                                 fp_mask=self._mask.data_ptr(), rebin=self._rebin.data_ptr())
        nbytes = _lib.load().sb_sh_scratch_bytes(self._plan)
        if nbytes == 0:
            raise ValueError('SH: geometry does not fit the kernel limits')
        if self._dft == 'split_bf16' and not _lib.load().sb_sh_split_bf16_supported(self._plan):
            raise ValueError(f'SH: no split-BF16 tensor-core kernel for np_sub={p}, cutsize={g.cutsize}, '
                             f'subap_npx={g.subap_npx}')
        self._forward = 'sb_sh_forward' if self._dft == 'fp32' else 'sb_sh_forward_split_bf16'
        if self._laser_launch_tel is not None:
            self._setup_lgs(g, in_ef, field)
        self._scratch = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self._in_ef = in_ef
        if g.do_interpolation:
            # edge extrapolation tables from the pupil amplitude (sh.py:452-458)
            s1, s2 = extrapolation_tables(in_ef.A.detach().cpu().numpy(), do_ext_2_pix=True)
            t1, t2 = per_pixel_tables(s1, s2)
            self._ext1 = torch.as_tensor(t1, device=dev)
            self._ext2 = torch.as_tensor(t2, device=dev)
            yy, xx = interp_coords(in_ef.size, (field, field), g.rot_angle, g.xy_shift[0], g.xy_shift[1])
            self._yy = torch.as_tensor(yy, device=dev)
            self._xx = torch.as_tensor(xx, device=dev)
            self._phase_ext = torch.empty_like(in_ef.phaseInNm)
            self._wf1_A = torch.empty((field, field), dtype=self.dtype, device=dev)
            self._wf1_phase = torch.empty((field, field), dtype=self.dtype, device=dev)
        self._photon_scale = self._current_photon_scale()
        self.build_stream(allow_parallel=False)

    def _setup_lgs(self, g, in_ef, field):
        """Kernel object and DFT tables of the laser-guide-star form (sh.py:289-321)."""
        N = g.fft_size
        if not _lib.load().sb_sh_lgs_supported(self._plan, N):
            raise ValueError(f'SH: no laser-guide-star kernel for np_sub={g.ovs_np_sub}, fft_size={N}, '
                             f'cutsize={g.cutsize}, subap_npx={g.subap_npx}')
        llt = self._laser_launch_tel
        wf1_pitch = in_ef.pixel_pitch * in_ef.size[0] / field
        pxscale = self._wavelengthInNm / 1e9 / (wf1_pitch * N) * RAD2ASEC
        pupil_size_m = in_ef.pixel_pitch * in_ef.size[0]
        n = g.n_lenses
        if len(llt.tel_pos) == 0:
            self._kernelobj = GaussianConvolutionKernel(dimx=n, dimy=n, pxscale=pxscale, pupil_size_m=pupil_size_m,
                                                        dimension=N, spot_size=llt.spot_size, oversampling=1,
                                                        return_fft=True, positive_shift_tt=True,
                                                        target_device_idx=self.target_device_idx)
        else:
            theta = llt.beacon_tt if len(llt.beacon_tt) != 0 else [0.0, 0.0]
            self._kernelobj = ConvolutionKernel(dimx=n, dimy=n, pxscale=pxscale, pupil_size_m=pupil_size_m,
                                                dimension=N, launcher_pos=llt.tel_pos, seeing=0.0,
                                                launcher_size=llt.spot_size, zfocus=llt.beacon_focus, theta=theta,
                                                oversampling=1, return_fft=True, positive_shift_tt=True,
                                                target_device_idx=self.target_device_idx)
        w_full_t, w_dft, v_inv_t = lgs_tables(g.ovs_np_sub, N, g.cutpixels, g.cutsize)
        dev = self.device
        self._lgs_w = [torch.as_tensor(np.ascontiguousarray(t).view(np.float32).reshape(-1), device=dev)
                       for t in (w_full_t, w_dft, v_inv_t)]
        self._lgs = _lib.ShLgsTables(fft_size=N, w_full_t=self._lgs_w[0].data_ptr(), w_dft=self._lgs_w[1].data_ptr(),
                                     v_inv_t=self._lgs_w[2].data_ptr(),
                                     kernel_spectra=self._kernelobj.kernels.data_ptr())
        self._prepare_kernels()

    def _prepare_kernels(self):
        """Recompute the kernels when their parameters changed (sh.py:330-347);
        the kernel tensors keep their addresses, so a captured graph sees the
        new values."""
        if len(self._laser_launch_tel.tel_pos) != 0:
            alt = self.inputs['sodium_altitude'].get(self.target_device_idx)
            inten = self.inputs['sodium_intensity'].get(self.target_device_idx)
            if alt is None or inten is None:
                raise ValueError('sodium_altitude and sodium_intensity must be provided')
            alt, inten = alt.value, inten.value
        else:
            alt = inten = None
        before = self._kernelobj._kernel_fn
        self._kernelobj.prepare_for_sh(sodium_altitude=alt, sodium_intensity=inten, current_time=self.current_time)
        if self._kernelobj._kernel_fn != before:
            # the kernels were written on the current stream; the step may run on another
            torch.cuda.current_stream(self.device).synchronize()

    def _current_photon_scale(self):
        ef = self._in_ef
        return float(ef.S0) * (ef.pixel_pitch ** 2)

    def trigger_code(self):
        g = self.geometry
        ef = self._in_ef
        st = self.stream_handle()
        if g.do_interpolation:
            n_in = ef.phaseInNm.numel()
            _lib.call('sb_edge_extrapolate', ef.phaseInNm.data_ptr(), self._ext1.data_ptr(), self._ext2.data_ptr(),
                      n_in, self._phase_ext.data_ptr(), st)
            _lib.call('sb_interp2d_field', ef.A.data_ptr(), self._phase_ext.data_ptr(), ef.size[0], ef.size[1],
                      self._yy.data_ptr(), self._xx.data_ptr(), self._yy.numel(), self._wf1_A.data_ptr(),
                      self._wf1_phase.data_ptr(), st)
            A, P = self._wf1_A, self._wf1_phase
        else:
            A, P = ef.A, ef.phaseInNm
        if self._kernelobj is not None:
            _lib.call('sb_sh_forward_lgs', C_plan(self._plan), ctypes.byref(self._lgs), A.data_ptr(), P.data_ptr(),
                      ef.A.data_ptr(), ef.A.numel(), self._photon_scale, self._out_i.i.data_ptr(),
                      self._scratch.data_ptr(), self._scratch.numel(), st)
            return
        _lib.call(self._forward, C_plan(self._plan), A.data_ptr(), P.data_ptr(), ef.A.data_ptr(), ef.A.numel(),
                  self._photon_scale, self._out_i.i.data_ptr(), self._scratch.data_ptr(), self._scratch.numel(), st)

    def prepare_trigger(self, t):
        super().prepare_trigger(t)
        if self._kernelobj is not None:
            self._prepare_kernels()
        if self._photon_scale is not None and self._current_photon_scale() != self._photon_scale:
            # S0 or pitch changed: the captured graph holds the old value
            self._photon_scale = self._current_photon_scale()
            self.cuda_graph = None
            self.build_stream(allow_parallel=False)

    def post_trigger(self):
        super().post_trigger()
        self._out_i.generation_time = self.current_time


def C_plan(plan):
    import ctypes
    return ctypes.byref(plan)
