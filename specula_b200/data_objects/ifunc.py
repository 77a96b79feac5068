"""Influence functions: (n_modes x n_valid_pixels) over a pupil mask
(mirrors specula/data_objects/ifunc.py:16-165).

``type_str='zernike'`` builds orthonormalised Zernike modes on the mask with
specula_b200.lib.zernike (the reference's compute_zern_ifunc); 'zonal'
builds thin-plate-spline actuator functions with
specula_b200.lib.zonal_ifunc on the object's device (the reference's
compute_zonal_ifunc).  'kl' and 'mixed' raise NotImplementedError, as in the
reference: a KL basis comes from
specula_b200.lib.modal_basis.make_modal_base_from_ifs_fft (zonal functions
plus an M2C), passed here as ``ifunc=``.
"""
import numpy as np
import torch

from specula_b200.base_data_obj import BaseDataObj


class IFunc(BaseDataObj):
    def __init__(self, ifunc=None, type_str: str = None, mask=None, npixels: int = None, nzern: int = None,
                 obsratio: float = None, diaratio: float = None, start_mode: int = None, nmodes: int = None,
                 n_act: int = None, circ_geom: bool = True, angle_offset: float = 0, do_mech_coupling: bool = False,
                 coupling_coeffs: list = (0.31, 0.05), do_slaving: bool = False, slaving_thr: float = 0.1,
                 idx_modes=None, target_device_idx=None, precision=None):
        super().__init__(precision=precision, target_device_idx=target_device_idx)
        if ifunc is None:
            if type_str is None:
                raise ValueError('At least one of ifunc and type must be set')
            if mask is not None:
                mask = (np.asarray(mask.cpu() if isinstance(mask, torch.Tensor) else mask) > 0).astype(np.float32)
            if npixels is None:
                raise ValueError('If ifunc is not set, then npixels must be set!')
            t = type_str.lower()
            if t in ('zern', 'zernike'):
                from specula_b200.lib.zernike import compute_zern_ifunc
                ifunc, mask = compute_zern_ifunc(npixels, nzern=nmodes, obsratio=obsratio, diaratio=diaratio,
                                                 mask=mask)
            elif t == 'zonal':
                from specula_b200.lib.zonal_ifunc import compute_zonal_ifunc
                ifunc, mask = compute_zonal_ifunc(npixels, n_act, dtype=self.dtype, circ_geom=circ_geom,
                                                  angle_offset=angle_offset, do_mech_coupling=do_mech_coupling,
                                                  coupling_coeffs=coupling_coeffs, do_slaving=do_slaving,
                                                  slaving_thr=slaving_thr,
                                                  obsratio=0.0 if obsratio is None else obsratio,
                                                  diaratio=1.0 if diaratio is None else diaratio, mask=mask,
                                                  device=self.device)
            elif t in ('kl', 'mixed'):
                raise NotImplementedError(f'IFunc type {type_str!r}: build the basis with '
                                          'specula_b200.lib.modal_basis.make_modal_base_from_ifs_fft')
            else:
                raise ValueError(f'Invalid ifunc type {type_str}')
        ifunc = np.asarray(ifunc.cpu() if isinstance(ifunc, torch.Tensor) else ifunc)
        mask = np.asarray(mask.cpu() if isinstance(mask, torch.Tensor) else mask)
        self._mask_np = mask
        self._influence_function = self._tensor(ifunc)
        self._mask_inf_func = self._tensor(mask)
        self._idx_np = np.flatnonzero(mask.ravel()).astype(np.int32)
        self.cut(start_mode=start_mode, nmodes=nmodes, idx_modes=idx_modes)

    @property
    def influence_function(self):
        return self._influence_function

    @influence_function.setter
    def influence_function(self, ifunc):
        self._influence_function = self._tensor(ifunc)

    @property
    def mask_inf_func(self):
        return self._mask_inf_func

    @property
    def idx_inf_func(self):
        """Flattened row-major indices of the mask pixels (int32, host)."""
        return self._idx_np

    @property
    def size(self):
        return tuple(self._influence_function.shape)

    def cut(self, start_mode=None, nmodes=None, idx_modes=None):
        nrows, ncols = self._influence_function.shape
        start_mode = 0 if start_mode is None else start_mode
        if idx_modes is not None:
            sel = torch.as_tensor(np.asarray(idx_modes), device=self.device)
            self._influence_function = (self._influence_function[sel, :] if ncols > nrows
                                        else self._influence_function[:, sel]).contiguous()
            return
        if nmodes is None:
            nmodes = nrows if ncols > nrows else ncols
        if ncols > nrows:
            self._influence_function = self._influence_function[start_mode:nmodes, :].contiguous()
        else:
            self._influence_function = self._influence_function[:, start_mode:nmodes].contiguous()
