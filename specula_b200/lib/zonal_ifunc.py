"""Zonal influence functions by thin-plate splines (restates
specula/lib/compute_zonal_ifunc.py:6-164 on the device, float64 splines).

Actuators sit on a square n_act x n_act grid spanning [0, dim] or, with
``circ_geom``, on rings (1, 6, 12, ... actuators, ring spacing dim/n_act,
scaled by n_act/(n_act-1) for odd n_act).  Actuator i's function is the
thin-plate spline through 1 at actuator i and 0 at its neighbours within
9 dim / n_act (all actuators when that reaches dim/2, else pixels farther
than 0.8 of that radius are set to 0): with phi(r) = r^2 log r,
solve Phi w = e_i on the actuators and evaluate sum_j w_j phi(|p - x_j|)
at the pixel corners (0..dim-1).  Options as the reference:

* mechanical coupling: after each actuator's function is computed, every
  function becomes itself plus c0 times the sum of the functions within one
  actuator pitch (itself included) plus c1 times those within two pitches,
  i.e. cube <- C cube after each actuator, as the reference's loop does;
* slaving: actuators whose peak inside the pupil is below ``slaving_thr`` of
  their overall peak are slaved to the master actuators within 1.1 pitches
  (weights 1 / number of masters of each slave) and removed.

Returns (n_act_tot x n_pupil_pixels influence functions, mask[, coordinates]).
"""
import math

import numpy as np
import torch

from specula_b200.lib.make_mask import make_mask


def _tps(r):
    return torch.where(r > 0, r * r * torch.log(torch.where(r > 0, r, torch.ones_like(r))), torch.zeros_like(r))


def actuator_coordinates(dim, n_act, circ_geom=False, angle_offset=0.0):
    """(x, y) float64 arrays and the actuator pitch, as compute_zonal_ifunc.py:21-56."""
    step = float(dim) / float(n_act)
    if circ_geom:
        if n_act % 2 == 0:
            na = np.arange(round((n_act + 1) / 2)) * 6
        else:
            step *= float(n_act) / float(n_act - 1)
            na = np.arange(round(n_act / 2)) * 6
        na[0] = 1
        ang, rad = [], []
        for ia, n_ang in enumerate(na):
            for ja in range(int(n_ang)):
                ang.append(360. / n_ang * ja + angle_offset)
                rad.append(ia * step)
        ang, rad = np.array(ang), np.array(rad)
        x = rad * np.cos(np.radians(ang)) + dim / 2
        y = rad * np.sin(np.radians(ang)) + dim / 2
    else:
        gx, gy = np.meshgrid(np.linspace(0, dim, n_act), np.linspace(0, dim, n_act))
        x, y = gx.ravel(), gy.ravel()
    return x, y, step


def compute_zonal_ifunc(dim, n_act, dtype=torch.float32, circ_geom=False, angle_offset=0,
                        do_mech_coupling=False, coupling_coeffs=(0.31, 0.05), do_slaving=False, slaving_thr=0.1,
                        obsratio=0.0, diaratio=1.0, mask=None, return_coordinates=False, device='cuda'):
    if mask is None:
        mask = make_mask(dim, obsratio, diaratio)
    mask = np.asarray(mask).astype(float)
    idx = np.flatnonzero(mask.ravel())
    x, y, step = actuator_coordinates(dim, n_act, circ_geom, angle_offset)
    n_tot = len(x)
    f64 = dict(dtype=torch.float64, device=device)
    xa, ya = torch.as_tensor(x, **f64), torch.as_tensor(y, **f64)
    gy, gx = torch.meshgrid(torch.arange(dim, **f64), torch.arange(dim, **f64), indexing='ij')
    gx, gy = gx.reshape(-1), gy.reshape(-1)
    cube = torch.zeros((n_tot, dim * dim), dtype=dtype, device=device)
    reach = 9 * dim / n_act
    local = reach < dim / 2
    if do_mech_coupling:
        d = torch.sqrt((xa[:, None] - xa[None, :]) ** 2 + (ya[:, None] - ya[None, :]) ** 2)
        C = (torch.eye(n_tot, **f64) + coupling_coeffs[0] * (d <= step).to(torch.float64) +
             coupling_coeffs[1] * ((d > step) & (d <= 2 * step)).to(torch.float64)).to(dtype)
    for i in range(n_tot):
        if local:
            near = torch.nonzero(torch.sqrt((xa - xa[i]) ** 2 + (ya - ya[i]) ** 2) <= reach).flatten()
        else:
            near = torch.arange(n_tot, device=device)
        px, py = xa[near], ya[near]
        A = _tps(torch.sqrt((px[:, None] - px[None, :]) ** 2 + (py[:, None] - py[None, :]) ** 2))
        rhs = (near == i).to(torch.float64)
        w = torch.linalg.solve(A, rhs)
        val = _tps(torch.sqrt((gx[:, None] - px[None, :]) ** 2 + (gy[:, None] - py[None, :]) ** 2)) @ w
        if local:
            far = torch.sqrt((gx - xa[i]) ** 2 + (gy - ya[i]) ** 2) > 0.8 * reach
            val = torch.where(far, torch.zeros_like(val), val)
        cube[i] = val.to(dtype)
        if do_mech_coupling:
            cube = C @ cube
    coords = np.vstack((x, y))
    if do_slaving:
        idx_t = torch.as_tensor(idx, device=device)
        max_in = cube[:, idx_t].max(dim=1).values
        max_all = cube.max(dim=1).values
        master = (max_in >= slaving_thr * max_all).cpu().numpy()
        d = np.sqrt((x[:, None] - x[None, :]) ** 2 + (y[:, None] - y[None, :]) ** 2)
        S = np.zeros((n_tot, n_tot))
        S[np.ix_(master, ~master)] = (d <= 1.1 * step)[np.ix_(master, ~master)]
        S /= np.maximum(1.0, S.sum(axis=0))[None, :]
        cube = cube + (torch.as_tensor(S, device=device).to(dtype) @ cube)
        cube = cube[torch.as_tensor(np.flatnonzero(master), device=device)]
        coords = coords[:, master]
    ifs = cube[:, torch.as_tensor(idx, device=device)].contiguous()
    if return_coordinates:
        return ifs, mask, coords
    return ifs, mask
