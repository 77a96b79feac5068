"""KL modal basis from zonal influence functions (restates
specula/lib/modal_base_generator.py:1-367 on the device, in float64).

make_modal_base_from_ifs_fft:

1. modes to remove: piston, then Noll Zernikes 2..zern_modes+1 on the pupil,
   orthonormalised (QR) and made zero-mean / unit-RMS, projected onto the
   span of the influence functions (pinv); ``filt_modes`` only add empty
   rows, as in the reference (they shorten the basis);
2. each mode in turn is removed from every influence function;
3. geometric covariance F F^T / n_pix, SVD, whitening M = U / sqrt(S) on the
   first n_act - n_removed vectors (optionally more cut by a condition
   number bound);
4. turbulence covariance of the filtered functions from their Fourier
   transforms on an oversampled grid and the von Karman phase spectrum:
   Re(X^T diag(PS) conj(X)) / (n_pix^2 (os D)^2), computed as Y^T Y with
   Y = [Re X; Im X] sqrt(PS) (one real GEMM);
5. SVD of M^T C M; the KL modes are F^T M U2 and the modes-to-commands
   matrix K M U2 (with the Zernike modes first when requested).

Singular vectors are defined up to sign (and within degenerate subspaces),
so individual modes can differ from the reference's by a sign or a rotation
among modes of equal variance; the singular values and the spanned
subspaces agree.
"""
import numpy as np
import torch
from scipy.special import gamma

from specula_b200.lib.zernike import polar_grid, zernike


def phase_spectrum_constant():
    """Von Karman phase PSD constant (modal_base_generator.py:33)."""
    return (gamma(11.0 / 6.0) ** 2 / (2.0 * np.pi ** (11.0 / 3.0))) * (24.0 * gamma(6.0 / 5.0) / 5.0) ** (5.0 / 6.0)


def generate_phase_spectrum(f, r0, L0):
    return phase_spectrum_constant() * r0 ** (-5.0 / 3.0) * (f ** 2 + (1.0 / L0) ** 2) ** (-11.0 / 6.0)


def generate_distance_grid(N, M=None, device='cuda'):
    """sqrt(fx^2 + fy^2) in FFT order: index k <= N/2 -> k, else N - k."""
    M = N if M is None else M
    fx = torch.arange(N, dtype=torch.float64, device=device)
    fx = torch.where(fx <= N / 2, fx, N - fx)
    fy = torch.arange(M, dtype=torch.float64, device=device)
    fy = torch.where(fy <= M / 2, fy, M - fy)
    return torch.sqrt(fy[:, None] ** 2 + fx[None, :] ** 2)


def compute_ifs_covmat(pupil_mask, diameter, influence_functions, r0, L0, oversampling=2, chunk=256):
    """Turbulence covariance of the influence functions (float64)."""
    mask = torch.as_tensor(np.asarray(pupil_mask) > 0, device=influence_functions.device)
    idx = torch.nonzero(mask.reshape(-1)).flatten()
    n_pix = int(idx.numel())
    n_act = influence_functions.shape[0]
    size = max(mask.shape)
    Nf = oversampling * size
    f = generate_distance_grid(Nf, device=influence_functions.device) / (oversampling * diameter)
    w = torch.sqrt(generate_phase_spectrum(f, r0, L0)).reshape(-1)
    Y = []
    for a0 in range(0, n_act, chunk):
        blk = influence_functions[a0:a0 + chunk].to(torch.float64)
        sup = torch.zeros((blk.shape[0], Nf, Nf), dtype=torch.float64, device=blk.device)
        flat = torch.zeros((blk.shape[0], mask.shape[0] * mask.shape[1]), dtype=torch.float64, device=blk.device)
        flat[:, idx] = blk
        sup[:, :mask.shape[0], :mask.shape[1]] = flat.view(-1, mask.shape[0], mask.shape[1])
        ft = torch.fft.fft2(sup).reshape(blk.shape[0], -1)
        Y.append(torch.cat((ft.real * w, ft.imag * w), dim=1))
    Y = torch.cat(Y, dim=0)
    cov = Y @ Y.t()
    return cov / (n_pix ** 2 * (oversampling * diameter) ** 2)


def make_orto_modes(array):
    """Orthonormal rows spanning ``array``'s rows (QR, utils.py:51-84)."""
    if array.shape[1] > array.shape[0]:
        q, _ = torch.linalg.qr(array.t())
        return q.t()
    q, _ = torch.linalg.qr(array)
    return q


def make_modal_base_from_ifs_fft(pupil_mask, diameter, influence_functions, r0, L0, zern_modes=0,
                                 oversampling=2, filt_modes=None, if_max_condition_number=None, verbose=False,
                                 dtype=torch.float32):
    """(kl_basis n_modes x n_pix, m2c n_act x n_modes, {'S1', 'S2'}) on the
    influence functions' device; ``dtype`` of the returned bases."""
    F0 = torch.as_tensor(influence_functions)
    dev = F0.device
    F0 = F0.to(torch.float64)
    mask = np.asarray(pupil_mask) > 0
    idx = np.flatnonzero(mask.ravel())
    n_pix = len(idx)
    if F0.shape[1] != n_pix:
        raise ValueError(f'influence_functions should have shape (n_actuators, {n_pix})')
    n_act = F0.shape[0]
    n_rem = 1 + zern_modes + (0 if filt_modes is None else int(np.asarray(filt_modes).shape[0]))
    R = torch.zeros((n_rem, n_pix), dtype=torch.float64, device=dev)
    R[0] = 1.0
    coef_zern = None
    if zern_modes > 0:
        rho, theta = polar_grid(mask.shape[0], np.float64)
        for k in range(zern_modes):
            z = zernike(k + 2, rho, theta, np.float64)
            R[k + 1] = torch.as_tensor(z.ravel()[idx], device=dev)
        R = make_orto_modes(R)
        for k in range(1, zern_modes + 1):
            R[k] -= R[k].mean()
            R[k] /= torch.sqrt(torch.mean(R[k] ** 2))
        # pseudo-inverse with scipy's default cutoff for the basis precision
        # (max(M, N) * eps of ``dtype`` times the largest singular value)
        rtol = max(F0.shape) * torch.finfo(dtype).eps
        coef_zern = R @ torch.linalg.pinv(F0, rtol=rtol)
        R = coef_zern @ F0
    coef = torch.zeros((n_rem, n_act), dtype=torch.float64, device=dev)
    F = F0.clone()
    for m in range(n_rem):
        mode = R[m]
        norm = torch.dot(mode, mode)
        if norm > 0:
            coef[m] = (F @ mode) / norm
            F -= coef[m][:, None] * mode[None, :]
    U1, S1, _ = torch.linalg.svd((F @ F.t()) / n_pix)
    n_keep = n_act - n_rem
    if if_max_condition_number is not None:
        cond = S1[0] / S1[n_act - n_rem - 1]
        if cond > if_max_condition_number:
            n_cut = int(torch.count_nonzero(S1[:n_act - n_rem] < S1[0] / if_max_condition_number))
            n_rem += n_cut
            n_keep = n_act - n_rem
    if verbose:
        print(f'KL basis: {n_keep} modes from {n_act} actuators, condition {float(S1[0] / S1[n_keep - 1]):.3g}')
    M = torch.zeros((n_act, n_act), dtype=torch.float64, device=dev)
    M[:, :n_keep] = U1[:, :n_keep] / torch.sqrt(S1[:n_keep])[None, :]
    C = compute_ifs_covmat(mask, diameter, F, r0, L0, oversampling)
    U2, S2, _ = torch.linalg.svd(M.t() @ C @ M)
    Bp = M @ U2
    kl = (F.t() @ Bp[:, :n_keep]).t()
    if zern_modes > 0:
        kl = torch.cat((R[1:zern_modes + 1], kl), dim=0)
        K = torch.eye(n_act, dtype=torch.float64, device=dev) - coef_zern[1:zern_modes + 1].t() @ coef[1:zern_modes + 1]
        m2c = torch.cat((coef_zern[1:zern_modes + 1].t(), K @ Bp[:, :n_keep]), dim=1)
    else:
        K = torch.eye(n_act, dtype=torch.float64, device=dev) - torch.outer(coef[0], coef[0])
        m2c = K @ Bp[:, :n_keep]
    return kl.to(dtype).contiguous(), m2c.to(dtype).contiguous(), {'S1': S1, 'S2': S2}
