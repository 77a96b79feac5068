"""The interaction-matrix contraction on the lenslet-major copy of the
influence functions (sb_intmat_lenslet_ifunc + sb_intmat_contract_lenslets)
against the gather contraction (sb_intmat_contract), bit for bit, and against
a float64 host contraction: IM[m][j] = scale * sum_px J[j][px] IF[m][px]
over the pixels of slope j's sub-aperture (im_rec_calibrator.py:58-63 in its
small-amplitude limit)."""
import numpy as np
import pytest

torch = pytest.importorskip('torch')

from tests.cases import rel_max_err  # noqa: E402

pytestmark = pytest.mark.gpu

HOST_TOL = 1e-5


def _system(P, n=12, n_modes=37, seed=0):
    """Random sub-aperture map, mirror mask (some field pixels outside it),
    Jacobian, fluxes (one zero, two below the CoG cut-off) and influence
    functions."""
    rng = np.random.default_rng(seed)
    field = n * P
    field_ld = field + 8
    valid = np.flatnonzero(rng.random(n * n) < 0.7).astype(np.int32)
    n_valid = valid.size
    slot = np.full(n * n, -1, np.int32)
    slot[valid] = np.arange(n_valid, dtype=np.int32)
    inside = rng.random((field, field)) < 0.9
    n_cols = int(inside.sum())
    ld_if = (n_cols + 31) // 32 * 32
    pix2col = np.full((field, field_ld), -1, np.int32)
    pix2col[:, :field][inside] = np.arange(n_cols, dtype=np.int32)
    jac = rng.standard_normal((2, n_valid, P * P)).astype(np.float32)
    tot = rng.uniform(0.5, 2.0, n_valid).astype(np.float32)
    tot[0] = 0.0
    tot[1:3] = 1e-5                  # below 1e-3 * mean: inactive
    IF = np.zeros((n_modes, ld_if), np.float32)
    IF[:, :n_cols] = rng.standard_normal((n_modes, n_cols))
    return dict(P=P, n=n, field_ld=field_ld, valid=valid, slot=slot, pix2col=pix2col, jac=jac, tot=tot, IF=IF,
                ld_if=ld_if, n_modes=n_modes, n_valid=n_valid)


def _host(s, scale):
    """float64 contraction with the CoG cut-off of sh_slopec.py:400."""
    P, n, nv = s['P'], s['n'], s['n_valid']
    tot = s['tot'].astype(np.float64)
    act = (tot > 0) & (1.0 / np.where(tot > 0, tot, 1.0) <= 1.0 / (tot.mean() * 1e-3))
    im = np.zeros((s['n_modes'], 2 * nv))
    for k, L in enumerate(s['valid']):
        if not act[k]:
            continue
        li, lj = divmod(int(L), n)
        cols = s['pix2col'][li * P:(li + 1) * P, lj * P:(lj + 1) * P].ravel()
        f = np.where(cols >= 0, s['IF'][:, np.maximum(cols, 0)].astype(np.float64), 0.0)
        im[:, k] = f @ s['jac'][0, k].astype(np.float64)
        im[:, nv + k] = f @ s['jac'][1, k].astype(np.float64)
    return scale * im


@pytest.mark.parametrize('P', [4, 8])
def test_lenslet_contraction_equals_gather(cuda, P):
    from specula_b200 import _lib
    s = _system(P)
    dev = torch.device('cuda', 0)
    t = {k: torch.as_tensor(s[k], device=dev) for k in ('valid', 'slot', 'pix2col', 'jac', 'tot', 'IF')}
    nv, nm, scale = s['n_valid'], s['n_modes'], -2.0
    stream = torch.cuda.current_stream().cuda_stream
    ifl = torch.full((nm, nv, P, P), float('nan'), device=dev)
    _lib.call('sb_intmat_lenslet_ifunc', t['IF'].data_ptr(), nm, s['ld_if'], t['valid'].data_ptr(), nv, P, s['n'],
              s['field_ld'], t['pix2col'].data_ptr(), ifl.data_ptr(), stream)
    im_l = torch.full((nm, 2 * nv), float('nan'), device=dev)
    im_g = torch.full((nm, 2 * nv), float('nan'), device=dev)
    _lib.call('sb_intmat_contract_lenslets', t['jac'].data_ptr(), t['tot'].data_ptr(), nv, P, ifl.data_ptr(), nm,
              scale, im_l.data_ptr(), stream)
    _lib.call('sb_intmat_contract', t['jac'].data_ptr(), t['tot'].data_ptr(), nv, P, s['n'], s['field_ld'],
              t['slot'].data_ptr(), t['pix2col'].data_ptr(), t['IF'].data_ptr(), nm, s['ld_if'], scale,
              im_g.data_ptr(), stream)
    torch.cuda.synchronize()
    _lib.call('sb_device_status')
    # the copy: every sample of each valid sub-aperture, 0 outside the mirror
    li, lj = np.divmod(s['valid'], s['n'])
    r, c = np.meshgrid(np.arange(P), np.arange(P), indexing='ij')
    cols = s['pix2col'][li[:, None, None] * P + r[None], lj[:, None, None] * P + c[None]]   # [s][r][c]
    want = np.where(cols >= 0, s['IF'][:, np.maximum(cols, 0)], 0.0).transpose(0, 1, 3, 2)  # [m][s][c][r]
    assert np.array_equal(ifl.cpu().numpy(), want)
    assert torch.equal(im_l, im_g)
    ref = _host(s, scale)
    assert rel_max_err(im_l.cpu().numpy(), ref) <= HOST_TOL
    assert float(im_l[:, 0].abs().max()) == 0.0 and float(im_l[:, 1].abs().max()) == 0.0   # cut-off
    # without fluxes every valid sub-aperture contributes
    _lib.call('sb_intmat_contract_lenslets', t['jac'].data_ptr(), 0, nv, P, ifl.data_ptr(), nm, scale,
              im_l.data_ptr(), stream)
    _lib.call('sb_intmat_contract', t['jac'].data_ptr(), 0, nv, P, s['n'], s['field_ld'], t['slot'].data_ptr(),
              t['pix2col'].data_ptr(), t['IF'].data_ptr(), nm, s['ld_if'], scale, im_g.data_ptr(), stream)
    torch.cuda.synchronize()
    assert torch.equal(im_l, im_g)
    assert float(im_l[:, 0].abs().max()) > 0


def test_calibration_system_contraction_forms_agree(cuda):
    """On the 500-Zernike calibration system with the CoG cut-off applied,
    the default (lenslet-major) contraction, the TMA row contraction and the
    gather contraction give the same matrix bit for bit."""
    from specula_b200.calibration import ShCalibrationSystem
    cal = ShCalibrationSystem()
    adj = cal.adjoint
    assert adj.contraction == 'lenslet'
    assert adj.lenslet_ifunc(cal.dm._IF, cal.dm._ld, cal._pix2col) is not None
    forms = {}
    for form in ('lenslet', 'rows', 'gather'):
        adj.contraction = form
        forms[form] = cal.adjoint_intmat()
    adj.contraction = 'lenslet'
    torch.cuda.synchronize()
    assert torch.equal(forms['lenslet'], forms['gather'])
    assert torch.equal(forms['rows'], forms['gather'])
    assert float(forms['lenslet'].abs().max()) > 0
