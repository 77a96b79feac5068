"""Zonal influence functions and the KL modal basis (setup-time, row a18)
against the reference's own outputs (tests/golden/kl_fp32.npz, written by
make_golden.py --kl from lib/compute_zonal_ifunc.py and
lib/modal_base_generator.py), on CPU tensors; tests/test_gpu_modal_basis.py
runs the same on the GPU.

The reference computes in float32 and these functions in float64, and
singular vectors are defined up to sign and, for modes of equal variance, up
to a rotation: singular values are compared within 1e-4 of the largest,
each KL mode by its normalised correlation with the reference's (>= 0.999;
for a degenerate pair the pair's subspace), each mode's RMS against 1 as
test/test_modal_basis.py does, and the m2c columns of separated modes up to
sign within 1e-2."""
import numpy as np
import pytest
import torch

ZONAL = [('sq64', 64, 8, False, False, False, 0.0), ('circ128_slaved', 128, 8, True, False, True, 0.4),
         ('sq32_coupled', 32, 5, False, True, False, 0.0)]
KL = [('sq64', 8.0, 0.2, 25.0, 0, 2), ('circ128_slaved', 8.0, 0.2, 25.0, 5, 1)]


@pytest.fixture(scope='module')
def kl_golden():
    import os
    with np.load(os.path.join(os.path.dirname(__file__), 'golden', 'kl_fp32.npz')) as z:
        return {k: z[k] for k in z.files}


def zonal(name, device):
    from specula_b200.lib.zonal_ifunc import compute_zonal_ifunc
    _, dim, n_act, circ, coup, slav, obs = [c for c in ZONAL if c[0] == name][0]
    return compute_zonal_ifunc(dim, n_act, circ_geom=circ, do_mech_coupling=coup, do_slaving=slav, obsratio=obs,
                               return_coordinates=True, device=device)


def check_zonal(g, name, device):
    f, m, c = zonal(name, device)
    assert f.shape[0] == int(g['zonal/%s/n_act' % name])
    assert np.array_equal(m, g['zonal/%s/mask' % name])
    assert np.allclose(c, g['zonal/%s/coords' % name], rtol=0, atol=1e-12)
    ref = g['zonal/%s/ifs' % name]
    got = f[torch.as_tensor(g['zonal/%s/ifs_index' % name], device=f.device)].double().cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
    return f, m


def check_kl(g, name, device):
    from specula_b200.lib.modal_basis import make_modal_base_from_ifs_fft
    _, diam, r0, L0, nz, ovs = [c for c in KL if c[0] == name][0]
    f, m, _ = zonal(name, device)
    kl, m2c, sv = make_modal_base_from_ifs_fft(m, diam, f, r0, L0, zern_modes=nz, oversampling=ovs)
    key = 'kl/%s' % name
    n = int(g[key + '/n_modes'])
    assert kl.shape[0] == n and m2c.shape == (f.shape[0], n)
    S1, S2 = sv['S1'].cpu().numpy(), sv['S2'].cpu().numpy()
    for ours, ref in ((S1, g[key + '/S1']), (S2, g[key + '/S2'])):
        assert np.abs(ours[:n] - ref[:n]).max() <= 1e-4 * ref.max()
    # the reference's own check: every mode has unit RMS (places=2)
    rms = torch.sqrt(torch.mean(kl.double() ** 2, dim=1)).cpu().numpy()
    assert np.all(np.abs(rms - 1.0) < 5e-3)
    ref_kl = torch.as_tensor(g[key + '/kl_basis'], dtype=torch.float64, device=kl.device)
    k = ref_kl.shape[0]
    a = kl[:k].double()
    a = a / a.norm(dim=1, keepdim=True)
    b = ref_kl / ref_kl.norm(dim=1, keepdim=True)
    ov = (a @ b.t()).cpu().numpy()                 # normalised correlations
    # groups of modes of (nearly) equal variance: the Zernike modes first, then the KL modes by S2
    var = np.concatenate((np.full(nz, np.nan), S2[:n - nz]))[:k]
    i = 0
    while i < k:
        j = i + 1
        while j < k and not np.isnan(var[i]) and abs(var[j] - var[i]) <= 1e-3 * abs(var[i]):
            j += 1
        if j == i + 1:
            assert abs(ov[i, i]) >= 0.999, (name, i, ov[i, i])
            ref_c = g[key + '/m2c'][:, i].astype(np.float64)
            got_c = m2c[:, i].double().cpu().numpy()
            got_c *= np.sign(np.dot(got_c, ref_c)) or 1.0
            assert np.abs(got_c - ref_c).max() <= 1e-2 * np.abs(ref_c).max(), (name, i)
        else:
            blk = ov[i:j, i:j]
            assert np.sum(blk ** 2) >= 0.998 * (j - i), (name, i, j)
        i = j
    return kl, m2c, sv


@pytest.mark.parametrize('name', [c[0] for c in ZONAL])
def test_zonal_ifunc_matches_reference(kl_golden, name):
    check_zonal(kl_golden, name, 'cpu')


@pytest.mark.parametrize('name', [c[0] for c in KL])
def test_kl_basis_matches_reference(kl_golden, name):
    check_kl(kl_golden, name, 'cpu')


def test_ifunc_zonal_type():
    from specula_b200.data_objects.ifunc import IFunc
    from specula_b200.lib.zonal_ifunc import compute_zonal_ifunc
    f = IFunc(type_str='zonal', npixels=64, n_act=8, circ_geom=False, target_device_idx=-1)
    ref, _ = compute_zonal_ifunc(64, 8, circ_geom=False, device='cpu')
    assert torch.equal(f.influence_function.cpu(), ref)
    with pytest.raises(NotImplementedError):
        IFunc(type_str='kl', npixels=64, nmodes=10, target_device_idx=-1)
