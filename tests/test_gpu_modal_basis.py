"""Zonal influence functions and the KL basis computed on the GPU (cuSOLVER
SVD / QR / solves and cuFFT through torch, float64) against the reference's
outputs, with the checks and tolerances of tests/test_modal_basis.py."""
import pytest

from tests.test_modal_basis import KL, ZONAL, check_kl, check_zonal, kl_golden  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name', [c[0] for c in ZONAL])
def test_zonal_ifunc_on_gpu(cuda, kl_golden, name):  # noqa: F811
    check_zonal(kl_golden, name, 'cuda')


@pytest.mark.parametrize('name', [c[0] for c in KL])
def test_kl_basis_on_gpu(cuda, kl_golden, name):  # noqa: F811
    check_kl(kl_golden, name, 'cuda')
