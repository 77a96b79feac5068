"""FITS image I/O and the phase-screen cache (no GPU): round trips checked
with the independent harness reader, a hand-built file with scaling and an
IMAGE extension, the cache file names against the reference's own
(tests/golden/phasescreen_names.json, written by make_golden.py --psnames),
and the cache itself on CPU tensors."""
import json
import os

import numpy as np
import pytest
import torch

from specula_b200.lib import fits_io
from specula_b200.lib.phasescreen_manager import phasescreen_names, phasescreens_manager
from tests.golden import fits_min

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize('dtype', [np.float32, np.float64, np.int16, np.int32, np.uint8])
def test_roundtrip(tmp_path, dtype):
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((37, 53)) * 100).astype(dtype)
    p = str(tmp_path / 'a.fits')
    fits_io.writeto(p, a, header={'VERSION': 1, 'TAG': "it's", 'PITCH': 0.05})
    assert os.path.getsize(p) % 2880 == 0
    b = fits_io.getdata(p)
    assert b.dtype == np.dtype(dtype) and np.array_equal(a, b)
    hdr = fits_io.getheader(p)
    assert hdr['NAXIS1'] == 53 and hdr['NAXIS2'] == 37 and hdr['VERSION'] == 1
    assert hdr['TAG'] == "it's" and hdr['PITCH'] == 0.05
    (h2, d2), = fits_min.read_hdus(p)              # independent reader
    assert np.array_equal(d2, a)
    with pytest.raises(OSError):
        fits_io.writeto(p, a)
    fits_io.writeto(p, a[:3], overwrite=True)
    assert fits_io.getdata(p).shape == (3, 53)


def _card(text):
    return text.ljust(80).encode('ascii')


def _hdu(cards, payload=b''):
    head = b''.join(_card(c) for c in cards) + _card('END')
    head += b' ' * (-len(head) % 2880)
    return head + payload + b'\0' * (-len(payload) % 2880)


def test_hand_built_file_with_scaling_and_extension(tmp_path):
    raw = np.arange(6, dtype='>i2').reshape(2, 3)
    f = _hdu(['SIMPLE  =                    T', 'BITPIX  =                    8', 'NAXIS   =                    0',
              'EXTEND  =                    T'])
    f += _hdu(["XTENSION= 'IMAGE   '           / image extension", 'BITPIX  =                   16',
               'NAXIS   =                    2', 'NAXIS1  =                    3', 'NAXIS2  =                    2',
               'PCOUNT  =                    0', 'GCOUNT  =                    1', 'BSCALE  =                  0.5',
               'BZERO   =                 10.0'], raw.tobytes())
    p = tmp_path / 'h.fits'
    p.write_bytes(f)
    assert fits_io.getdata(str(p)) is None
    d = fits_io.getdata(str(p), ext=1)
    assert np.array_equal(d, np.arange(6).reshape(2, 3) * 0.5 + 10.0)


def test_phasescreen_names_match_reference():
    cases = json.load(open(os.path.join(HERE, 'golden', 'phasescreen_names.json')))
    for c in cases:
        L0 = c['L0']
        for i, s in enumerate(c['seeds']):
            L0i = L0[i] if len(L0) == len(c['seeds']) else L0[0]
            assert phasescreen_names(s, c['dimension'], c['pixel_pitch'], L0i, c['precision'])[0] == c['names'][i]


def test_cache_writes_then_reads(tmp_path):
    d = str(tmp_path / 'screens')
    a = phasescreens_manager([25.0], 64, 0.05, d, precision=1, seed=[1, 2], device='cpu')
    names = sorted(os.listdir(d))
    assert names == sorted(phasescreen_names(s, 64, 0.05, 25.0, 1)[0] for s in (1, 2))
    assert all(x.dtype == torch.float32 and x.shape == (64, 64) for x in a)
    stored = fits_io.getdata(os.path.join(d, names[0]))
    assert stored.dtype == np.float32
    b = phasescreens_manager([25.0], 64, 0.05, d, precision=1, seed=[1, 2], device='cpu')
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    # a file under one of the reference's alternative spellings is found too
    alt = phasescreen_names(5, 64, 0.05, 25.0, 1)[2]
    fits_io.writeto(os.path.join(d, alt), np.full((64, 64), 7.0, np.float32))
    c, = phasescreens_manager([25.0], 64, 0.05, d, precision=1, seed=[5], device='cpu')
    assert float(c[0, 0]) == 7.0
    with pytest.raises(ValueError):
        phasescreens_manager([25.0, 30.0, 40.0], 64, 0.05, d, seed=[1, 2], device='cpu')
