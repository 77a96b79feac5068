"""Minimal FITS image I/O (the subset of astropy.io.fits the SCAO path uses:
``getdata`` and ``writeto`` of one image per file, as in
specula/lib/phasescreen_manager.py:36-48 and
specula/processing_objects/atmo_evolution.py:155).

FITS (NASA/IAU FITS Standard 4.0): a header of 80-character ASCII cards
ending with ``END``, padded with spaces to a multiple of 2880 bytes, then the
image in big-endian order with NAXIS1 the fastest axis, padded with zeros to
a multiple of 2880 bytes.  Reading follows IMAGE extensions (``ext``) and
applies BSCALE / BZERO; writing makes a primary HDU and, with write_hdus,
IMAGE extensions after it.
"""
import os

import numpy as np

BLOCK = 2880
CARD = 80
_BITPIX_DTYPE = {8: '>u1', 16: '>i2', 32: '>i4', 64: '>i8', -32: '>f4', -64: '>f8'}
_DTYPE_BITPIX = {np.dtype(np.uint8): 8, np.dtype(np.int16): 16, np.dtype(np.int32): 32, np.dtype(np.int64): 64,
                 np.dtype(np.float32): -32, np.dtype(np.float64): -64}


def _value(text):
    text = text.split('/')[0].strip() if not text.lstrip().startswith("'") else text.strip()
    if text.startswith("'"):
        end = text.find("'", 1)
        while end != -1 and end + 1 < len(text) and text[end + 1] == "'":   # doubled quote
            end = text.find("'", end + 2)
        return text[1:end].replace("''", "'").rstrip()
    if text in ('T', 'F'):
        return text == 'T'
    try:
        return int(text)
    except ValueError:
        try:
            return float(text.replace('D', 'E'))
        except ValueError:
            return text


def _read_header(f):
    cards = {}
    while True:
        block = f.read(BLOCK)
        if len(block) < BLOCK:
            raise ValueError('FITS: truncated header')
        for k in range(0, BLOCK, CARD):
            card = block[k:k + CARD].decode('ascii', 'replace')
            key = card[:8].strip()
            if key == 'END':
                return cards
            if card[8:10] == '= ':
                cards[key] = _value(card[10:])


def _data_bytes(hdr):
    naxis = int(hdr.get('NAXIS', 0))
    if naxis == 0:
        return 0, ()
    shape = tuple(int(hdr['NAXIS%d' % i]) for i in range(naxis, 0, -1))
    n = int(np.prod(shape)) * abs(int(hdr['BITPIX'])) // 8
    n *= int(hdr.get('GCOUNT', 1))
    n += int(hdr.get('PCOUNT', 0))
    return n, shape


def getheader(path, ext=0):
    with open(path, 'rb') as f:
        for _ in range(ext):
            n, _ = _data_bytes(_read_header(f))
            f.seek((n + BLOCK - 1) // BLOCK * BLOCK, os.SEEK_CUR)
        return _read_header(f)


def getdata(path, ext=0):
    """The image of HDU ``ext`` as a native-endian numpy array (scaled to
    float64 when BSCALE / BZERO are present)."""
    with open(path, 'rb') as f:
        for _ in range(ext):
            n, _ = _data_bytes(_read_header(f))
            f.seek((n + BLOCK - 1) // BLOCK * BLOCK, os.SEEK_CUR)
        hdr = _read_header(f)
        n, shape = _data_bytes(hdr)
        if n == 0:
            return None
        bitpix = int(hdr['BITPIX'])
        if bitpix not in _BITPIX_DTYPE:
            raise ValueError(f'FITS: unsupported BITPIX {bitpix}')
        count = int(np.prod(shape))
        data = np.fromfile(f, dtype=_BITPIX_DTYPE[bitpix], count=count)
        if data.size != count:
            raise ValueError('FITS: truncated data')
    data = data.reshape(shape).astype(data.dtype.newbyteorder('='))
    if 'BSCALE' in hdr or 'BZERO' in hdr:
        data = data * float(hdr.get('BSCALE', 1.0)) + float(hdr.get('BZERO', 0.0))
    return data


def _card(key, value, comment=''):
    if isinstance(value, bool):
        v = ('T' if value else 'F').rjust(20)
    elif isinstance(value, (int, np.integer)):
        v = str(int(value)).rjust(20)
    elif isinstance(value, (float, np.floating)):
        v = repr(float(value)).upper().rjust(20)
    else:
        v = ("'" + str(value).replace("'", "''").ljust(8) + "'").ljust(20)
    text = f'{key:<8}= {v}'
    if comment:
        text += ' / ' + comment
    if len(text) > CARD:
        raise ValueError(f'FITS: card for {key} longer than 80 characters')
    return text.ljust(CARD)


def _hdu_bytes(data, header, primary):
    if data is None:
        a, bitpix, shape = None, 8, ()
    else:
        a = np.asarray(data)
        if a.dtype not in _DTYPE_BITPIX:
            raise ValueError(f'FITS: unsupported dtype {a.dtype}')
        bitpix, shape = _DTYPE_BITPIX[a.dtype], a.shape
    if primary:
        cards = [_card('SIMPLE', True, 'conforms to FITS standard')]
    else:
        cards = [_card('XTENSION', 'IMAGE', 'image extension')]
    cards += [_card('BITPIX', bitpix), _card('NAXIS', len(shape))]
    cards += [_card('NAXIS%d' % (i + 1), n) for i, n in enumerate(reversed(shape))]
    cards += [_card('EXTEND', True)] if primary else [_card('PCOUNT', 0), _card('GCOUNT', 1)]
    for k, v in (header or {}).items():
        if len(k) > 8:
            raise ValueError(f'FITS: keyword {k} longer than 8 characters')
        cards.append(_card(k.upper(), v))
    cards.append('END'.ljust(CARD))
    head = ''.join(cards).encode('ascii')
    head += b' ' * (-len(head) % BLOCK)
    if a is None:
        return head
    body = np.ascontiguousarray(a).astype(a.dtype.newbyteorder('>'), copy=False).tobytes()
    return head + body + b'\0' * (-len(body) % BLOCK)


def write_hdus(path, hdus, overwrite=False):
    """Write [(data or None, header dict), ...]: the first as the primary HDU,
    the others as IMAGE extensions."""
    if os.path.exists(path) and not overwrite:
        raise OSError(f'FITS: {path} exists')
    tmp = path + '.tmp'
    with open(tmp, 'wb') as f:
        for k, (data, header) in enumerate(hdus):
            f.write(_hdu_bytes(data, header, primary=(k == 0)))
    os.replace(tmp, path)


def writeto(path, data, header=None, overwrite=False):
    """Write ``data`` as the primary image of a new FITS file; ``header``:
    extra (key, value) cards (keys of at most 8 characters)."""
    write_hdus(path, [(data, header)], overwrite=overwrite)
