"""Minimal FITS image reader (primary HDU + IMAGE extensions), harness only.

FITS = 2880-byte blocks; each header is 80-character cards up to ``END``;
image data is big-endian with NAXIS1 the fastest axis.  Enough to read the
reference's test/data fixtures without astropy.
"""
import numpy as np

_BLOCK = 2880
_DT = {8: '>u1', 16: '>i2', 32: '>i4', 64: '>i8', -32: '>f4', -64: '>f8'}


def _parse_header(buf, pos):
    cards = {}
    while True:
        block = buf[pos:pos + _BLOCK]
        if len(block) < _BLOCK:
            raise ValueError('truncated FITS header')
        pos += _BLOCK
        for k in range(0, _BLOCK, 80):
            card = block[k:k + 80].decode('ascii', 'replace')
            key = card[:8].strip()
            if key == 'END':
                return cards, pos
            if card[8:10] == '= ':
                val = card[10:].split('/')[0].strip()
                if val.startswith("'"):
                    val = val.strip("'").strip()
                elif val in ('T', 'F'):
                    val = val == 'T'
                else:
                    try:
                        val = int(val)
                    except ValueError:
                        try:
                            val = float(val.replace('D', 'E'))
                        except ValueError:
                            pass
                cards[key] = val


def read_hdus(path):
    """List of (header dict, numpy array or None) for every HDU."""
    buf = open(path, 'rb').read()
    pos = 0
    out = []
    while pos < len(buf):
        hdr, pos = _parse_header(buf, pos)
        naxis = hdr.get('NAXIS', 0)
        shape = tuple(hdr['NAXIS%d' % i] for i in range(naxis, 0, -1))
        n = int(np.prod(shape)) if naxis else 0
        bitpix = hdr['BITPIX']
        nbytes = n * abs(bitpix) // 8
        data = None
        if n:
            data = np.frombuffer(buf[pos:pos + nbytes], dtype=_DT[bitpix]).reshape(shape)
            data = data.astype(data.dtype.newbyteorder('='))
            if 'BSCALE' in hdr or 'BZERO' in hdr:
                data = data * hdr.get('BSCALE', 1) + hdr.get('BZERO', 0)
        pos += (nbytes + _BLOCK - 1) // _BLOCK * _BLOCK
        out.append((hdr, data))
    return out
