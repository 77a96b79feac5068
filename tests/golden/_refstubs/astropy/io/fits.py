"""Minimal in-memory FITS stand-in for importing the reference (harness only).

writeto/append keep arrays in a process-local dict keyed by file name, so
reference objects that save and restore calibration products inside one
golden-generation run still work. Nothing is written to disk.
"""
import numpy as np

_store = {}


class Header(dict):
    def append(self, card):
        k, v = card[:2]
        self[k] = v

    def update(self, other=None, **kw):
        if other:
            dict.update(self, other)
        dict.update(self, kw)


class _HDU:
    def __init__(self, data=None, header=None, name=None):
        self.data = None if data is None else np.array(data)
        self.header = Header(header or {})
        self.name = name


PrimaryHDU = _HDU
ImageHDU = _HDU


class HDUList(list):
    def writeto(self, filename, overwrite=False):
        _store[str(filename)] = [(_h.data, _h.header) for _h in self]

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def flush(self):
        pass


def writeto(filename, data, header=None, overwrite=False):
    _store[str(filename)] = [(np.array(data), Header(header or {}))]


def append(filename, data, header=None):
    _store.setdefault(str(filename), []).append((np.array(data), Header(header or {})))


def open(filename, mode='readonly', **kw):
    hl = HDUList()
    for d, h in _store[str(filename)]:
        hl.append(_HDU(d, h))
    return hl


def getdata(filename, ext=0, **kw):
    return _store[str(filename)][ext][0]


def getheader(filename, ext=0, **kw):
    return _store[str(filename)][ext][1]
