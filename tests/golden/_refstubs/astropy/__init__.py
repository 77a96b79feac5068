"""Harness-only stand-in for astropy (absent from this image).

Only used by tests/golden/make_golden.py to import the reference package on
CPU. It implements the tiny subset of astropy.io.fits that the reference's
module-level imports and the objects driven by the golden script touch.
"""
