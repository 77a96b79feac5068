"""CPU oracle for the closed-loop Shack-Hartmann step — TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy (and SciPy where the reference itself calls
SciPy), the reference's CPU algorithm for every function on the SCAO SH step:
AtmoEvolution shift, AtmoPropagation, SH (edge extrapolation, Interp2D,
field build, FFT, |E|^2, field stop, cut, toccd, photon normalisation), CCD,
ShSlopec, Modalrec, IIR integrator, DM projection and push-pull interaction
matrices.  Each function cites the reference file:line it follows (paths are
relative to the SPECULA project root).

Rules that keep it honest:
  * Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
    ``--impl reference`` legs of ``bench.py`` may import this package, and
    only as the checker or as the timed CPU baseline.  The product package
    ``specula_b200`` never imports it and has no CPU fallback.
  * The oracle is pinned against golden vectors made by running the reference
    itself (``tests/golden/make_golden.py``) and against the reference's own
    committed FITS fixtures (converted by the same script).
"""

from . import masks, sh, ccd, slopec, control, atmo  # noqa: F401
