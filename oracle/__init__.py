"""CPU oracle for the KMM channel substep (TEST INFRASTRUCTURE ONLY).

This package is a plain FP64 numpy restatement of the reference solver's hot
path (PoongBack KMM channel DNS with a passive scalar).  It exists only to
check the CUDA implementation: the tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it,
nothing else may.  The product path (``channel_passive_b200``) never imports,
calls or links anything from here and fails loudly when its CUDA library is
missing.

Parity pinning
--------------
* ``bspline``: pinned against the reference's only numerical known-answer test
  (tests/test_bspline.cpp:4-26: n=32, GSL order 7, stretch 0 and 0.99; sum of
  integration weights = 2 within 1e-12, D0 rows sum to 1, D1..D4 rows sum to 0
  within 1e-11 * sum|row|), plus exactness of the derivative operators on
  polynomials of degree < order.
* ``labs``: pinned by solving against dense numpy LU on the same packed
  matrices (the reference's packed-band LU is an exact-arithmetic LU without
  pivoting, module_labs.f90:3487-3636).
* ``kmm``: pinned by analytic known answers (laminar Poiseuille fixed point
  under constant flux, divergence-free output, Hermitian kx=0 plane) because
  the reference ships no trajectory golden (README.md:57-58) and cannot be
  built in this container (no gfortran, MPI, FFTW, GSL, HDF5).  FFTW and GSL
  are not vendored in the reference; the oracle restates their published
  algorithms (unnormalised DFT with FFTW's sign conventions; de Boor B-spline
  recursion with GSL's knot / Greville / Gauss-Legendre conventions).
"""
