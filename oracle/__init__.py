"""CPU FP64 oracle for the DIABLO 3 channel step (test infrastructure only).

This package is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it.
It restates the reference Fortran (``for/fft.f90``, ``for/channel.f90``,
``for/boundary.f90``, ``for/domain.f90``, ``for/flow.f90``, ``for/advance.f90``,
``for/les.f90``) in numpy, loop nest by loop nest, on arrays in the
reference's own memory layout.

Parity status: the reference Fortran cannot be built here (no gfortran, MPI,
FFTW, HDF5 or toml-f) and ships no tests or fixtures, so the solver restatement
is "parity unpinned" against the Fortran itself.  It is pinned instead by the
analytic known-answer tests in ``tests/test_oracle_kat.py`` and, for the
wall-normal grid, by golden vectors produced by the reference's own Python
grid tool (``tests/golden/make_golden.py``).
"""
