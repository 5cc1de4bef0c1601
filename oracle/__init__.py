"""CPU oracle for the dense symmetric / generalized eigensolve (TEST INFRASTRUCTURE ONLY).

Nothing in the product library imports this package.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` use it, and only as the checker or as the timed CPU
baseline, never as the thing measured or shipped.

Contents
--------
``lapack``   ctypes bindings to the LAPACK call chain the reference makes (dpotrf, dsygst, dsytrd, dstedc, dormtr,
             dtrsm, plus dsyevd/dsygvd as independent drivers).  The reference links Apple Accelerate
             (Sources/CLAPACK/include/CLAPACK.h:9-105); here the same routines come from OpenBLAS 0.3.30 as bundled
             with scipy 1.18.1 (``scipy.libs/libscipy_openblas-*.so``, symbols ``scipy_d*_``).
``inputs``   seeded generators for the five benchmark configurations (standard n=412, generalized n=1204/1788,
             the uneven 124-1788 batch, the n=588 density/adjoint batch).
``metrics``  the accuracy measures of the reference's EigenBench (Sources/EigenBench/main.swift:231-251) plus the
             generalized backward error, S-orthogonality and the rotation-invariant density-matrix error.
``fermi``    Fermi occupations and the density matrix (scripts/kernels/refine.f90:85-132) and an FP64
             Daleckii-Krein gradient of the Fermi-smeared density (no reference counterpart).
"""
