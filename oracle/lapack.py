"""The reference's LAPACK call chain on the CPU, through ctypes (TEST INFRASTRUCTURE ONLY: the oracle).

The reference's eigensolve is LAPACK's: xTB's SCC cycle calls potrf once per geometry, then per cycle dsygst (or the
congruence H' = X^T H X), dsytrd, dstedc, dormtr and dtrsm (xTB's eigensolve call stack;
Sources/Diagonalization/Exports.swift:6-115 replaces sytrd/stedc/ormtr with Swift ports of the same LAPACK semantics;
CLAPACK.h:9-105 lists the routines).
The reference's own Swift/Accelerate code cannot be built here (no Swift toolchain, Accelerate is macOS only, the xtb
submodule holding sytrd.c is empty).  This module therefore binds the identical LAPACK routines from OpenBLAS 0.3.30,
the copy that ships with scipy 1.18.1 (exported as ``scipy_<name>_``; Fortran calling convention: every argument by
reference, 32-bit integers, hidden string lengths appended).

Every function takes and returns numpy arrays in Fortran (column-major) order, mirroring the LAPACK argument meaning.
"""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

_lib = None


def _load():
    global _lib
    if _lib is None:
        import scipy  # noqa: F401  (locates scipy.libs)
        base = os.path.dirname(os.path.dirname(scipy.__file__))
        cands = sorted(glob.glob(os.path.join(base, "scipy.libs", "libscipy_openblas*.so")))
        if not cands:
            raise RuntimeError("OpenBLAS from scipy.libs not found; the oracle needs it")
        _lib = C.CDLL(cands[0])
    return _lib


def _fn(name):
    return getattr(_load(), "scipy_" + name + "_")


_I = C.c_int
_D = C.c_double
_P = C.c_void_p
_L = C.c_size_t


def _ip(x):
    return C.byref(_I(int(x)))


def _dp(x):
    return C.byref(_D(float(x)))


def _sp(x):
    return C.byref(C.c_float(float(x)))


def _ptr(a):
    return a.ctypes.data_as(_P)


def _ch(s):
    return C.c_char_p(s.encode())


def set_threads(n: int) -> None:
    """openblas_set_num_threads for the oracle's BLAS (used by the timed CPU baseline)."""
    getattr(_load(), "scipy_openblas_set_num_threads")(C.c_int(int(n)))


def get_threads() -> int:
    return int(getattr(_load(), "scipy_openblas_get_num_threads")())


def _fa(a, dtype):
    return np.asfortranarray(np.array(a, dtype=dtype, copy=True))


# --------------------------------------------------------------------------------------------------------------------
# xsytrd (UPLO='U'): A -> reflectors above the superdiagonal, d, e, tau.  Same contract as xtb_dsytrd_upper
# (Exports.swift:8-16) and xtb_ssytrd_upper (:19-27).

def sytrd_upper(a, dtype=np.float64):
    a = _fa(a, dtype)
    n = a.shape[0]
    d = np.zeros(max(n, 1), dtype)
    e = np.zeros(max(n - 1, 1), dtype)
    tau = np.zeros(max(n - 1, 1), dtype)
    lwork = max(1, n * 64)
    work = np.zeros(lwork, dtype)
    info = _I(0)
    f = _fn("dsytrd" if dtype == np.float64 else "ssytrd")
    f(_ch("U"), _ip(n), _ptr(a), _ip(n), _ptr(d), _ptr(e), _ptr(tau), _ptr(work), _ip(lwork), C.byref(info), _L(1))
    assert info.value == 0, info.value
    return a, d[:n], e[: max(n - 1, 0)], tau[: max(n - 1, 0)]


# xstedc (COMPZ='I'): eigenpairs of the symmetric tridiagonal (d, e).  Contract of xtb_dstedc (Exports.swift:88-101).

def stedc(d, e, dtype=np.float64):
    d = np.array(d, dtype=dtype, copy=True)
    n = d.shape[0]
    ee = np.zeros(max(n - 1, 1), dtype)
    ee[: n - 1] = np.asarray(e, dtype)[: n - 1]
    z = np.zeros((n, n), dtype, order="F")
    lwork = 1 + 4 * n + n * n
    liwork = 3 + 5 * n
    work = np.zeros(lwork, dtype)
    iwork = np.zeros(liwork, np.int32)
    info = _I(0)
    f = _fn("dstedc" if dtype == np.float64 else "sstedc")
    f(_ch("I"), _ip(n), _ptr(d), _ptr(ee), _ptr(z), _ip(max(n, 1)), _ptr(work), _ip(lwork), _ptr(iwork),
      _ip(liwork), C.byref(info), _L(1))
    return d, z, info.value


# xormtr ('L', 'U', 'N'): z = Q z with Q from sytrd_upper.  Contract of xtb_dormtr_upper (Exports.swift:56-65).

def ormtr_upper(a, tau, z, dtype=np.float64):
    a = _fa(a, dtype)
    z = _fa(z, dtype)
    n, m = z.shape
    tt = np.zeros(max(n - 1, 1), dtype)
    tt[: n - 1] = np.asarray(tau, dtype)[: n - 1]
    lwork = max(1, m * 64)
    work = np.zeros(lwork, dtype)
    info = _I(0)
    f = _fn("dormtr" if dtype == np.float64 else "sormtr")
    f(_ch("L"), _ch("U"), _ch("N"), _ip(n), _ip(m), _ptr(a), _ip(n), _ptr(tt), _ptr(z), _ip(n), _ptr(work),
      _ip(lwork), C.byref(info), _L(1), _L(1), _L(1))
    assert info.value == 0, info.value
    return z


def potrf_upper(s):
    """dpotrf('U'): S = U^T U.  Returns (U with the strictly lower part zeroed, info)."""
    s = _fa(s, np.float64)
    n = s.shape[0]
    info = _I(0)
    _fn("dpotrf")(_ch("U"), _ip(n), _ptr(s), _ip(n), C.byref(info), _L(1))
    return np.triu(s), info.value


def sygst_upper(h, u):
    """dsygst(itype=1, 'U'): upper triangle of U^-T H U^-1 (returned symmetrised)."""
    h = _fa(h, np.float64)
    u = _fa(u, np.float64)
    n = h.shape[0]
    info = _I(0)
    _fn("dsygst")(_ip(1), _ch("U"), _ip(n), _ptr(h), _ip(n), _ptr(u), _ip(n), C.byref(info), _L(1))
    assert info.value == 0, info.value
    up = np.triu(h)
    return up + np.triu(up, 1).T


def trsm_upper_left(u, c):
    """dtrsm('L', 'U', 'N', 'N'): C = U^-1 C (back-transformation to the generalized basis)."""
    u = _fa(u, np.float64)
    c = _fa(c, np.float64)
    n, m = c.shape
    _fn("dtrsm")(_ch("L"), _ch("U"), _ch("N"), _ch("N"), _ip(n), _ip(m), _dp(1.0), _ptr(u), _ip(n), _ptr(c),
                 _ip(n), _L(1), _L(1), _L(1), _L(1))
    return c


def syevd(a, dtype=np.float64):
    """xsyevd('V', 'U'): the independent LAPACK driver (the reference's EigenBench pins every variant to it,
    Sources/EigenBench/main.swift:505-531)."""
    a = _fa(a, dtype)
    n = a.shape[0]
    w = np.zeros(n, dtype)
    lwork = 1 + 6 * n + 2 * n * n
    liwork = 3 + 5 * n
    work = np.zeros(lwork, dtype)
    iwork = np.zeros(liwork, np.int32)
    info = _I(0)
    f = _fn("dsyevd" if dtype == np.float64 else "ssyevd")
    f(_ch("V"), _ch("U"), _ip(n), _ptr(a), _ip(n), _ptr(w), _ptr(work), _ip(lwork), _ptr(iwork), _ip(liwork),
      C.byref(info), _L(1), _L(1))
    assert info.value == 0, info.value
    return w, a


def sygvd(h, s):
    """dsygvd(itype=1, 'V', 'U'): H C = S C diag(w), C^T S C = I."""
    a = _fa(h, np.float64)
    b = _fa(s, np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    lwork = 1 + 6 * n + 2 * n * n
    liwork = 3 + 5 * n
    work = np.zeros(lwork)
    iwork = np.zeros(liwork, np.int32)
    info = _I(0)
    _fn("dsygvd")(_ip(1), _ch("V"), _ch("U"), _ip(n), _ptr(a), _ip(n), _ptr(b), _ip(n), _ptr(w), _ptr(work),
                  _ip(lwork), _ptr(iwork), _ip(liwork), C.byref(info), _L(1), _L(1))
    return w, a, np.triu(b), info.value


# --------------------------------------------------------------------------------------------------------------------
# The full chains, stage by stage, as the reference's SCC eigensolve runs them (potrf, sygst, sytrd, stedc, ormtr, trsm).

def syevd_chain(a):
    """Standard problem: dsytrd -> dstedc -> dormtr (config: n=412, all eigenpairs)."""
    ar, d, e, tau = sytrd_upper(a)
    w, z, info = stedc(d, e)
    assert info == 0, info
    z = ormtr_upper(ar, tau, z)
    return w, z


def sygvd_chain(h, s):
    """Generalized problem: dpotrf -> dsygst -> dsytrd -> dstedc -> dormtr -> dtrsm."""
    u, info = potrf_upper(s)
    assert info == 0, info
    hp = sygst_upper(h, u)
    w, z = syevd_chain(hp)
    c = trsm_upper_left(u, z)
    return w, c
