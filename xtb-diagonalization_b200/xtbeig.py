"""Python host binding of libxtbeig.so: the C ABI of include/xtb_eig.h through ctypes.

The names and argument meaning follow the reference's exports (Sources/Diagonalization/Exports.swift:6-138: Fortran
by-reference arguments, column-major arrays, LAPACK semantics) so that callers and tests read like xTB's call sites;
numpy arrays are passed in Fortran order and the in/out arrays are updated in place, as LAPACK does.  Every call runs
on the GPU; if the shared library is missing this module raises instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxtbeig.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "xtb_eig.h")

_lib = None

_I = C.c_int
_P = C.c_void_p


def header_symbols(path: str = HEADER):
    """Function names declared in include/xtb_eig.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xtb_\w+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with xtb-diagonalization_b200/build.py")
        _lib = C.CDLL(LIB_PATH)
        _lib.xtb_gpu_last_error.restype = C.c_char_p
        _lib.xtb_gpu_version.restype = C.c_char_p
        _lib.xtb_gpu_get_option.restype = C.c_long
        _lib.xtb_gpu_set_option.argtypes = [C.c_char_p, C.c_long]
        _lib.xtb_gpu_get_option.argtypes = [C.c_char_p]
        _lib.xtb_dsyevd_device.argtypes = [_I, _P, _I, _P, _P]
        _lib.xtb_dsygvd_device.argtypes = [_I, _P, _I, _P, _I, _P, _P]
        _lib.xtb_dsygvd_density_adjoint.argtypes = [_I, _P, _I, _P, _I, C.c_double, C.c_double, _P, _I, _P, _I, _P,
                                                    _I, _P, _P, _I]
        _lib.xtb_dsygvd_batched.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P]
        _lib.xtb_dsygvd_batched_device.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P]
        _lib.xtb_dsygvd_refine_device.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _I, _P]
        _lib.xtb_gpu_autotune.argtypes = [_I, _I, _P]
        _lib.xtb_dsygvd_density_adjoint_batched.argtypes = [_I] + [_P] * 14
        _lib.xtb_dsygvd_factor_device.argtypes = [_I, _P, _I, _P, _I, _P]
        _lib.xtb_dsygvd_factored_device.argtypes = [_I, _P, _I, _P, _I, _P, _I, _P, _P]
        _lib.xtb_dgemm_device.argtypes = [_I, _I, _I, _I, _I, C.c_double, _P, _I, _P, _I, C.c_double, _P, _I, _P]
        _lib.xtb_gpu_tuned_plan.argtypes = [_I, _I, C.c_char_p, _I]
        _lib.xtb_sgemm_tc_device.argtypes = [_I, _I, _I, _I, _I, C.c_float, _P, _I, _P, _I, C.c_float, _P, _I, _I,
                                             _P]
        _lib.xtb_gpu_stage_name.restype = C.c_char_p
        _lib.xtb_gpu_stage_name.argtypes = [_I]
        _lib.xtb_gpu_stage_ms.restype = C.c_double
        _lib.xtb_gpu_stage_ms.argtypes = [_I]
        _lib.xtb_gpu_launch_count.restype = C.c_longlong
        _lib.xtb_dsygvd_lowest_device.argtypes = [_I, _I, _P, _I, _P, _I, _P, _P]
        _lib.xtb_gpu_scc_set_precision.argtypes = [C.c_double, _I, _I]
        _lib.xtb_gpu_scc_cycle.argtypes = [_I, C.c_double]
        _lib.xtb_gpu_scc_report.argtypes = [_P, _P, _P]
    return _lib


def _ref(v):
    return C.byref(_I(int(v)))


def _p(a):
    return a.ctypes.data_as(_P)


def _f(a, dtype):
    a = np.asarray(a)
    if a.dtype != dtype or not a.flags.f_contiguous:
        raise TypeError(f"expected a Fortran-ordered {np.dtype(dtype).name} array")
    return a


class GPUError(RuntimeError):
    pass


def last_status() -> int:
    return int(lib().xtb_gpu_last_status())


def last_error() -> str:
    return lib().xtb_gpu_last_error().decode()


def _raise_if_failed(name):
    st = last_status()
    if st != 0:
        raise GPUError(f"{name}: {last_error()} (status {st})")


def version() -> str:
    return lib().xtb_gpu_version().decode()


def set_option(name: str, value: int) -> None:
    r = lib().xtb_gpu_set_option(name.encode(), int(value))
    if r == -1:
        raise KeyError(name)
    if r != 0:
        raise ValueError(f"{name}={value} out of range")


def get_option(name: str) -> int:
    return int(lib().xtb_gpu_get_option(name.encode()))


def set_device(device: int) -> None:
    """Select the CUDA device of this thread's later library calls."""
    if lib().xtb_gpu_set_device(int(device)) != 0:
        raise GPUError(last_error())


def stage_times():
    """[(stage, ms)] of the calling thread's last call (with set_option("stage_timing", 1))."""
    L = lib()
    return [(L.xtb_gpu_stage_name(i).decode(), float(L.xtb_gpu_stage_ms(i))) for i in range(L.xtb_gpu_stage_count())]


def scc_set_precision(fp32_rmsq: float, fp32_maxiter: int = 160, fp32_refine: int = 0) -> None:
    """Start an SCC run under the FP32-early / FP64-to-convergence policy of the calling thread
    (xtb_gpu_scc_set_precision; fp32_rmsq 0 turns it off)."""
    rc = lib().xtb_gpu_scc_set_precision(float(fp32_rmsq), int(fp32_maxiter), int(fp32_refine))
    if rc != 0:
        raise ValueError(f"xtb_gpu_scc_set_precision returned {rc}")


def scc_cycle(cycle: int, rmsq: float) -> int:
    """Precision (32 or 64) of this SCC cycle's solves, or 0 when the caller must rerun the SCC in FP64."""
    return int(lib().xtb_gpu_scc_cycle(int(cycle), float(rmsq)))


def scc_report():
    """(policy on, FP32 cycles, restarted, precision in effect) of the calling thread."""
    a, b, c = _I(0), _I(0), _I(0)
    on = lib().xtb_gpu_scc_report(C.byref(a), C.byref(b), C.byref(c))
    return bool(on), a.value, bool(b.value), c.value


def launch_count() -> int:
    """Kernel launches the library has issued so far."""
    return int(lib().xtb_gpu_launch_count())


# ---------------------------------------------------------------------------------------------- xtb sytrd.c ABI

def xtb_dsytrd_upper(n, a, lda, d, e, tau, work=None):
    """call xtb_dsytrd_upper(n, a, lda, d, e, tau, work): in place on a (lda x n), d, e, tau."""
    _f(a, np.float64)
    work = np.zeros(max(1, n * 32)) if work is None else work
    lib().xtb_dsytrd_upper(_ref(n), _p(a), _ref(lda), _p(d), _p(e), _p(tau), _p(work))
    _raise_if_failed("xtb_dsytrd_upper")


def xtb_ssytrd_upper(n, a, lda, d, e, tau, work=None):
    _f(a, np.float32)
    work = np.zeros(max(1, n * 32), np.float32) if work is None else work
    lib().xtb_ssytrd_upper(_ref(n), _p(a), _ref(lda), _p(d), _p(e), _p(tau), _p(work))
    _raise_if_failed("xtb_ssytrd_upper")


def xtb_dsytrd_full(n, a, lda, d, e, tau, work=None):
    _f(a, np.float64)
    work = np.zeros(max(1, n * 32)) if work is None else work
    lib().xtb_dsytrd_full(_ref(n), _p(a), _ref(lda), _p(d), _p(e), _p(tau), _p(work))
    _raise_if_failed("xtb_dsytrd_full")


def xtb_dormtr_upper(n, m, a, lda, tau, z, ldz, work=None):
    _f(z, np.float64)
    work = np.zeros(max(1, 32 * (2 * n + 2 * m + 32))) if work is None else work
    lib().xtb_dormtr_upper(_ref(n), _ref(m), _p(a), _ref(lda), _p(tau), _p(z), _ref(ldz), _p(work))
    _raise_if_failed("xtb_dormtr_upper")


def xtb_sormtr_upper(n, m, a, lda, tau, z, ldz, work=None):
    _f(z, np.float32)
    work = np.zeros(max(1, 32 * (2 * n + 2 * m + 32)), np.float32) if work is None else work
    lib().xtb_sormtr_upper(_ref(n), _ref(m), _p(a), _ref(lda), _p(tau), _p(z), _ref(ldz), _p(work))
    _raise_if_failed("xtb_sormtr_upper")


def xtb_dstedc(n, d, e, z, ldz, work=None, lwork=None, iwork=None, liwork=None) -> int:
    """call xtb_dstedc(n, d, e, z, ldz, work, lwork, iwork, liwork, info); returns info."""
    lwork = 1 + 4 * n + n * n if lwork is None else lwork
    liwork = 3 + 5 * n if liwork is None else liwork
    work = np.zeros(max(1, lwork)) if work is None else work
    iwork = np.zeros(max(1, liwork), np.int32) if iwork is None else iwork
    info = _I(0)
    lib().xtb_dstedc(_ref(n), _p(d), _p(e), _p(z), _ref(ldz), _p(work), _ref(lwork), _p(iwork), _ref(liwork),
                     C.byref(info))
    return info.value


def xtb_sstedc(n, d, e, z, ldz, work=None, lwork=None, iwork=None, liwork=None) -> int:
    lwork = 1 + 4 * n + n * n if lwork is None else lwork
    liwork = 3 + 5 * n if liwork is None else liwork
    work = np.zeros(max(1, lwork), np.float32) if work is None else work
    iwork = np.zeros(max(1, liwork), np.int32) if iwork is None else iwork
    info = _I(0)
    lib().xtb_sstedc(_ref(n), _p(d), _p(e), _p(z), _ref(ldz), _p(work), _ref(lwork), _p(iwork), _ref(liwork),
                     C.byref(info))
    return info.value


def xtb_dsymmetrize_pad(n, src, lds, dst, ldd):
    lib().xtb_dsymmetrize_pad(_ref(n), _p(src), _ref(lds), _p(dst), _ref(ldd))
    _raise_if_failed("xtb_dsymmetrize_pad")


# ---------------------------------------------------------------------------------------------- whole solves

def dsyevd(a, jobz="V", uplo="U"):
    """LAPACK dsyevd on the GPU: returns (w, z or None, info); a is not modified."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    n = a.shape[0]
    w = np.zeros(n)
    info = _I(0)
    lib().xtb_dsyevd_gpu(jobz.encode(), uplo.encode(), _ref(n), _p(a), _ref(max(1, n)), _p(w), None, _ref(1), None,
                         _ref(1), C.byref(info))
    return w, (a if jobz.upper() == "V" else None), info.value


def dsygvd(a, b, jobz="V", uplo="U"):
    """LAPACK dsygvd (itype 1) on the GPU: returns (w, C, factor, info); inputs are not modified."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    b = np.array(b, dtype=np.float64, order="F", copy=True)
    n = a.shape[0]
    w = np.zeros(n)
    info = _I(0)
    lib().xtb_dsygvd_gpu(_ref(1), jobz.encode(), uplo.encode(), _ref(n), _p(a), _ref(max(1, n)), _p(b),
                         _ref(max(1, n)), _p(w), None, _ref(1), None, _ref(1), C.byref(info))
    return w, a, b, info.value


def dsygvd_device(n, a_ptr, lda, b_ptr, ldb, w_ptr, stream=0) -> int:
    """Device-pointer solve (column-major device buffers, e.g. torch tensors' data_ptr())."""
    return int(lib().xtb_dsygvd_device(int(n), _P(a_ptr), int(lda), _P(b_ptr), int(ldb), _P(w_ptr),
                                       _P(stream) if stream else None))


def dsygvd_lowest_device(n, m, a_ptr, lda, b_ptr, ldb, w_ptr, stream=0) -> int:
    """xtb_dsygvd_lowest_device: every eigenvalue and the eigenvectors of the m smallest (device buffers)."""
    return int(lib().xtb_dsygvd_lowest_device(int(n), int(m), _P(a_ptr), int(lda), _P(b_ptr), int(ldb), _P(w_ptr),
                                              _P(stream) if stream else None))


def dsygvd_lowest(h, s, m):
    """Host convenience over xtb_dsygvd_lowest_device (torch moves the arrays): returns (w, C[:, :m], info); m = 0
    means every vector."""
    import torch

    n = np.asarray(h).shape[0]
    dev = torch.device("cuda", torch.cuda.current_device())
    H = torch.from_numpy(np.ascontiguousarray(np.asfortranarray(h, dtype=np.float64).T)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(np.asfortranarray(s, dtype=np.float64).T)).to(dev)
    W = torch.zeros(max(n, 1), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    info = dsygvd_lowest_device(n, m, H.data_ptr(), max(n, 1), S.data_ptr(), max(n, 1), W.data_ptr())
    torch.cuda.synchronize(dev)
    c = H.cpu().numpy().T
    return W.cpu().numpy()[:n], np.asfortranarray(c[:, : (m if m else n)]), info


def dsygvd_refine_device(n, h_ptr, ldh, s_ptr, lds, c_ptr, ldc, w_ptr, iters=2, stream=0) -> int:
    """FP64 refinement of approximate generalized eigenvectors c (device buffers); returns info."""
    return int(lib().xtb_dsygvd_refine_device(int(n), _P(h_ptr), int(ldh), _P(s_ptr), int(lds), _P(c_ptr), int(ldc),
                                              _P(w_ptr), int(iters), _P(stream) if stream else None))


def dsygvd_factor_device(n, b_ptr, ldb, x_ptr, ldx, stream=0) -> int:
    """xtb_dsygvd_factor_device: S = U^T U in place (U in b's upper triangle) and X = U^-1, on device pointers."""
    return lib().xtb_dsygvd_factor_device(n, b_ptr, ldb, x_ptr, ldx, stream)


def dsygvd_factored_device(n, a_ptr, lda, u_ptr, ldu, x_ptr, ldx, w_ptr, stream=0) -> int:
    """xtb_dsygvd_factored_device: the generalized solve with a factorization from dsygvd_factor_device."""
    return lib().xtb_dsygvd_factored_device(n, a_ptr, lda, u_ptr, ldu, x_ptr, ldx, w_ptr, stream)


def dgemm_device(transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, stream=0) -> int:
    """xtb_dgemm_device: FP64 GEMM on device pointers (option "dgemm_engine": 0 DMMA, 1 int8 Ozaki from 512^3 up, the
    default, 2 Ozaki at every size)."""
    return lib().xtb_dgemm_device(transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, stream)


def autotune(n: int, precision: int = 64, stream=0) -> dict:
    """xtb_gpu_autotune: time the candidate plans for size n and keep the fastest; returns the tuned plan."""
    rc = lib().xtb_gpu_autotune(n, precision, stream)
    if rc != 0:
        raise RuntimeError(f"xtb_gpu_autotune({n}, {precision}) returned {rc}: {last_error()}")
    return tuned_plan(n, precision)


def tuned_plan(n: int, precision: int = 64):
    """The tuned plan of (n, precision) as a dict, or None if that size was not tuned."""
    buf = C.create_string_buffer(256)
    if lib().xtb_gpu_tuned_plan(n, precision, buf, 256) < 0:
        return None
    out = {}
    for kv in buf.value.decode().split():
        k, v = kv.split("=")
        out[k] = float(v) if k == "ms" else int(v)
    return out


def sgemm_tc_device(transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, passes=3,
                    stream=0) -> int:
    """xtb_sgemm_tc_device: FP32 GEMM on the tcgen05 tensor cores (3xTF32 or TF32) on device pointers."""
    return lib().xtb_sgemm_tc_device(transa, transb, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc, passes,
                                     stream)


def dsyevd_device(n, a_ptr, lda, w_ptr, stream=0) -> int:
    return int(lib().xtb_dsyevd_device(int(n), _P(a_ptr), int(lda), _P(w_ptr), _P(stream) if stream else None))


def dsygvd_batched(hs, ss):
    """Batch of generalized problems; returns lists (w_i, C_i, U_i), the info array and the call's return value."""
    count = len(hs)
    a = [np.array(h, dtype=np.float64, order="F", copy=True) for h in hs]
    b = [np.array(s, dtype=np.float64, order="F", copy=True) for s in ss]
    ns = np.array([x.shape[0] for x in a], np.int32)
    w = [np.zeros(max(x.shape[0], 1)) for x in a]
    ap = (C.c_void_p * count)(*[x.ctypes.data for x in a])
    bp = (C.c_void_p * count)(*[x.ctypes.data for x in b])
    wp = (C.c_void_p * count)(*[x.ctypes.data for x in w])
    info = np.zeros(count, np.int32)
    ld = np.maximum(ns, 1).astype(np.int32)
    ret = lib().xtb_dsygvd_batched(count, _p(ns), ap, _p(ld), bp, _p(ld), wp, _p(info))
    return [x[:m] for x, m in zip(w, ns)], a, b, info, int(ret)


def dsygvd_batched_device(ns, a_ptrs, ldas, b_ptrs, ldbs, w_ptrs, stream=0):
    """Device-pointer batch: ns, ldas, ldbs int sequences, *_ptrs device addresses.  Returns (info array, ret)."""
    count = len(ns)
    ns = np.asarray(ns, np.int32)
    ldas = np.asarray(ldas, np.int32)
    ldbs = np.asarray(ldbs, np.int32)
    ap = (C.c_void_p * count)(*[int(x) for x in a_ptrs])
    bp = (C.c_void_p * count)(*[int(x) for x in b_ptrs])
    wp = (C.c_void_p * count)(*[int(x) for x in w_ptrs])
    info = np.zeros(count, np.int32)
    ret = lib().xtb_dsygvd_batched_device(count, _p(ns), ap, _p(ldas), bp, _p(ldbs), wp, _p(info),
                                          _P(stream) if stream else None)
    return info, int(ret)


def density_adjoint(h, s, kt, mu, wbar):
    """dL/dH, dL/dS of L = sum(wbar o P), P = C diag(2/(1+exp((e-mu)/kT))) C^T; returns (dH, dS, e, C, info)."""
    h = np.asfortranarray(h, dtype=np.float64)
    s = np.asfortranarray(s, dtype=np.float64)
    wbar = np.asfortranarray(wbar, dtype=np.float64)
    n = h.shape[0]
    dh = np.zeros((n, n), order="F")
    ds = np.zeros((n, n), order="F")
    e = np.zeros(n)
    c = np.zeros((n, n), order="F")
    info = lib().xtb_dsygvd_density_adjoint(n, _p(h), n, _p(s), n, float(kt), float(mu), _p(wbar), n, _p(dh), n,
                                            _p(ds), n, _p(e), _p(c), n)
    return dh, ds, e, c, int(info)


# ---------------------------------------------------------------------------------------------- convenience


def density_adjoint_batched(hs, ss, kts, mus, wbars):
    """xtb_dsygvd_density_adjoint_batched on lists of host arrays: returns (list of dL/dH, list of dL/dS, infos)."""
    count = len(hs)
    hs = [np.asfortranarray(h, dtype=np.float64) for h in hs]
    ss = [np.asfortranarray(s, dtype=np.float64) for s in ss]
    ws = [np.asfortranarray(w, dtype=np.float64) for w in wbars]
    ns = np.array([h.shape[0] for h in hs], np.int32)
    dhs = [np.zeros((m, m), order="F") for m in ns]
    dss = [np.zeros((m, m), order="F") for m in ns]
    arr = lambda xs: (C.c_void_p * count)(*[x.ctypes.data for x in xs])
    kt = np.asarray(kts, np.float64)
    mu = np.asarray(mus, np.float64)
    info = np.zeros(count, np.int32)
    rc = lib().xtb_dsygvd_density_adjoint_batched(count, _p(ns), arr(hs), _p(ns), arr(ss), _p(ns), _p(kt), _p(mu),
                                                  arr(ws), _p(ns), arr(dhs), _p(ns), arr(dss), _p(ns), _p(info))
    if rc < 0:
        raise RuntimeError(f"xtb_dsygvd_density_adjoint_batched returned {rc}: {last_error()}")
    return dhs, dss, info

def sytrd_upper(a, dtype=np.float64):
    """Functional form: returns (A_out, d, e, tau) like oracle.lapack.sytrd_upper."""
    a = np.array(a, dtype=dtype, order="F", copy=True)
    n = a.shape[0]
    d = np.zeros(max(n, 1), dtype)
    e = np.zeros(max(n - 1, 1), dtype)
    tau = np.zeros(max(n - 1, 1), dtype)
    (xtb_dsytrd_upper if dtype == np.float64 else xtb_ssytrd_upper)(n, a, n, d, e, tau)
    return a, d[:n], e[: max(n - 1, 0)], tau[: max(n - 1, 0)]


def stedc(d, e, dtype=np.float64):
    d = np.array(d, dtype=dtype, copy=True)
    n = d.shape[0]
    ee = np.zeros(max(n - 1, 1), dtype)
    ee[: n - 1] = np.asarray(e, dtype)[: n - 1]
    z = np.zeros((n, n), dtype, order="F")
    info = (xtb_dstedc if dtype == np.float64 else xtb_sstedc)(n, d, ee, z, max(n, 1))
    return d, z, info


def ormtr_upper(a, tau, z, dtype=np.float64):
    a = np.array(a, dtype=dtype, order="F", copy=True)
    z = np.array(z, dtype=dtype, order="F", copy=True)
    n, m = z.shape
    tt = np.zeros(max(n - 1, 1), dtype)
    tt[: n - 1] = np.asarray(tau, dtype)[: n - 1]
    (xtb_dormtr_upper if dtype == np.float64 else xtb_sormtr_upper)(n, m, a, n, tt, z, n)
    return z
