"""Whole solves on the GPU against the oracle on the benchmark configurations' inputs.

Bars (FP64 path): eigenvalue error <= 1e-10 Eh against the oracle and against the exact spectrum the inputs are built
with; backward error ||HC - SCe|| / (||H|| n eps) <= 10; S-orthogonality <= 1e-12; density matrix (aufbau at the
HOMO/LUMO gap, invariant to signs and to rotations inside degenerate subspaces) within 1e-9 of the oracle's.
"""
import numpy as np
import pytest

from oracle import fermi, inputs, lapack, metrics

pytestmark = pytest.mark.gpu


def test_config1_standard_n412(xe):
    a, lam = inputs.standard(412, seed=0)
    w_ref, z_ref = lapack.syevd_chain(a)
    w, z, info = xe.dsyevd(a)
    assert info == 0
    dw, res, orth = metrics.eigen_accuracy(a, lam, w, z)
    assert dw < 1e-12 and res < 1e-13 and orth < 1e-12
    assert np.max(np.abs(w - w_ref)) < 1e-12
    # the 8-fold cluster (1e-6 apart) resolved
    assert np.all(np.diff(w) > 0)


def test_syevd_lower_and_values_only(xe):
    a, lam = inputs.standard(100, seed=3)
    w, z, info = xe.dsyevd(np.tril(a) + np.triu(np.full_like(a, 9.0), 1), uplo="L")
    assert info == 0
    np.testing.assert_allclose(w, lam, atol=1e-12)
    w2, z2, info2 = xe.dsyevd(a, jobz="N")
    assert info2 == 0 and z2 is None
    np.testing.assert_allclose(w2, lam, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 5, 64, 65, 130, 300])
def test_sygvd_small(xe, n):
    h, s, lam = inputs.generalized(n, seed=20 + n)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0
    assert np.max(np.abs(w - lam)) < 1e-10
    assert np.max(np.abs(w - w_ref)) < 1e-12
    assert metrics.backward_error(h, s, w, c) < 10
    assert metrics.s_orthogonality(s, c) < 1e-12
    u_ref, _ = lapack.potrf_upper(s)
    np.testing.assert_allclose(np.triu(u), u_ref, atol=1e-12)
    np.testing.assert_array_equal(np.tril(u, -1), np.tril(s, -1))
    if n >= 2:
        occ = metrics.aufbau(n, n // 2)
        assert metrics.density_error(c, c_ref, occ) < 1e-9


def test_sygvd_lower(xe):
    n = 90
    h, s, lam = inputs.generalized(n, seed=5)
    w, c, l, info = xe.dsygvd(np.tril(h), np.tril(s), uplo="L")
    assert info == 0
    np.testing.assert_allclose(w, lam, atol=1e-11)
    u_ref, _ = lapack.potrf_upper(s)
    np.testing.assert_allclose(np.tril(l), u_ref.T, atol=1e-12)


@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("n", [90, 300])
def test_sygvd_host_reads_and_returns_one_triangle(xe, uplo, n):
    """The host-pointer dsygvd reads only the triangles uplo names and, as LAPACK, leaves B's other triangle as the
    caller passed it (the transfers move only the referenced triangles): sentinels there change nothing."""
    h, s, lam = inputs.generalized(n, seed=60 + n)
    tri = np.triu if uplo == "U" else np.tril
    other = (lambda x: np.tril(x, -1)) if uplo == "U" else (lambda x: np.triu(x, 1))
    hs = tri(h) + other(np.full_like(h, 7.5))
    ss = tri(s) + other(np.full_like(s, -3.25))
    w, c, f, info = xe.dsygvd(hs, ss, uplo=uplo)
    assert info == 0
    np.testing.assert_allclose(w, lam, atol=1e-11)
    assert metrics.backward_error(h, s, w, c) < 10
    np.testing.assert_array_equal(other(f), other(ss))
    u_ref, _ = lapack.potrf_upper(s)
    np.testing.assert_allclose(tri(f), u_ref if uplo == "U" else u_ref.T, atol=1e-12)


@pytest.mark.parametrize("n", [1100, 1600])
def test_host_solve_matches_device_solve(xe, n):
    """From n = 1024 the host-pointer dsygvd computes C = (X Q) Z in column blocks and copies each to the host while
    the next is formed; the eigenvectors and eigenvalues are bit for bit those of the device-pointer solve."""
    import torch

    h, s, lam = inputs.generalized(n, seed=80 + n)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0
    dev = torch.device("cuda", 0)
    xe.set_device(0)
    H = torch.from_numpy(np.asfortranarray(h).T.copy()).to(dev)  # row-major storage of H^T = H: column-major H
    S = torch.from_numpy(np.asfortranarray(s).T.copy()).to(dev)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    assert xe.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr()) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(W.cpu().numpy(), w)
    np.testing.assert_array_equal(H.cpu().numpy().T, c)


def test_config2_generalized_n1204(xe):
    h, s, lam = inputs.generalized(1204, seed=1)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0
    assert np.max(np.abs(w - w_ref)) <= 1e-10
    assert np.max(np.abs(w - lam)) <= 1e-10
    assert metrics.backward_error(h, s, w, c) < 10
    assert metrics.s_orthogonality(s, c) < 1e-12
    assert metrics.density_error(c, c_ref, metrics.aufbau(1204, 602)) <= 1e-9


def test_not_positive_definite_info(xe):
    n = 70
    h, s, _ = inputs.generalized(n, seed=2)
    s = s.copy()
    s[40, 40] = -1.0
    w, c, u, info = xe.dsygvd(h, s)
    _, info_ref = lapack.potrf_upper(s)
    assert info_ref > 0
    assert info == n + info_ref


def test_invalid_arguments(xe):
    import ctypes

    info = ctypes.c_int(0)
    n = ctypes.c_int(4)
    bad = ctypes.c_int(2)
    one = ctypes.c_int(1)
    buf = np.zeros(16)
    xe.lib().xtb_dsygvd_gpu(ctypes.byref(ctypes.c_int(2)), b"V", b"U", ctypes.byref(n), xe._p(buf),
                            ctypes.byref(n), xe._p(buf), ctypes.byref(n), xe._p(buf), None, ctypes.byref(one), None,
                            ctypes.byref(one), ctypes.byref(info))
    assert info.value == -1
    xe.lib().xtb_dsyevd_gpu(b"V", b"U", ctypes.byref(n), xe._p(buf), ctypes.byref(bad), xe._p(buf), None,
                            ctypes.byref(one), None, ctypes.byref(one), ctypes.byref(info))
    assert info.value == -5


@pytest.mark.parametrize("temp", [300.0, 1000.0])
def test_density_adjoint_matches_dk_oracle(xe, temp):
    n = 96
    h, s, lam = inputs.generalized(n, seed=40)
    kt = fermi.kt_of(temp)
    mu = 0.5 * (lam[n // 2 - 1] + lam[n // 2])
    rng = np.random.default_rng(1)
    wb = rng.standard_normal((n, n))
    wb = wb + wb.T
    dh, ds, e, c, info = xe.density_adjoint(h, s, kt, mu, wb)
    assert info == 0
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    gh, gs = fermi.dk_gradient(c_ref, w_ref, wb, mu, kt)
    scale_h = max(1.0, np.abs(gh).max())
    scale_s = max(1.0, np.abs(gs).max())
    assert np.max(np.abs(dh - gh)) < 1e-9 * scale_h
    assert np.max(np.abs(ds - gs)) < 1e-9 * scale_s


def _batch_problems(sizes, seed0=1000):
    return [inputs.generalized(n, seed=seed0 + i) for i, n in enumerate(sizes)]


@pytest.mark.parametrize("workers", [1, 3, 4])
def test_batched_uneven(xe, workers):
    """Uneven batch (the batch configuration's construction at small sizes, an empty problem included): every
    problem within the FP64 bars, and bit for bit the single-problem call's result whatever the worker count."""
    sizes = [37, 130, 64, 9, 200, 0, 311, 1, 96]
    probs = [inputs.generalized(n, seed=1000 + i) if n else (np.zeros((0, 0)), np.zeros((0, 0)), np.zeros(0))
             for i, n in enumerate(sizes)]
    old = xe.get_option("batch_workers")
    xe.set_option("batch_workers", workers)
    try:
        w, c, u, info, ret = xe.dsygvd_batched([p[0] for p in probs], [p[1] for p in probs])
    finally:
        xe.set_option("batch_workers", old)
    assert ret == 0 and np.all(info == 0)
    for (h, s, lam), wi, ci, ui in zip(probs, w, c, u):
        n = h.shape[0]
        if n == 0:
            continue
        assert np.max(np.abs(wi - lam)) < 1e-10
        assert metrics.backward_error(h, s, wi, ci) < 10
        w1, c1, u1, info1 = xe.dsygvd(h, s)
        assert info1 == 0
        np.testing.assert_array_equal(wi, w1)
        np.testing.assert_array_equal(ci, c1)
        np.testing.assert_array_equal(np.triu(ui), np.triu(u1))


def test_batched_grid_policy(xe):
    """Option "batch_grid" = 1: inside a batch each resident reduction takes the fewest CTAs that hold its rows in
    shared memory (a handful for small problems instead of one per four rows).  Every problem meets the FP64 bars,
    and the result is bit for bit the single-problem call's: the reduction's sums do not depend on its grid."""
    sizes = [37, 130, 64, 200, 311, 96, 640]
    probs = _batch_problems(sizes, seed0=5000)
    old = {k: xe.get_option(k) for k in ("batch_grid", "batch_workers", "precision")}
    try:
        xe.set_option("batch_workers", 4)
        for precision in (64, 32):
            xe.set_option("precision", precision)
            xe.set_option("batch_grid", 1)
            w, c, u, info, ret = xe.dsygvd_batched([p[0] for p in probs], [p[1] for p in probs])
            assert ret == 0 and np.all(info == 0)
            xe.set_option("batch_grid", 0)
            for (h, s, lam), wi, ci in zip(probs, w, c):
                n = h.shape[0]
                assert np.max(np.abs(wi - lam)) < 1e-10
                assert metrics.backward_error(h, s, wi, ci) < 10
                w1, c1, _, info1 = xe.dsygvd(h, s)
                assert info1 == 0
                np.testing.assert_array_equal(wi, w1)
                np.testing.assert_array_equal(ci, c1)
    finally:
        for k, v in old.items():
            xe.set_option(k, v)


def test_batched_failure_is_per_problem(xe):
    """A non-SPD overlap in one problem fails that problem only (info = n + failing column, as dsygvd) and the call
    returns its info; the other problems are solved."""
    sizes = [80, 70, 120]
    probs = _batch_problems(sizes, seed0=2000)
    hs = [p[0] for p in probs]
    ss = [p[1].copy() for p in probs]
    ss[1][40, 40] = -1.0
    _, info_ref = lapack.potrf_upper(ss[1])
    w, c, u, info, ret = xe.dsygvd_batched(hs, ss)
    assert info[1] == 70 + info_ref and info[0] == 0 and info[2] == 0
    assert ret == info[1]
    assert "problem 1" in xe.last_error()
    for i in (0, 2):
        assert np.max(np.abs(w[i] - probs[i][2])) < 1e-10


def test_batched_invalid_arguments(xe):
    import ctypes as C

    lib = xe.lib()
    ns = np.array([10, 5], np.int32)
    lds = np.array([10, 4], np.int32)  # lda < n for problem 1
    a = [np.zeros((10, 10), order="F"), np.zeros((5, 5), order="F")]
    w = [np.zeros(10), np.zeros(5)]
    ap = (C.c_void_p * 2)(*[x.ctypes.data for x in a])
    wp = (C.c_void_p * 2)(*[x.ctypes.data for x in w])
    info = np.zeros(2, np.int32)
    assert lib.xtb_dsygvd_batched(2, ns.ctypes.data, ap, lds.ctypes.data, ap, ns.ctypes.data, wp,
                                  info.ctypes.data) == -2
    assert lib.xtb_dsygvd_batched(-1, ns.ctypes.data, ap, ns.ctypes.data, ap, ns.ctypes.data, wp,
                                  info.ctypes.data) == -1
    assert lib.xtb_dsygvd_batched(0, None, None, None, None, None, None, None) == 0


def test_batched_device_repeated_graph_replay(xe):
    """Device-pointer batch repeated on the same buffers (eager, captured, replayed): each call bit for bit the host
    batch's result, and work queued on the caller's stream before the call (the input restore) is seen."""
    import torch

    sizes = [150, 61, 233, 90, 12]
    probs = _batch_problems(sizes, seed0=3000)
    w_ref, c_ref, u_ref, info_ref, ret = xe.dsygvd_batched([p[0] for p in probs], [p[1] for p in probs])
    assert ret == 0
    dev = torch.device("cuda", 0)
    xe.set_device(0)
    stream = torch.cuda.Stream(dev)
    H0 = [torch.from_numpy(np.ascontiguousarray(p[0])).to(dev) for p in probs]
    S0 = [torch.from_numpy(np.ascontiguousarray(p[1])).to(dev) for p in probs]
    H = [torch.empty_like(x) for x in H0]
    S = [torch.empty_like(x) for x in S0]
    W = [torch.empty(n, dtype=torch.float64, device=dev) for n in sizes]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(4):
            for i in range(len(sizes)):
                H[i].copy_(H0[i])
                S[i].copy_(S0[i])
            info, r = xe.dsygvd_batched_device(sizes, [x.data_ptr() for x in H], sizes, [x.data_ptr() for x in S],
                                               sizes, [x.data_ptr() for x in W], stream.cuda_stream)
            assert r == 0 and np.all(info == 0)
            for i in range(len(sizes)):
                np.testing.assert_array_equal(W[i].cpu().numpy(), w_ref[i])
                np.testing.assert_array_equal(H[i].cpu().numpy().T, c_ref[i])


@pytest.mark.parametrize("graphs", [0, 1])
def test_device_api_repeated_calls_graph_replay(xe, graphs):
    """Device-pointer solves repeated on the same buffers: eager first call, captured second, replayed after; every
    call must give the host entry point's result, bit for bit the same across calls."""
    import torch

    n = 300
    h, s, lam = inputs.generalized(n, seed=77)
    w_ref, c_ref, u_ref, info = xe.dsygvd(h, s)
    assert info == 0
    dev = torch.device("cuda", 0)
    xe.set_device(0)
    stream = torch.cuda.Stream(dev)
    H0 = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    S0 = torch.from_numpy(np.ascontiguousarray(s)).to(dev)
    H, S = torch.empty_like(H0), torch.empty_like(S0)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    old = xe.get_option("graphs")
    xe.set_option("graphs", graphs)
    try:
        outs = []
        with torch.cuda.stream(stream):
            for _ in range(4):
                H.copy_(H0)
                S.copy_(S0)
                assert xe.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream) == 0
                outs.append((W.cpu().numpy().copy(), H.cpu().numpy().T.copy()))
    finally:
        xe.set_option("graphs", old)
    for w, c in outs:
        np.testing.assert_array_equal(w, outs[0][0])
        np.testing.assert_array_equal(c, outs[0][1])
    np.testing.assert_allclose(outs[0][0], w_ref, rtol=0, atol=1e-12)
    assert metrics.density_error(outs[0][1], c_ref, metrics.aufbau(n, n // 2)) < 1e-9


@pytest.mark.parametrize("precision", [64, 32])
def test_backtransform_orders_agree(xe, precision):
    """Option "backtransform": 1 (default) forms X Q beside the tridiagonal eigensolve and finishes with C = (X Q) Z;
    0 applies ormtr to Z and then X.  Both orders meet the bars against the oracle on the same input, and their
    eigenvalues agree to rounding."""
    n = 700
    h, s, lam = inputs.generalized(n, seed=90)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    old = (xe.get_option("backtransform"), xe.get_option("precision"))
    out = {}
    try:
        xe.set_option("precision", precision)
        for order in (0, 1):
            xe.set_option("backtransform", order)
            w, c, u, info = xe.dsygvd(h, s)
            assert info == 0
            assert np.max(np.abs(w - lam)) < 1e-10 and np.max(np.abs(w - w_ref)) < 1e-10
            assert metrics.backward_error(h, s, w, c) < 10
            assert metrics.s_orthogonality(s, c) < (1e-12 if precision == 64 else 1e-9)
            assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9
            out[order] = w
    finally:
        xe.set_option("backtransform", old[0])
        xe.set_option("precision", old[1])
    assert np.max(np.abs(out[0] - out[1])) < 1e-12
