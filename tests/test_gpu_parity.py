"""GPU parity of every xtb sytrd.c ABI entry point against the oracle (the reference's LAPACK call chain).

Tolerances (FP64): eigenvalues within 5e-14 * n * ||A||_max of the oracle's; tridiagonal entries within 1e-11 * n *
||A||_max (two Householder reductions of the same matrix agree to rounding, amplified by at most the growth of the
trailing updates); the back-transformation of the oracle's own reflectors within 1e-13 * n; eigenvector residual and
orthogonality at the oracle's level (<= 1e-13 * n).  FP32 entry points: the same checks with 1e-4 scaled bounds.
Sizes cover the reference's edge-case sweep of small and odd n (LOG.md:190-194: n = 3-131) and the panel boundaries
of the reference's blocked code (32, 33, 64, 65).
"""
import numpy as np
import pytest

from oracle import inputs, lapack, metrics

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 7, 16, 17, 31, 32, 33, 64, 65, 100, 131, 257, 412]


def _sym(n, seed):
    return inputs.random_symmetric(n, seed)


@pytest.mark.parametrize("n", SIZES)
def test_dsytrd_upper_matches_lapack(xe, n):
    a = _sym(n, 10 + n)
    ar_ref, d_ref, e_ref, tau_ref = lapack.sytrd_upper(a)
    ar, d, e, tau = xe.sytrd_upper(a)
    scale = np.abs(a).max() * max(n, 1)
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(e, e_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(tau, tau_ref, rtol=0, atol=1e-11 * max(n, 1))
    # reflectors above the superdiagonal, diagonal and superdiagonal in LAPACK layout
    np.testing.assert_allclose(np.triu(ar), np.triu(ar_ref), rtol=0, atol=1e-10 * max(n, 1))
    # strictly lower triangle untouched
    assert np.array_equal(np.tril(ar, -1), np.tril(a, -1))
    # eigenvalues of (d, e) are the matrix's
    w = lapack.stedc(d, e)[0]
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a), rtol=0, atol=5e-14 * scale)


@pytest.mark.parametrize("n", [5, 33, 131])
def test_dsytrd_leading_dimension_padding(xe, n):
    lda = n + 3
    a = _sym(n, 77 + n)
    buf = np.asfortranarray(np.full((lda, n), 7.25))
    buf[:n, :n] = a
    d = np.zeros(n)
    e = np.zeros(max(n - 1, 1))
    tau = np.zeros(max(n - 1, 1))
    xe.xtb_dsytrd_upper(n, buf, lda, d, e, tau)
    assert np.all(buf[n:, :] == 7.25), "rows beyond n (lda padding) must not change"
    _, d_ref, e_ref, _ = lapack.sytrd_upper(a)
    np.testing.assert_allclose(d, d_ref, atol=1e-11 * n * np.abs(a).max())


@pytest.mark.parametrize("n", [3, 33, 100])
def test_dsytrd_full_matches_upper(xe, n):
    a = _sym(n, 5 + n)
    ar, d, e, tau = xe.sytrd_upper(a)
    af = np.asfortranarray(a.copy())
    d2, e2, t2 = np.zeros(n), np.zeros(max(n - 1, 1)), np.zeros(max(n - 1, 1))
    xe.xtb_dsytrd_full(n, af, n, d2, e2, t2)
    np.testing.assert_array_equal(d, d2)
    np.testing.assert_array_equal(e, e2[: n - 1])


@pytest.mark.parametrize("n", [2, 3, 17, 33, 64, 65, 131, 412])
@pytest.mark.parametrize("m_frac", [1.0, 0.5])
def test_dormtr_upper_matches_lapack(xe, n, m_frac):
    a = _sym(n, 200 + n)
    ar, d, e, tau = lapack.sytrd_upper(a)
    m = max(1, int(n * m_frac))
    rng = np.random.default_rng(n)
    z = np.asfortranarray(rng.standard_normal((n, m)))
    z_ref = lapack.ormtr_upper(ar, tau, z)
    z_gpu = xe.ormtr_upper(ar, tau, z)
    np.testing.assert_allclose(z_gpu, z_ref, rtol=0, atol=1e-13 * n * np.abs(z).max())


@pytest.mark.parametrize("n", SIZES)
def test_dstedc_matches_lapack(xe, n):
    d, e = inputs.random_tridiagonal(n, 300 + n)
    w_ref, z_ref, info_ref = lapack.stedc(d, e)
    w, z, info = xe.stedc(d, e)
    assert info == 0 and info_ref == 0
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    scale = max(np.abs(d).max(), np.abs(e).max() if n > 1 else 0.0) * max(n, 1)
    np.testing.assert_allclose(w, w_ref, rtol=0, atol=5e-14 * scale)
    assert np.all(np.diff(w) >= 0)
    dw, res, orth = metrics.eigen_accuracy(t, w_ref, w, z)
    assert res < 1e-13 * max(n, 1)
    assert orth < 1e-13 * max(n, 1)


def test_dstedc_toeplitz_exact(xe):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
    w, z, info = xe.stedc(g["toe25_d"], g["toe25_e"])
    assert info == 0
    np.testing.assert_allclose(w, g["toe25_lam"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("kind", ["zero_offdiag", "diagonal_ties", "split", "glued_wilkinson"])
def test_dstedc_deflation_cases(xe, kind):
    n = 64
    rng = np.random.default_rng(9)
    if kind == "zero_offdiag":
        d, e = rng.uniform(-1, 1, n), np.zeros(n - 1)
    elif kind == "diagonal_ties":
        d, e = np.repeat(np.array([0.5, -0.25, 1.0, 0.0]), n // 4), 1e-9 * rng.uniform(-1, 1, n - 1)
    elif kind == "split":
        d, e = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n - 1)
        e[::7] = 0.0
    else:  # Wilkinson-like W21+ blocks glued by small off-diagonals: pathologically close eigenvalue pairs
        m = 21
        blk = np.abs(np.arange(m) - m // 2).astype(float)
        d = np.tile(blk, 3)[:n] if 3 * m >= n else np.resize(blk, n)
        d = np.resize(blk, n)
        e = np.ones(n - 1)
        e[m - 1::m] = 1e-8
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    w_ref = np.linalg.eigvalsh(t)
    w, z, info = xe.stedc(d, e)
    assert info == 0
    scale = max(np.abs(d).max(), np.abs(e).max(), 1e-300) * n
    np.testing.assert_allclose(w, w_ref, rtol=0, atol=5e-14 * scale)
    _, res, orth = metrics.eigen_accuracy(t, w_ref, w, z)
    assert res < 1e-13 * n and orth < 1e-13 * n


@pytest.mark.parametrize("n", [1, 4, 33, 100])
def test_dsymmetrize_pad_exact(xe, n):
    lds, ldd = n + 2, n + 5
    rng = np.random.default_rng(n)
    src = np.asfortranarray(rng.standard_normal((lds, n)))
    dst = np.asfortranarray(np.full((ldd, n), -3.0))
    xe.xtb_dsymmetrize_pad(n, src, lds, dst, ldd)
    up = np.triu(src[:n, :n])
    np.testing.assert_array_equal(dst[:n, :n], up + np.triu(up, 1).T)
    assert np.all(dst[n:, :] == -3.0)


@pytest.mark.parametrize("n", [3, 33, 100, 257])
def test_fp32_entry_points(xe, n):
    a = _sym(n, 900 + n).astype(np.float32)
    ar_ref, d_ref, e_ref, tau_ref = lapack.sytrd_upper(a, np.float32)
    ar, d, e, tau = xe.sytrd_upper(a, np.float32)
    scale = float(np.abs(a).max()) * n
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=2e-5 * scale)
    np.testing.assert_allclose(e, e_ref, rtol=0, atol=2e-5 * scale)
    w_ref = np.linalg.eigvalsh(a.astype(np.float64))
    w, z, info = xe.stedc(d, e, np.float32)
    assert info == 0
    np.testing.assert_allclose(w, w_ref, rtol=0, atol=1e-5 * scale)
    z2 = xe.ormtr_upper(ar, tau, z, np.float32)
    dw, res, orth = metrics.eigen_accuracy(a.astype(np.float64), w_ref, w, z2)
    assert res < 1e-5 * n and orth < 1e-5 * n


def test_workspace_query(xe):
    n = 10
    work = np.zeros(1)
    iwork = np.zeros(1, np.int32)
    info = xe.xtb_dstedc(n, np.zeros(n), np.zeros(n), np.zeros((n, n), order="F"), n, work, -1, iwork, -1)
    assert info == 0 and work[0] == 1 + 4 * n + n * n and iwork[0] == 3 + 5 * n


def test_repeatable_bits(xe):
    """Same input, same bits (the reference's FNV-1a check of (d, e), Sources/EigenBench/main.swift:253-266)."""
    a = _sym(300, 4)
    h1 = metrics.fnv1a(*xe.sytrd_upper(a)[1:3])
    h2 = metrics.fnv1a(*xe.sytrd_upper(a)[1:3])
    assert h1 == h2
    w1, z1, _ = xe.stedc(*inputs.random_tridiagonal(300, 1))
    w2, z2, _ = xe.stedc(*inputs.random_tridiagonal(300, 1))
    assert np.array_equal(w1, w2) and np.array_equal(z1, z2)


@pytest.fixture(params=[16, 32, 64])
def leaf(xe, request):
    old = xe.get_option("dc_leaf")
    xe.set_option("dc_leaf", request.param)
    yield request.param
    xe.set_option("dc_leaf", old)


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 31, 32, 33, 63, 64, 65, 100, 131, 257, 412, 1204])
def test_dstedc_leaf_solver_matches_lapack(xe, leaf, n):
    """Option "dc_leaf": the subtrees of at most 16 / 32 / 64 are diagonalised directly (Jacobi, one CTA each) and
    the merge levels below them skipped.  Same bars as the 1 x 1 leaves: eigenvalues within 5e-14 n ||T|| of dstedc,
    residual and orthogonality <= 1e-13 n, ascending order."""
    d, e = inputs.random_tridiagonal(n, 700 + n)
    w_ref, _, info_ref = lapack.stedc(d, e)
    w, z, info = xe.stedc(d, e)
    assert info == 0 and info_ref == 0
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    scale = max(np.abs(d).max(), np.abs(e).max() if n > 1 else 0.0) * max(n, 1)
    np.testing.assert_allclose(w, w_ref, rtol=0, atol=5e-14 * scale)
    assert np.all(np.diff(w) >= 0)
    _, res, orth = metrics.eigen_accuracy(t, w_ref, w, z)
    assert res < 1e-13 * max(n, 1) and orth < 1e-13 * max(n, 1)


@pytest.mark.parametrize("kind", ["zero_offdiag", "diagonal_ties", "split", "glued_wilkinson", "toeplitz"])
def test_dstedc_leaf_solver_hard_cases(xe, leaf, kind):
    n = 150
    rng = np.random.default_rng(19)
    if kind == "zero_offdiag":
        d, e = rng.uniform(-1, 1, n), np.zeros(n - 1)
    elif kind == "diagonal_ties":
        d, e = np.repeat(np.array([0.5, -0.25, 1.0, 0.0, 0.5]), n // 5), 1e-9 * rng.uniform(-1, 1, n - 1)
    elif kind == "split":
        d, e = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n - 1)
        e[::7] = 0.0
    elif kind == "glued_wilkinson":
        blk = np.abs(np.arange(21) - 10).astype(float)
        d, e = np.resize(blk, n), np.ones(n - 1)
        e[20::21] = 1e-8
    else:
        d, e = np.full(n, 2.0), np.full(n - 1, -1.0)
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    w_ref = np.linalg.eigvalsh(t)
    w, z, info = xe.stedc(d, e)
    assert info == 0
    scale = max(np.abs(d).max(), np.abs(e).max(), 1e-300) * n
    np.testing.assert_allclose(w, w_ref, rtol=0, atol=5e-14 * scale)
    _, res, orth = metrics.eigen_accuracy(t, w_ref, w, z)
    assert res < 1e-13 * n and orth < 1e-13 * n


@pytest.mark.parametrize("n", [300, 1204])
def test_sygvd_with_leaf_solver(xe, leaf, n):
    h, s, lam = inputs.generalized(n, seed=800 + n)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0
    assert np.max(np.abs(w - lam)) < 1e-10 and np.max(np.abs(w - w_ref)) < 1e-12
    assert metrics.backward_error(h, s, w, c) < 10
    assert metrics.s_orthogonality(s, c) < 1e-12
    assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9


@pytest.mark.parametrize("tail", [128, 64, 0])
@pytest.mark.parametrize("n", [2, 64, 65, 127, 128, 129, 300, 700])
def test_dsytrd_tail_stage(xe, tail, n):
    """Option "sytrd_tail" (default 64): the resident reduction's last columns (every column of a matrix of at most
    that order) run on one CTA in shared memory; the grid kernel hands the trailing block over.  Both sides of the
    hand-over size match LAPACK dsytrd with the sytrd bars; 0 keeps the grid kernel throughout."""
    old = xe.get_option("sytrd_tail")
    xe.set_option("sytrd_tail", tail)
    try:
        a = _sym(n, 700 + n)
        ar_ref, d_ref, e_ref, tau_ref = lapack.sytrd_upper(a)
        ar, d, e, tau = xe.sytrd_upper(a)
    finally:
        xe.set_option("sytrd_tail", old)
    scale = np.abs(a).max() * n
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(e, e_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(tau, tau_ref, rtol=0, atol=1e-11 * n)
    np.testing.assert_allclose(np.triu(ar), np.triu(ar_ref), rtol=0, atol=1e-10 * n)
    assert np.array_equal(np.tril(ar, -1), np.tril(a, -1))
    w = lapack.stedc(d, e)[0]
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a), rtol=0, atol=5e-14 * scale)


@pytest.mark.parametrize("n", [100, 128, 129, 500])
def test_ssytrd_tail_stage(xe, n):
    a = _sym(n, 750 + n).astype(np.float32)
    _, d_ref, e_ref, _ = lapack.sytrd_upper(a, np.float32)
    ar, d, e, tau = xe.sytrd_upper(a, np.float32)
    scale = float(np.abs(a).max()) * n
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=2e-5 * scale)
    np.testing.assert_allclose(e, e_ref, rtol=0, atol=2e-5 * scale)
    w = lapack.stedc(d.astype(np.float64), e.astype(np.float64))[0]
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a.astype(np.float64)), rtol=0, atol=2e-5 * scale)
