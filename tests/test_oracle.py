"""The oracle pinned to known answers and to the golden fixtures (CPU only).

The reference's own check is "every variant against dsyevd on the same matrix" (Sources/EigenBench/main.swift:505-531)
with FP64 eigenvalue errors <= 5.3e-14 on random n = 3-131 (reference LOG.md:190-194).  Here the oracle chain
(dsytrd -> dstedc -> dormtr, and potrf/sygst/trsm for the generalized problem) is checked against spectra that are
exact by construction and against the independent LAPACK drivers dsyevd/dsygvd.
"""
import os

import numpy as np
import pytest

from oracle import fermi, inputs, lapack, metrics

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 33, 64])
def test_sytrd_chain_matches_golden(n):
    a = GOLD[f"sym{n}_a"]
    ar, d, e, tau = lapack.sytrd_upper(a)
    scale = max(1.0, np.abs(a).max())
    np.testing.assert_allclose(d, GOLD[f"sym{n}_d"], rtol=0, atol=1e-12 * scale * n)
    np.testing.assert_allclose(e, GOLD[f"sym{n}_e"], rtol=0, atol=1e-12 * scale * n)
    np.testing.assert_allclose(tau, GOLD[f"sym{n}_tau"], rtol=0, atol=1e-12 * n)
    w, z, info = lapack.stedc(d, e)
    assert info == 0
    np.testing.assert_allclose(w, GOLD[f"sym{n}_evals"], rtol=0, atol=1e-13 * scale * n)


def test_known_spectrum_standard():
    a, lam = GOLD["std48_a"], GOLD["std48_lam"]
    w, z = lapack.syevd_chain(a)
    dw, res, orth = metrics.eigen_accuracy(a, lam, w, z)
    assert dw < 1e-14 and res < 1e-14 and orth < 1e-13


def test_known_spectrum_generalized():
    h, s, lam = GOLD["gen40_h"], GOLD["gen40_s"], GOLD["gen40_lam"]
    w, c = lapack.sygvd_chain(h, s)
    assert np.max(np.abs(w - lam)) < 1e-13
    np.testing.assert_allclose(w, GOLD["gen40_w"], rtol=0, atol=1e-13)
    assert metrics.backward_error(h, s, w, c) < 10
    assert metrics.s_orthogonality(s, c) < 1e-13
    w2, c2, _, info = lapack.sygvd(h, s)
    assert info == 0
    assert metrics.density_error(c, c2, metrics.aufbau(40, 20)) < 1e-12


def test_toeplitz_tridiagonal_exact():
    w, z, info = lapack.stedc(GOLD["toe25_d"], GOLD["toe25_e"])
    assert info == 0
    np.testing.assert_allclose(w, GOLD["toe25_lam"], rtol=0, atol=1e-14)


def test_config_generators_exact_spectra():
    a, lam = inputs.standard(64, seed=0)
    np.testing.assert_allclose(np.linalg.eigvalsh(a), lam, atol=1e-13)
    # the 8-value cluster 1e-6 apart
    cl = np.sort(lam)[(np.abs(np.sort(lam) + 0.25) < 1e-5)]
    assert len(cl) == 8 and np.allclose(np.diff(cl), 1e-6, atol=1e-12)
    h, s, lam = inputs.generalized(64, seed=1)
    assert np.linalg.eigvalsh(s)[0] >= 0.05 - 1e-12
    w = lapack.sygvd(h, s)[0]
    np.testing.assert_allclose(w, lam, atol=1e-13)
    assert lam[32] - lam[31] >= 0.05


def test_batch_sizes_reproducible():
    a = inputs.batch_sizes(256, seed=3)
    b = inputs.batch_sizes(256, seed=3)
    assert a == b and min(a) >= 124 and max(a) <= 1788 and len(a) == 256


def test_fermi_bisection_counts_electrons():
    e = np.linspace(-1, 1, 50)
    mu, f = fermi.fermi_mu(e, 20.0, fermi.kt_of(300.0))
    assert abs(f.sum() - 20.0) < 1e-6
    assert e[19] < mu < e[20]


def test_dk_gradient_matches_finite_differences():
    n = 24
    h, s, lam = inputs.generalized(n, seed=7)
    w, c = lapack.sygvd_chain(h, s)
    mu = 0.5 * (w[n // 2 - 1] + w[n // 2])
    kt = fermi.kt_of(1000.0)
    rng = np.random.default_rng(0)
    wb = rng.standard_normal((n, n))
    wb = wb + wb.T
    gh, gs = fermi.dk_gradient(c, w, wb, mu, kt)

    def loss(hh, ss):
        ww, cc = lapack.sygvd_chain(hh, ss)
        return float(np.sum(wb * fermi.density(cc, ww, mu, kt)))

    step = 1e-6
    for (i, j) in [(0, 0), (3, 5), (10, 2), (n - 1, n - 2)]:
        e = np.zeros((n, n))
        e[i, j] = 1.0
        e[j, i] = 1.0
        mult = 1.0 if i == j else 2.0
        fd_h = (loss(h + step * e, s) - loss(h - step * e, s)) / (2 * step)
        fd_s = (loss(h, s + step * e) - loss(h, s - step * e)) / (2 * step)
        assert abs(fd_h - mult * gh[i, j]) < 1e-6 * max(1.0, abs(fd_h))
        assert abs(fd_s - mult * gs[i, j]) < 1e-6 * max(1.0, abs(fd_s))


def test_divided_differences_near_degenerate_finite():
    e = np.array([-0.1, 0.0, 1e-12, 2e-12, 0.3])
    d1, d2 = fermi.divided_differences(e, 0.0, fermi.kt_of(300.0))
    assert np.all(np.isfinite(d1)) and np.all(np.isfinite(d2))
    # the near-degenerate pairs approach the derivative
    assert abs(d1[1, 2] - d1[1, 1]) < 1e-6 * abs(d1[1, 1])


def test_fnv_hash_stable():
    assert metrics.fnv1a(np.zeros(2)) == metrics.fnv1a(np.zeros(2))
    assert metrics.fnv1a(np.zeros(2)) != metrics.fnv1a(np.ones(2))


def _fp32_start(h, s):
    import scipy.linalg as sla

    w32, c32 = sla.eigh(h.astype(np.float32), s.astype(np.float32))
    return c32.astype(np.float64)


@pytest.mark.parametrize("n", [120, 400])
def test_refine_oracle_from_fp32(n):
    """Two refinement steps from an FP32 solve reach FP64 accuracy (the mixed path's bar)."""
    from oracle import refine

    h, s, lam = inputs.generalized(n, seed=5)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c = refine.refine(h, s, _fp32_start(h, s), iters=2)
    assert np.max(np.abs(w - lam)) < 1e-12
    assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-10
    assert metrics.s_orthogonality(s, c) < 1e-10


def test_refine_oracle_cluster():
    """A cluster of 6 eigenvalues 1e-9 Eh apart: resolved by the exact cluster solve, not by first-order division."""
    from oracle import refine

    n = 90
    rng = np.random.default_rng(11)
    s = inputs.overlap(n, rng)
    lam = np.sort(rng.uniform(-1.0, 0.5, n))
    lam[40:46] = -0.3 + np.arange(6) * 1e-9
    lam = np.sort(lam)
    ws, vs = np.linalg.eigh(s)
    shalf = (vs * np.sqrt(ws)) @ vs.T
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    h = shalf @ (q * lam) @ q.T @ shalf
    h = 0.5 * (h + h.T)
    w, c = refine.refine(h, s, _fp32_start(h, s), iters=2)
    assert np.max(np.abs(w - lam)) < 1e-12
    assert metrics.s_orthogonality(s, c) < 1e-10
    assert metrics.backward_error(h, s, w, c) < 10


def test_bench_inputs_are_the_oracle_inputs():
    """bench.py builds the timed pair itself (both bench arms solve those bytes); they must equal the oracle's."""
    import bench

    for n, seed in ((1, 0), (7, 3), (120, 2)):
        h, s, lam = inputs.generalized(n, seed=seed)
        hb, sb, lb = bench.build_generalized(n, seed)
        np.testing.assert_array_equal(hb, h)
        np.testing.assert_array_equal(sb, s)
        np.testing.assert_array_equal(lb, lam)
    assert bench.bench_config(1788, 2) == bench.bench_config(1788, 2)
