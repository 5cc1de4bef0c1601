"""CPU checks of the numpy emulation of the int8 Ozaki GEMM (oracle/ozaki.py), the bit-exact checker of the GPU engine.

The emulation must itself be an FP64-accurate product before it can stand in for one: against the exact product
(long double accumulation of FP64 inputs) it stays within its stated bound K 2^-47 max|row| max|col| for rows scaled
over 2^+-40, it multiplies integer matrices exactly, every slice is an integer in [-64, 64], and the 8 slices
reconstruct each entry to 2^-57 of its row's scale.
"""
import numpy as np
import pytest

from oracle import ozaki


@pytest.mark.parametrize("m,k,n", [(1, 1, 1), (5, 7, 3), (130, 300, 70), (64, 1000, 64)])
def test_emulation_within_bound_of_exact(m, k, n):
    rng = np.random.default_rng(m + k + n)
    a = rng.standard_normal((m, k)) * np.ldexp(1.0, rng.integers(-40, 41, size=(m, 1)))
    b = rng.standard_normal((k, n))
    c = ozaki.gemm(a, b)
    exact = a.astype(np.longdouble) @ b.astype(np.longdouble)
    assert np.all(np.abs(c - exact).astype(np.float64) <= ozaki.error_bound(a, b))


def test_emulation_integer_products_exact():
    rng = np.random.default_rng(1)
    a = rng.integers(-3000, 3000, size=(40, 50)).astype(np.float64)
    b = rng.integers(-3000, 3000, size=(50, 30)).astype(np.float64)
    np.testing.assert_array_equal(ozaki.gemm(a, b), a @ b)


def test_slices_are_small_integers_and_reconstruct():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((20, 33)) * np.ldexp(1.0, rng.integers(-30, 31, size=(20, 1)))
    x[3] = 0.0
    sl, e = ozaki.split_rows(x)
    assert np.all(sl == np.rint(sl)) and np.abs(sl).max() <= 64
    recon = sum(np.ldexp(sl[p], -7 * (p + 1)) for p in range(ozaki.SLICES))
    err = np.abs(np.ldexp(recon, e[:, None]) - x)
    assert np.all(err <= np.ldexp(1.0, e - 57)[:, None])
    assert np.all(sl[:, 3] == 0)


def test_alpha_beta_power_of_two():
    rng = np.random.default_rng(3)
    a, b, c = rng.standard_normal((9, 11)), rng.standard_normal((11, 7)), rng.standard_normal((9, 7))
    np.testing.assert_array_equal(ozaki.gemm(a, b, 1.0, -0.5, c), -0.5 * c + ozaki.gemm(a, b))
