"""GPU checks of the per-geometry / per-cycle split (xtb_dsygvd_factor_device + xtb_dsygvd_factored_device).

xTB factors S once per geometry and solves a new H every SCC cycle.  Checked: the factored solve gives the same
eigenpairs as the full device solve on the same inputs (bit for bit: the same kernels run on the same U and X), for
FP64 and mixed precision; one factorization serves several H (each against the oracle with the FP64 path's bars:
eigenvalues within 1e-10 Eh, backward error <= 10, S-orthogonality <= 1e-12, density within 1e-9); U matches LAPACK's
dpotrf and the strict lower triangle of S is left untouched; a non-SPD S reports info = n + i.
"""
import numpy as np
import pytest

from oracle import inputs, lapack, metrics

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch

    # column-major n x n data: the transpose of a row-major view
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).to(torch.device("cuda", 0))


def _host(t):
    return t.cpu().numpy().T


@pytest.fixture
def prec(xe):
    old = xe.get_option("precision")
    yield xe
    xe.set_option("precision", old)


@pytest.mark.parametrize("precision", [64, 32])
def test_factored_equals_full_solve(prec, precision):
    import torch

    xe = prec
    xe.set_device(0)
    xe.set_option("precision", precision)
    n = 257
    h, s, lam = inputs.generalized(n, seed=111)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    # full solve
    A, B = _dev(h), _dev(s)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    assert xe.dsygvd_device(n, A.data_ptr(), n, B.data_ptr(), n, W.data_ptr(), stream.cuda_stream) == 0
    torch.cuda.synchronize(dev)
    # factor + factored solve
    A2, B2 = _dev(h), _dev(s)
    X = torch.empty((n, n), dtype=torch.float64, device=dev)
    W2 = torch.empty(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    assert xe.dsygvd_factor_device(n, B2.data_ptr(), n, X.data_ptr(), n, stream.cuda_stream) == 0
    assert xe.dsygvd_factored_device(n, A2.data_ptr(), n, B2.data_ptr(), n, X.data_ptr(), n, W2.data_ptr(),
                                     stream.cuda_stream) == 0
    torch.cuda.synchronize(dev)
    assert torch.equal(W, W2)
    assert torch.equal(A, A2)
    assert torch.equal(torch.triu(B.T), torch.triu(B2.T))


def test_one_factorization_many_cycles(prec):
    import torch

    xe = prec
    xe.set_device(0)
    xe.set_option("precision", 64)
    n = 300
    h, s, lam = inputs.generalized(n, seed=112)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    B = _dev(s)
    X = torch.empty((n, n), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    assert xe.dsygvd_factor_device(n, B.data_ptr(), n, X.data_ptr(), n, stream.cuda_stream) == 0
    torch.cuda.synchronize(dev)
    u = _host(B)
    u_ref, _ = lapack.potrf_upper(s)
    np.testing.assert_allclose(np.triu(u), u_ref, atol=1e-12)
    np.testing.assert_array_equal(np.tril(u, -1), np.tril(s, -1))
    rng = np.random.default_rng(5)
    for cycle in range(3):
        d = rng.standard_normal((n, n)) * 1e-3
        hc = h + (d + d.T) / 2
        w_ref, c_ref = lapack.sygvd_chain(hc, s)
        A = _dev(hc)
        W = torch.empty(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        assert xe.dsygvd_factored_device(n, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n, W.data_ptr(),
                                         stream.cuda_stream) == 0
        torch.cuda.synchronize(dev)
        w, c = W.cpu().numpy(), _host(A)
        assert np.max(np.abs(w - w_ref)) < 1e-10
        assert metrics.backward_error(hc, s, w, c) < 10
        assert metrics.s_orthogonality(s, c) < 1e-12
        assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9


def test_factor_not_positive_definite(prec):
    import torch

    xe = prec
    xe.set_device(0)
    n = 40
    _, s, _ = inputs.generalized(n, seed=113)
    s = s.copy()
    s[7, 7] = -1.0
    B = _dev(s)
    X = torch.empty((n, n), dtype=torch.float64, device=torch.device("cuda", 0))
    torch.cuda.synchronize()
    info = xe.dsygvd_factor_device(n, B.data_ptr(), n, X.data_ptr(), n, 0)
    assert info == n + 8, info
