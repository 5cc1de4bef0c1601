"""GPU checks of the FP64 GEMM from int8 tcgen05 products (option "dgemm_engine" = 2 of xtb_dgemm_device: Ozaki at
every size; the default 1 takes it from 512^3 up).

  - bit for bit against the numpy emulation of the same splitting (oracle/ozaki.py) for every transpose combination,
    ragged sizes (M, N not multiples of the 128 x 64 tile, K not a multiple of the 64-deep K block), padded leading
    dimensions, alpha and a power-of-two beta, and rows scaled over 2^+-40;
  - against the exact product (long double) within the engine's bound K 2^-47 max|row| max|col|, and at least as
    close as the FP64 DMMA engine's bound 2 K eps |op(A)| |op(B)| on the same data;
  - integer data is multiplied exactly; k = 0 gives beta C; a row holding a NaN or an Inf gives NaN in its row;
    K above 65000 is refused (the int32 accumulators' exactness bound);
  - at n = 1788 against torch's FP64 product;
  - generalized solves whose large GEMMs (congruence, back-transform, refinement) run on the engine meet the FP64
    path's bars against the LAPACK oracle (eigenvalues within 1e-10 Eh, density within 1e-9), in FP64 and mixed
    precision.
"""
import numpy as np
import pytest

from oracle import inputs, lapack, metrics, ozaki

pytestmark = pytest.mark.gpu


@pytest.fixture
def oz(xe):
    old = xe.get_option("dgemm_engine")
    xe.set_option("dgemm_engine", 2)
    yield xe
    xe.set_option("dgemm_engine", old)


def _mats(m, n, k, ta, tb, seed, scale_rows=0.0, pad=0):
    rng = np.random.default_rng(seed)
    opa = rng.standard_normal((m, k))
    if scale_rows:
        opa *= np.ldexp(1.0, rng.integers(-int(scale_rows), int(scale_rows) + 1, size=(m, 1)))
    opb = rng.standard_normal((k, n))
    c = rng.standard_normal((m, n))
    return opa, opb, c


def _run(xe, opa, opb, c, ta, tb, alpha, beta, pad=0):
    """Store op(A), op(B) as the transposes ask (column-major, leading dimension + pad), run xtb_dgemm_device."""
    import torch

    dev = torch.device("cuda", 0)
    m, k = opa.shape
    n = opb.shape[1]

    def store(x):  # column-major x with ld = max(rows, 1) + pad
        r, cc = x.shape
        ld = max(r, 1) + pad
        buf = torch.full((max(cc, 1), ld), 7.0, dtype=torch.float64)
        buf[:cc, :r] = torch.from_numpy(np.ascontiguousarray(x.T))
        return buf.to(dev), ld

    A, lda = store(opa.T if ta else opa)
    B, ldb = store(opb.T if tb else opb)
    C, ldc = store(c)
    torch.cuda.synchronize(dev)
    rc = xe.dgemm_device(ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta, C.data_ptr(), ldc, 0)
    torch.cuda.synchronize(dev)
    assert rc == 0, (rc, xe.last_error())
    out = C.cpu().numpy()
    assert np.all(out[:, m:] == 7.0)  # padding untouched
    return out[:n, :m].T


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (130, 70, 33), (257, 129, 300), (64, 192, 128), (300, 260, 1000)])
def test_ozaki_bit_exact_against_emulation(oz, ta, tb, mnk):
    m, n, k = mnk
    opa, opb, c = _mats(m, n, k, ta, tb, seed=m + 3 * n + 7 * k + ta + 2 * tb, scale_rows=40)
    out = _run(oz, opa, opb, c, ta, tb, 1.25, -0.5, pad=3)
    ref = ozaki.gemm(opa, opb, 1.25, -0.5, c)
    np.testing.assert_array_equal(out, ref)


@pytest.mark.parametrize("mnk", [(200, 180, 256), (129, 65, 777)])
def test_ozaki_accuracy_against_exact(oz, mnk):
    m, n, k = mnk
    opa, opb, _ = _mats(m, n, k, 0, 0, seed=11 + k)
    out = _run(oz, opa, opb, np.zeros((m, n)), 0, 0, 1.0, 0.0)
    exact = opa.astype(np.longdouble) @ opb.astype(np.longdouble)
    err = np.abs(out - exact).astype(np.float64)
    assert np.all(err <= ozaki.error_bound(opa, opb))
    dmma_bound = 2 * k * 2.0 ** -53 * (np.abs(opa) @ np.abs(opb))
    assert np.all(err <= dmma_bound)


def test_ozaki_integer_data_is_exact(oz):
    rng = np.random.default_rng(5)
    opa = rng.integers(-2000, 2000, size=(150, 300)).astype(np.float64)
    opb = rng.integers(-2000, 2000, size=(300, 90)).astype(np.float64)
    out = _run(oz, opa, opb, np.zeros((150, 90)), 0, 1, 1.0, 0.0)
    np.testing.assert_array_equal(out, opa @ opb)


def test_ozaki_k0_scales_c_and_nonfinite_rows(oz):
    import torch

    c = np.arange(12.0).reshape(4, 3)
    out = _run(oz, np.zeros((4, 0)), np.zeros((0, 3)), c, 0, 0, 2.0, 0.5)
    np.testing.assert_array_equal(out, 0.5 * c)
    opa, opb, c = _mats(70, 40, 50, 0, 0, seed=3)
    opa[5, 7] = np.nan
    opa[9, 0] = np.inf
    out = _run(oz, opa, opb, c, 0, 0, 1.0, 0.0)
    assert np.all(np.isnan(out[5])) and np.all(np.isnan(out[9]))
    rest = np.ones(70, bool)
    rest[[5, 9]] = False
    np.testing.assert_array_equal(out[rest], ozaki.gemm(opa[rest], opb))
    dev = torch.device("cuda", 0)
    A = torch.zeros(65001, dtype=torch.float64, device=dev)
    C = torch.zeros(1, dtype=torch.float64, device=dev)
    assert oz.dgemm_device(0, 0, 1, 1, 65001, 1.0, A.data_ptr(), 1, A.data_ptr(), 65001, 0.0, C.data_ptr(), 1, 0) != 0


def test_ozaki_n1788_matches_fp64(oz):
    import torch

    n = 1788
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(17)
    A = torch.randn((n, n), generator=g, dtype=torch.float64).to(dev)
    B = torch.randn((n, n), generator=g, dtype=torch.float64).to(dev)
    C = torch.empty((n, n), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    rc = oz.dgemm_device(0, 0, n, n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0, C.data_ptr(), n, 0)
    torch.cuda.synchronize(dev)
    assert rc == 0, oz.last_error()
    ref = B @ A  # the row-major views hold the transposes: C^T = B^T A^T
    absprod = B.abs() @ A.abs()
    assert bool(((C - ref).abs() <= 4 * n * 2.0 ** -53 * absprod).all())


@pytest.mark.parametrize("precision", [64, 32])
def test_solves_on_the_ozaki_engine_meet_the_fp64_bars(oz, precision):
    xe = oz
    old = xe.get_option("precision")
    xe.set_option("precision", precision)
    try:
        n = 700
        h, s, lam = inputs.generalized(n, seed=171)
        w_ref, c_ref = lapack.sygvd_chain(h, s)
        w, c, _, info = xe.dsygvd(h, s)
        assert info == 0, xe.last_error()
        assert np.max(np.abs(w - lam)) < 1e-10
        assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9
    finally:
        xe.set_option("precision", old)
