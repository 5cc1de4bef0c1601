"""GPU checks of the tcgen05 FP32 GEMM engine (xtb_sgemm_tc_device), the engine of the mixed solve's FP32 GEMMs.

Reference: the same FP32 inputs multiplied in FP64 (torch on the device).  Tolerances, elementwise against
|op(A)| |op(B)| (the sum of absolute products):
  3 passes (3xTF32):  4 (2^-20 + k 2^-24)   - two TF32 parts per operand, FP32 accumulation;
  1 pass  (TF32):     4 (2^-10 + k 2^-24)   - TF32 operands (10-bit mantissa).
Sizes cover single elements, tile edges (127-129, 31-33 deep), odd leading dimensions and the n = 1788 solve size;
all four transpose combinations (K-major and MN-major tensor-core operands); beta = 0 (C not read) and beta != 0.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(xe, ta, tb, m, n, k, alpha, beta, passes, seed, pad=0):
    import torch

    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(seed)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    lda, ldb, ldc = ar + pad, br + pad, m + pad
    # column-major storage: a (ar x ac, lda) is the transpose of a row-major (ac x lda) tensor
    A = torch.randn((ac, lda), generator=g, dtype=torch.float32).to(dev)
    B = torch.randn((bc, ldb), generator=g, dtype=torch.float32).to(dev)
    C = torch.randn((n, ldc), generator=g, dtype=torch.float32).to(dev)
    a = A[:, :ar].T.double()
    b = B[:, :br].T.double()
    opa = a.T if ta else a
    opb = b.T if tb else b
    c0 = C[:, :m].T.double()
    ref = alpha * (opa @ opb) + beta * c0
    absprod = opa.abs() @ opb.abs() + abs(beta) * c0.abs()
    C_orig = C.clone()
    torch.cuda.synchronize(dev)
    rc = xe.sgemm_tc_device(ta, tb, m, n, k, alpha, A.data_ptr(), lda, B.data_ptr(), ldb, beta, C.data_ptr(), ldc,
                            passes, 0)
    torch.cuda.synchronize(dev)
    assert rc == 0, (rc, xe.last_error())
    out = C[:, :m].T.double()
    if pad:
        assert torch.equal(C[:, m:], C_orig[:, m:]), "rows beyond m (ldc padding) must not change"
    return out, ref, absprod


CASES = [
    (1, 1, 1), (5, 7, 3), (31, 33, 17), (128, 128, 32), (127, 129, 33), (129, 127, 31), (200, 64, 300),
    (64, 300, 200), (300, 257, 1000),
]


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("mnk", CASES)
def test_sgemm_3xtf32_matches_fp64(xe, ta, tb, mnk):
    m, n, k = mnk
    out, ref, absprod = _run(xe, ta, tb, m, n, k, 1.0, 0.0, 3, seed=m * 7 + n * 3 + k + 10 * ta + 20 * tb)
    bound = 4 * (2.0 ** -20 + k * 2.0 ** -24) * absprod + 1e-30
    err = (out - ref).abs()
    assert bool((err <= bound).all()), float((err / bound).max())


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_sgemm_beta_and_padding(xe, ta, tb):
    m, n, k = 150, 90, 70
    out, ref, absprod = _run(xe, ta, tb, m, n, k, -0.75, 1.5, 3, seed=5 + ta + 2 * tb, pad=3)
    bound = 4 * (2.0 ** -20 + k * 2.0 ** -24) * absprod + 1e-30
    assert bool(((out - ref).abs() <= bound).all())


def test_sgemm_tf32_single_pass_is_tf32_accurate(xe):
    m, n, k = 256, 256, 512
    out1, ref, absprod = _run(xe, 0, 0, m, n, k, 1.0, 0.0, 1, seed=3)
    bound1 = 4 * (2.0 ** -10 + k * 2.0 ** -24) * absprod
    assert bool(((out1 - ref).abs() <= bound1).all())
    out3, ref3, _ = _run(xe, 0, 0, m, n, k, 1.0, 0.0, 3, seed=3)
    e1 = float((out1 - ref).abs().max())
    e3 = float((out3 - ref3).abs().max())
    # the split passes must buy back the TF32 truncation (what remains is the FP32 accumulation of k = 512 products)
    assert e3 * 20 < e1, (e1, e3)


def test_sgemm_solve_size(xe):
    n = 1788
    out, ref, absprod = _run(xe, 1, 0, n, n, n, 1.0, 0.0, 3, seed=42)
    bound = 4 * (2.0 ** -20 + n * 2.0 ** -24) * absprod
    assert bool(((out - ref).abs() <= bound).all())


def test_sgemm_argument_errors(xe):
    assert xe.sgemm_tc_device(2, 0, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 3, 0) == -1
    assert xe.sgemm_tc_device(0, 0, 4, 4, 4, 1.0, None, 3, None, 4, 0.0, None, 4, 3, 0) == -8
    assert xe.sgemm_tc_device(0, 0, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 2, 0) == -14
    assert xe.sgemm_tc_device(0, 0, 0, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 4, 3, 0) == 0


def _run_d(xe, ta, tb, m, n, k, alpha, beta, seed):
    import torch

    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(seed)
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    A = torch.randn((ac, ar), generator=g, dtype=torch.float64).to(dev)
    B = torch.randn((bc, br), generator=g, dtype=torch.float64).to(dev)
    C = torch.randn((n, m), generator=g, dtype=torch.float64).to(dev)
    opa = A.T.T if ta else A.T
    opb = B.T.T if tb else B.T
    ref = alpha * (opa @ opb) + beta * C.T
    absprod = opa.abs() @ opb.abs() + abs(beta) * C.T.abs()
    torch.cuda.synchronize(dev)
    rc = xe.dgemm_device(ta, tb, m, n, k, alpha, A.data_ptr(), ar, B.data_ptr(), br, beta, C.data_ptr(), m, 0)
    torch.cuda.synchronize(dev)
    assert rc == 0, (rc, xe.last_error())
    return C.T, ref, absprod


@pytest.mark.parametrize("engine", [0, 1])
@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (63, 65, 17), (130, 257, 129), (600, 500, 700)])
def test_dgemm_matches_fp64(xe, ta, tb, mnk, engine):
    """xtb_dgemm_device against torch's FP64 product, elementwise within 2 k eps |op(A)| |op(B)|: engine 0 (FP64
    DMMA) at every size, engine 1 (the default: int8 Ozaki from 512^3 up, DMMA below)."""
    m, n, k = mnk
    old = xe.get_option("dgemm_engine")
    xe.set_option("dgemm_engine", engine)
    try:
        out, ref, absprod = _run_d(xe, ta, tb, m, n, k, 1.25, -0.5, seed=m + 3 * n + 7 * k + ta + 2 * tb)
    finally:
        xe.set_option("dgemm_engine", old)
    bound = 2 * (k + 2) * 2.0 ** -53 * absprod + 1e-300
    assert bool(((out - ref).abs() <= bound).all())


@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("tb", [0, 1])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (31, 33, 17), (127, 129, 65), (200, 64, 300), (300, 257, 1000)])
@pytest.mark.parametrize("passes", [11, 13])
def test_sgemm_bf16_matches_fp64(xe, ta, tb, mnk, passes):
    """BF16 operands on kind::f16 (FP32 accumulation): passes 11 rounds each operand to BF16 (8-bit mantissa),
    bound 4 (2^-8 + k 2^-24) |op(A)| |op(B)|; passes 13 keeps hi*hi + hi*lo + lo*hi of a two-piece BF16 split,
    bound 4 (2^-16 + k 2^-24).  The operands are written K-major by the split pass whatever their storage, so all four
    transpose combinations run the same tensor-core layout."""
    m, n, k = mnk
    out, ref, absprod = _run(xe, ta, tb, m, n, k, 1.0, 0.0, passes, seed=m * 5 + n + k + 10 * ta + 20 * tb + passes)
    rel = 2.0 ** -8 if passes == 11 else 2.0 ** -16
    bound = 4 * (rel + k * 2.0 ** -24) * absprod + 1e-30
    err = (out - ref).abs()
    assert bool((err <= bound).all()), float((err / bound).max())


def test_sgemm_bf16_alpha_beta_and_padding(xe):
    out, ref, absprod = _run(xe, 0, 1, 129, 130, 131, -0.75, 0.5, 13, seed=4, pad=5)
    bound = 4 * (2.0 ** -16 + 131 * 2.0 ** -24) * absprod + 1e-30
    assert bool(((out - ref).abs() <= bound).all())
