"""Mixed precision on the GPU: FP32 reduction chain + FP64 refinement, and the refinement entry on its own.

Bars (the mixed path's target): eigenvalue error <= 1e-10 Eh against the exact spectrum and the oracle, density
matrix within 1e-9 of the oracle's, backward error <= 10 (in n eps ||H|| units), and S-orthogonality <= 1e-9 (two
first-order refinement steps from FP32 vectors; about 1e-12 at n >= 800, up to a few 1e-10 at small n).
"""
import numpy as np
import pytest

from oracle import inputs, lapack, metrics, refine

pytestmark = pytest.mark.gpu


@pytest.fixture
def mixed(xe):
    old = (xe.get_option("precision"), xe.get_option("refine_iters"))
    xe.set_option("precision", 32)
    xe.set_option("refine_iters", 2)
    yield xe
    xe.set_option("precision", old[0])
    xe.set_option("refine_iters", old[1])


def _check(h, s, lam, w, c, w_ref, c_ref, nocc):
    assert np.max(np.abs(w - lam)) < 1e-10
    assert np.max(np.abs(w - w_ref)) < 1e-10
    assert metrics.density_error(c, c_ref, metrics.aufbau(h.shape[0], nocc)) < 1e-9
    assert metrics.s_orthogonality(s, c) < 1e-9
    assert metrics.backward_error(h, s, w, c) < 10


@pytest.mark.parametrize("n", [1, 2, 17, 64, 130, 412])
def test_mixed_small(mixed, n):
    h, s, lam = inputs.generalized(n, seed=30 + n)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = mixed.dsygvd(h, s)
    assert info == 0
    _check(h, s, lam, w, c, w_ref, c_ref, n // 2)
    u_ref, _ = lapack.potrf_upper(s)
    assert np.max(np.abs(np.triu(u) - np.triu(u_ref))) < 1e-12


def test_mixed_config2_n1204(mixed):
    h, s, lam = inputs.generalized(1204, seed=1)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = mixed.dsygvd(h, s)
    assert info == 0
    _check(h, s, lam, w, c, w_ref, c_ref, 602)


def test_mixed_near_degenerate_cluster(mixed):
    """Six eigenvalues 1e-9 Eh apart below the gap: the refinement's exact cluster solve resolves them."""
    n = 300
    rng = np.random.default_rng(21)
    s = inputs.overlap(n, rng)
    lam = np.sort(rng.uniform(-1.0, 0.5, n))
    lam[100:106] = -0.3 + np.arange(6) * 1e-9
    lam = np.sort(lam)
    lam[n // 2:] += 0.05
    ws, vs = np.linalg.eigh(s)
    shalf = (vs * np.sqrt(ws)) @ vs.T
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    h = shalf @ (q * lam) @ q.T @ shalf
    h = np.asfortranarray(0.5 * (h + h.T))
    s = np.asfortranarray(s)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = mixed.dsygvd(h, s)
    assert info == 0
    _check(h, s, lam, w, c, w_ref, c_ref, n // 2)


def test_mixed_not_spd(mixed):
    n = 70
    h, s, _ = inputs.generalized(n, seed=2)
    s = s.copy()
    s[40, 40] = -1.0
    _, info_ref = lapack.potrf_upper(s)
    w, c, u, info = mixed.dsygvd(h, s)
    assert info == n + info_ref


def test_mixed_device_graph_replay(mixed):
    """Repeated device-pointer mixed solves (eager, captured, replayed) give identical bits."""
    import torch

    n = 257
    h, s, lam = inputs.generalized(n, seed=9)
    dev = torch.device("cuda", 0)
    mixed.set_device(0)
    stream = torch.cuda.Stream(dev)
    H0 = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    S0 = torch.from_numpy(np.ascontiguousarray(s)).to(dev)
    H, S = torch.empty_like(H0), torch.empty_like(S0)
    W = torch.empty(n, dtype=torch.float64, device=dev)
    outs = []
    with torch.cuda.stream(stream):
        for _ in range(4):
            H.copy_(H0)
            S.copy_(S0)
            assert mixed.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream) == 0
            outs.append((W.cpu().numpy().copy(), H.cpu().numpy().T.copy()))
    for w, c in outs[1:]:
        np.testing.assert_array_equal(w, outs[0][0])
        np.testing.assert_array_equal(c, outs[0][1])
    assert np.max(np.abs(outs[0][0] - lam)) < 1e-10


@pytest.mark.parametrize("iters", [1, 2, 3])
def test_refine_device_matches_oracle(xe, iters):
    """xtb_dsygvd_refine_device from the same perturbed start as the oracle's refinement: same eigenvalues and
    density to rounding, and FP64 accuracy after two steps."""
    import torch

    n = 200
    h, s, lam = inputs.generalized(n, seed=12)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    rng = np.random.default_rng(3)
    c0 = np.asfortranarray(c_ref + 2e-6 * rng.standard_normal(c_ref.shape))
    w_o, c_o = refine.refine(h, s, c0, iters)
    dev = torch.device("cuda", 0)
    xe.set_device(0)
    H = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(s)).to(dev)
    Cd = torch.from_numpy(np.ascontiguousarray(c0.T)).to(dev)  # row-major view of the column-major C
    W = torch.empty(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    info = xe.dsygvd_refine_device(n, H.data_ptr(), n, S.data_ptr(), n, Cd.data_ptr(), n, W.data_ptr(), iters)
    assert info == 0
    w = W.cpu().numpy()
    c = Cd.cpu().numpy().T
    assert np.max(np.abs(w - w_o)) < 1e-12
    assert metrics.density_error(c, c_o, metrics.aufbau(n, n // 2)) < 1e-11
    if iters >= 2:  # the oracle's own S-orthogonality after two steps here is 1.7e-11
        assert np.max(np.abs(w - lam)) < 1e-12
        assert metrics.s_orthogonality(s, c) < 1e-10


def test_refine_device_invalid_arguments(xe):
    assert xe.dsygvd_refine_device(-1, 0, 1, 0, 1, 0, 1, 0, 2) == -1
    assert xe.dsygvd_refine_device(4, 0, 3, 0, 4, 0, 4, 0, 2) == -3
    assert xe.dsygvd_refine_device(4, 0, 4, 0, 4, 0, 4, 0, 0) == -9
    assert xe.dsygvd_refine_device(0, 0, 1, 0, 1, 0, 1, 0, 2) == 0
    with pytest.raises(ValueError):
        xe.set_option("precision", 16)


def test_scc_policy_sets_the_precision_of_solves(xe):
    """The SCC precision policy of the calling thread: a cycle above the rmsq threshold solves in plain FP32 (about
    1e-6 accurate, xtb's FP32 mode) or FP32 + FP64 refinement (fp32_refine 1: the mixed path's bars); a cycle below
    it solves in FP64, bit for bit as the FP64 path; after fp32_maxiter cycles the run restarts in FP64."""
    n = 400
    h, s, lam = inputs.generalized(n, seed=95)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w64, c64, _, info = xe.dsygvd(h, s)
    assert info == 0
    try:
        xe.scc_set_precision(1e-3, fp32_maxiter=30, fp32_refine=0)
        assert xe.scc_cycle(1, -1.0) == 32
        w, c, _, info = xe.dsygvd(h, s)
        assert info == 0
        err = np.max(np.abs(w - lam))
        assert 1e-13 < err < 1e-4, err  # plain FP32 vectors: neither FP64-exact nor wrong
        assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-3
        assert xe.scc_cycle(2, 1e-4) == 64
        w, c, _, info = xe.dsygvd(h, s)
        assert info == 0
        np.testing.assert_array_equal(w, w64)
        np.testing.assert_array_equal(c, c64)
        xe.scc_set_precision(1e-3, fp32_maxiter=1, fp32_refine=1)
        assert xe.scc_cycle(1, -1.0) == 32
        w, c, _, info = xe.dsygvd(h, s)
        assert info == 0
        _check(h, s, lam, w, c, w_ref, c_ref, n // 2)
        assert xe.scc_cycle(2, 1e-2) == 0  # used FP32, not converged within 1 cycle: rerun in FP64
        assert xe.scc_cycle(1, -1.0) == 64
        w, c, _, info = xe.dsygvd(h, s)
        np.testing.assert_array_equal(w, w64)
    finally:
        xe.scc_set_precision(0.0)
