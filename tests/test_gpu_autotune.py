"""GPU checks of the autotuner (xtb_gpu_autotune) and of solve plans.

The tuner measures candidate plans on a synthetic generalized pair and keeps the fastest; with the option "autotune"
on, solves use the plan of the nearest tuned size.  Checked: the tuned plan is one of the candidates, solves under it
meet the FP64 path's bars against the oracle (eigenvalues within 1e-10 Eh, density within 1e-9), and a device solve
repeated on the same buffers after a plan change runs the new plan (the captured graph of the old plan is not
replayed: the launch count of the next call equals the new plan's eager launch count).
"""
import numpy as np
import pytest

from oracle import inputs, lapack, metrics

pytestmark = pytest.mark.gpu


@pytest.fixture
def restore(xe):
    keys = ("autotune", "reduction", "band_width", "precision", "ormtr_nb", "sytrd_grid", "dgemm_engine")
    old = {k: xe.get_option(k) for k in keys}
    yield xe
    for k, v in old.items():
        xe.set_option(k, v)


@pytest.mark.parametrize("precision", [64, 32])
def test_autotune_plan_and_solve(restore, precision):
    xe = restore
    n = 200
    plan = xe.autotune(n, precision)
    assert plan is not None and plan["ms"] > 0
    assert plan["reduction"] in (1, 2) and plan["band_width"] in (16, 32, 64)
    assert plan["ormtr_nb"] in (64, 128, 256) and plan["mixed_gemm"] in (0, 3) and plan["dgemm"] in (0, 1)
    xe.set_option("autotune", 1)
    xe.set_option("precision", precision)
    h, s, lam = inputs.generalized(n, seed=91)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0
    assert np.max(np.abs(w - lam)) < 1e-10
    assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9


def test_untuned_size_reports_none(xe):
    assert xe.tuned_plan(7, 64) is None


def test_plan_change_is_not_replayed_from_a_stale_graph(restore):
    import torch

    xe = restore
    xe.set_device(0)
    n = 300
    h, s, lam = inputs.generalized(n, seed=93)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    H0 = torch.from_numpy(h).to(dev)
    S0 = torch.from_numpy(s).to(dev)
    H, S = H0.clone(), S0.clone()
    W = torch.empty(n, dtype=torch.float64, device=dev)

    def solve():
        H.copy_(H0)
        S.copy_(S0)
        torch.cuda.synchronize(dev)
        c0 = xe.launch_count()
        info = xe.dsygvd_device(n, H.data_ptr(), n, S.data_ptr(), n, W.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize(dev)
        assert info == 0, xe.last_error()
        return xe.launch_count() - c0

    xe.set_option("autotune", 0)
    xe.set_option("reduction", 1)
    eager_one = solve()          # eager
    solve()                      # captured
    assert solve() == eager_one  # replayed: same kernels
    xe.set_option("reduction", 2)
    eager_two = solve()          # a new plan: runs eagerly, not the one-stage graph
    assert eager_two != eager_one
    np.testing.assert_allclose(W.cpu().numpy(), lam, atol=1e-10)
