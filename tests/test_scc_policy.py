"""The SCC precision policy (FP32-early / FP64-to-convergence with an FP64 restart), host logic only (no GPU).

This is the library-side form of xtb's SCC precision switch (reference LOG.md:317-363: FP32 eigensolves while the
density's RMS change is above a threshold, FP64 from then on; a run that used FP32 and does not converge within
fp32_maxiter cycles is rerun from its start with every eigensolve in FP64).  The state machine runs on the host, so
this test needs no GPU: it checks the precision each cycle gets, the latch, the restart signal and the argument
checks.
"""
import threading

import pytest

import xtbeig


@pytest.fixture
def policy():
    yield xtbeig
    xtbeig.scc_set_precision(0.0)


def test_fp32_early_then_fp64_latched(policy):
    policy.scc_set_precision(1e-3, fp32_maxiter=50, fp32_refine=0)
    assert policy.scc_cycle(1, -1.0) == 32
    assert policy.scc_cycle(2, 5e-2) == 32
    assert policy.scc_cycle(3, 2e-3) == 32
    assert policy.scc_cycle(4, 9e-4) == 64
    assert policy.scc_cycle(5, 5e-3) == 64  # latched: FP64 to convergence even if rmsq rises again
    on, fp32, restarted, prec = policy.scc_report()
    assert on and fp32 == 3 and not restarted and prec == 64


def test_restart_in_fp64_after_maxiter(policy):
    policy.scc_set_precision(1e-3, fp32_maxiter=4, fp32_refine=1)
    assert [policy.scc_cycle(c, 1e-2) for c in range(1, 5)] == [32, 32, 32, 32]
    assert policy.scc_cycle(5, 1e-2) == 0  # not converged within 4 cycles: rerun from the start
    assert policy.scc_report()[2]
    assert [policy.scc_cycle(c, 1e-2) for c in range(1, 4)] == [64, 64, 64]  # the rerun is FP64 throughout


def test_off_follows_the_precision_option(policy):
    policy.scc_set_precision(0.0)
    assert policy.scc_cycle(1, -1.0) == policy.get_option("precision")
    assert not policy.scc_report()[0]


def test_policy_is_per_thread(policy):
    policy.scc_set_precision(1e-3)
    assert policy.scc_cycle(1, -1.0) == 32
    seen = []
    t = threading.Thread(target=lambda: seen.append(policy.scc_report()))
    t.start()
    t.join()
    assert seen == [(False, 0, False, policy.get_option("precision"))]


def test_arguments(policy):
    for args in ((-1.0, 10, 0), (float("nan"), 10, 0), (1e-3, 0, 0), (1e-3, 10, 2)):
        with pytest.raises(ValueError):
            policy.scc_set_precision(*args)
    with pytest.raises(ValueError):
        policy.set_option("refine_iters", -1)
