"""Failure detection on the GPU without a GPU fault: a device wait that runs out of time.

Every spin wait in the library's kernels has a time limit (option "wait_limit_ms"): when it runs out, the kernel
records a barrier-timeout status in the device status word and returns, and the other CTAs see the status and return
too.  The reference's counterpart is the stall trap of its thread barrier (Sources/Diagonalization/Parallel.swift
:44-58).  The test hook "test_barrier_stall" makes the resident reduction's grid barriers wait for one CTA more than
the grid holds, so that no barrier can complete: the wait must run out after the limit, the call must report the
timeout (info -2001, last status 1, a message naming the barrier), and the next call on the same thread and device
must run normally and match the oracle.  Nothing here traps, asserts on the device or reads out of bounds; every
wait ends by its time limit.
"""
import time

import numpy as np
import pytest

from oracle import inputs, lapack, metrics

pytestmark = pytest.mark.gpu

LIMIT_MS = 30


@pytest.fixture
def stall(xe):
    old = xe.get_option("wait_limit_ms")
    xe.set_option("wait_limit_ms", LIMIT_MS)
    xe.set_option("test_barrier_stall", 1)
    yield xe
    xe.set_option("test_barrier_stall", 0)
    xe.set_option("wait_limit_ms", old)


def test_sygvd_barrier_timeout_then_recovers(stall):
    xe = stall
    n = 300
    h, s, lam = inputs.generalized(n, seed=81)
    t0 = time.perf_counter()
    w, c, u, info = xe.dsygvd(h, s)
    dt = time.perf_counter() - t0
    assert info == -2001, info
    assert xe.last_status() == 1
    assert "barrier" in xe.last_error()
    assert dt < 10.0  # the wait gave up after its limit instead of hanging
    xe.set_option("test_barrier_stall", 0)
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    w, c, u, info = xe.dsygvd(h, s)
    assert info == 0 and xe.last_status() == 0
    assert np.max(np.abs(w - lam)) < 1e-10 and np.max(np.abs(w - w_ref)) < 1e-12
    assert metrics.density_error(c, c_ref, metrics.aufbau(n, n // 2)) < 1e-9


def test_sytrd_barrier_timeout_status_then_recovers(stall):
    """The xtb sytrd.c entry has no info argument: the timeout is reported by xtb_gpu_last_status / last_error."""
    xe = stall
    n = 200
    a = inputs.random_symmetric(n, seed=82)
    with pytest.raises(xe.GPUError, match="barrier"):
        xe.sytrd_upper(a)
    assert xe.last_status() == 1
    xe.set_option("test_barrier_stall", 0)
    ar, d, e, tau = xe.sytrd_upper(a)
    _, d_ref, e_ref, _ = lapack.sytrd_upper(a)
    scale = np.abs(a).max() * n
    assert np.max(np.abs(d - d_ref)) < 1e-11 * scale
    assert np.max(np.abs(e - e_ref)) < 1e-11 * scale

