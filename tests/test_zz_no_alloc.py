"""The no-allocation reduction entry point, for callers that own all device memory themselves.

xtb_dsytrd_upper_noalloc serves callers that cannot let a library call cudaMalloc/cudaFree (their own pool or
allocator owns every byte on the GPU).  It takes the matrix and the outputs in device memory and keeps its scratch in
a static device array.  This test calls it through the C ABI twice in a row on fresh copies of the same matrix and
checks both results against the existing entry point xtb_dsytrd_upper, within the tolerance of the sytrd parity tests
(1e-11 * n * max|A| for d and e, 1e-11 * n for tau and the reflectors).  The file runs last so that a stop at the first
failure has already run every other test; it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest

from oracle import inputs

pytestmark = pytest.mark.gpu


def _bind(xe):
    fn = xe.lib().xtb_dsytrd_upper_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _run_noalloc(fn, a, stream=None):
    import torch

    n = a.shape[0]
    dev = torch.device("cuda", 0)
    # torch allocates the caller's buffers; column-major data is the transpose of torch's row-major view.
    ad = torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).to(dev)
    d = torch.zeros(n, dtype=torch.float64, device=dev)
    e = torch.zeros(max(n - 1, 1), dtype=torch.float64, device=dev)
    tau = torch.zeros(max(n - 1, 1), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    info = fn(n, ad.data_ptr(), n, d.data_ptr(), e.data_ptr(), tau.data_ptr(),
              stream.cuda_stream if stream is not None else None)
    torch.cuda.synchronize(dev)
    return info, ad.cpu().numpy().T, d.cpu().numpy(), e.cpu().numpy()[: n - 1], tau.cpu().numpy()[: n - 1]


def _check(a, out, ref):
    n = a.shape[0]
    info, ar, d, e, tau = out
    ar_ref, d_ref, e_ref, tau_ref = ref
    scale = np.abs(a).max() * n
    assert info == 0, info
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(e, e_ref, rtol=0, atol=1e-11 * scale)
    np.testing.assert_allclose(tau, tau_ref, rtol=0, atol=1e-11 * n)
    np.testing.assert_allclose(np.triu(ar), np.triu(ar_ref), rtol=0, atol=1e-11 * n)
    np.testing.assert_array_equal(np.tril(ar, -1), np.tril(a, -1))


@pytest.mark.parametrize("n", [1, 2, 37, 300, 1788])
def test_noalloc_matches_existing_entry_point_twice(xe, n):
    fn = _bind(xe)
    xe.set_device(0)
    a = inputs.random_symmetric(n, seed=500 + n)
    ref = xe.sytrd_upper(a)
    for _ in range(2):
        _check(a, _run_noalloc(fn, a), ref)


def test_noalloc_on_a_side_stream_between_other_solves(xe):
    """The static scratch keeps nothing that matters between calls: the entry point on a non-default stream, before
    and after a device-pointer solve of the library's allocating path on the same device, gives the same result."""
    import torch

    fn = _bind(xe)
    xe.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    n = 500
    a = inputs.random_symmetric(n, seed=900)
    ref = xe.sytrd_upper(a)
    _check(a, _run_noalloc(fn, a, stream), ref)
    h, s, lam = inputs.generalized(300, seed=901)
    H = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(s)).to(dev)
    W = torch.empty(300, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    assert xe.dsygvd_device(300, H.data_ptr(), 300, S.data_ptr(), 300, W.data_ptr(), stream.cuda_stream) == 0
    assert np.max(np.abs(W.cpu().numpy() - lam)) < 1e-10
    _check(a, _run_noalloc(fn, a, stream), ref)
    _check(a, _run_noalloc(fn, a), ref)


def test_noalloc_rejects_sizes_beyond_its_limit(xe):
    fn = _bind(xe)
    # Size checks happen before any device work: no device buffer is needed to see the rejection.
    assert fn(1793, None, 1793, None, None, None, None) == -1
    assert fn(-1, None, 1, None, None, None, None) == -1
    assert fn(10, None, 5, None, None, None, None) == -3
