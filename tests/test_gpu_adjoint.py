"""GPU checks of the Fermi-smeared density adjoint (xtb_dsygvd_density_adjoint and its batched form).

The adjoint is wrapped in a torch.autograd.Function (forward: P = C diag(f(e)) C^T from the library's generalized
solve; backward: the library's Daleckii-Krein adjoint), and checked
  - against central finite differences of the same forward (h = 1e-6, 64 random entries of H and of S, symmetric
    perturbations: dL/dh = G_ab + G_ba), at T = 100, 300 and 1000 K, within 1e-5 relative (the differences carry the
    solve's rounding ~1e-13 |L| / h);
  - against the FP64 CPU Daleckii-Krein oracle (numpy restatement on the LAPACK eigenpairs) at the differentiation
    workload's size n = 588 (294 occupied, mu at mid-gap), in FP64 and in mixed precision (the refined eigenpairs are
    FP64-accurate), within 1e-8 relative to the gradient's largest entry;
  - batched: several problems through xtb_dsygvd_density_adjoint_batched equal the single-problem call bit for bit.
"""
import numpy as np
import pytest

from oracle import fermi, inputs, lapack

pytestmark = pytest.mark.gpu


def _density_fn(xe):
    import torch

    class DensityMatrix(torch.autograd.Function):
        """P(H, S) = C diag(2 / (1 + exp((e - mu)/kT))) C^T for H C = S C diag(e), C^T S C = I (FP64, CPU tensors
        in, the solve and the adjoint on the GPU through the C ABI)."""

        @staticmethod
        def forward(ctx, h, s, kt, mu):
            w, c, _, info = xe.dsygvd(h.numpy(), s.numpy())
            if info != 0:
                raise RuntimeError(f"dsygvd info {info}")
            ctx.save_for_backward(h, s)
            ctx.kt, ctx.mu = kt, mu
            return torch.from_numpy(fermi.density(c, w, mu, kt))

        @staticmethod
        def backward(ctx, gp):
            h, s = ctx.saved_tensors
            wbar = 0.5 * (gp + gp.T)
            dh, ds, _, _, info = xe.density_adjoint(h.numpy(), s.numpy(), ctx.kt, ctx.mu, wbar.numpy())
            if info != 0:
                raise RuntimeError(f"adjoint info {info}")
            return torch.from_numpy(np.ascontiguousarray(dh)), torch.from_numpy(np.ascontiguousarray(ds)), None, None

    return DensityMatrix


@pytest.mark.parametrize("temp", [100.0, 300.0, 1000.0])
def test_autograd_adjoint_matches_central_differences(xe, temp):
    import torch

    n = 96
    h, s, lam = inputs.generalized(n, seed=140)
    kt = fermi.kt_of(temp)
    mu = 0.5 * (lam[n // 2 - 1] + lam[n // 2])
    rng = np.random.default_rng(7)
    w = rng.standard_normal((n, n))
    w = torch.from_numpy(w + w.T)
    fn = _density_fn(xe)
    H = torch.from_numpy(h.copy()).requires_grad_(True)
    S = torch.from_numpy(s.copy()).requires_grad_(True)
    loss = (w * fn.apply(H, S, kt, mu)).sum()
    loss.backward()
    gh, gs = H.grad.numpy(), S.grad.numpy()

    def lval(hh, ss):
        with torch.no_grad():
            return float((w * fn.apply(torch.from_numpy(hh), torch.from_numpy(ss), kt, mu)).sum())

    step = 1e-6
    idx = rng.integers(0, n, size=(64, 2))
    for a, b in idx:
        e = np.zeros((n, n))
        e[a, b] = 1.0
        e[b, a] = 1.0
        mult = 1.0 if a == b else 2.0  # dL/dh of a symmetric perturbation: G_ab + G_ba
        fd_h = (lval(h + step * e, s) - lval(h - step * e, s)) / (2 * step)
        fd_s = (lval(h, s + step * e) - lval(h, s - step * e)) / (2 * step)
        assert abs(fd_h - mult * gh[a, b]) < 1e-5 * max(1.0, abs(fd_h)), (a, b, fd_h, gh[a, b])
        assert abs(fd_s - mult * gs[a, b]) < 1e-5 * max(1.0, abs(fd_s)), (a, b, fd_s, gs[a, b])


@pytest.fixture
def prec(xe):
    old = xe.get_option("precision")
    yield xe
    xe.set_option("precision", old)


@pytest.mark.parametrize("precision", [64, 32])
def test_adjoint_n588_matches_dk_oracle(prec, precision):
    xe = prec
    xe.set_option("precision", precision)
    n = 588
    h, s, lam = inputs.generalized(n, seed=4)
    kt = fermi.kt_of(300.0)
    mu = 0.5 * (lam[293] + lam[294])
    rng = np.random.default_rng(4)
    wb = rng.standard_normal((n, n))
    wb = wb + wb.T
    dh, ds, e, c, info = xe.density_adjoint(h, s, kt, mu, wb)
    assert info == 0
    w_ref, c_ref = lapack.sygvd_chain(h, s)
    gh, gs = fermi.dk_gradient(c_ref, w_ref, wb, mu, kt)
    assert np.max(np.abs(dh - gh)) < 1e-8 * np.abs(gh).max()
    assert np.max(np.abs(ds - gs)) < 1e-8 * np.abs(gs).max()


def test_adjoint_batched_equals_single(xe):
    sizes = [60, 131, 200, 97]
    probs = [inputs.generalized(m, seed=150 + i) for i, m in enumerate(sizes)]
    rng = np.random.default_rng(9)
    wbars, kts, mus = [], [], []
    for (h, s, lam), temp in zip(probs, [100.0, 300.0, 1000.0, 300.0]):
        m = h.shape[0]
        wb = rng.standard_normal((m, m))
        wbars.append(wb + wb.T)
        kts.append(fermi.kt_of(temp))
        mus.append(0.5 * (lam[m // 2 - 1] + lam[m // 2]))
    dhs, dss, info = xe.density_adjoint_batched([p[0] for p in probs], [p[1] for p in probs], kts, mus, wbars)
    assert np.all(info == 0)
    for i, (h, s, _) in enumerate(probs):
        dh, ds, _, _, inf1 = xe.density_adjoint(h, s, kts[i], mus[i], wbars[i])
        assert inf1 == 0
        np.testing.assert_array_equal(dhs[i], dh)
        np.testing.assert_array_equal(dss[i], ds)
