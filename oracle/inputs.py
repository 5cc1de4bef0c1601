"""Seeded synthetic inputs for the five benchmark configurations (TEST INFRASTRUCTURE ONLY).

The reference reads real GFN2 H/S dumps (Sources/EigenBench/main.swift:159-174; none are in its repository) or
``random:N`` matrices (main.swift:151-158).  These generators stand in for the dumps with known spectra; every number
is drawn from ``numpy.random.default_rng(seed)`` in the order the code below draws it, so the same seed gives the same
bytes on every machine.

standard(n=412, seed=0)
    A = Q diag(lam) Q^T, Q = QR(standard normal n x n).  lam: n-8 values U[-1.2, 0.6] Eh plus a cluster of 8 values
    -0.25 + (i - 3.5) * 1e-6 Eh, i = 0..7.  A symmetrised as (A + A^T) / 2.
generalized(n, seed)
    S = I + G, G symmetric with zero diagonal, G_ij = 0.35 exp(-|i-j|/12) u_ij, u_ij ~ U[-1, 1] drawn as a full n x n
    matrix of which the strict upper triangle is used; S += (0.05 - lam_min(S)) I if lam_min(S) < 0.05.
    lam ~ U[-1.0, 0.5] Eh, sorted ascending, then lam[n//2:] += 0.05 (the HOMO/LUMO gap opened at index n//2, i.e. 602
    at n = 1204).  Q = QR(standard normal n x n).  H = S^1/2 Q diag(lam) Q^T S^1/2, symmetrised.
    The exact generalized eigenvalues of (H, S) are lam.
batch_sizes(count=256, seed=3)
    integer sizes U[124, 1788]; problem i is generalized(n_i, seed=1000 + i).
density_batch(count=32, n=588, seed=4)
    problem i is generalized(588, seed=4000 + i): gap at index 294 (294 occupied), mu at mid-gap.
"""
from __future__ import annotations

import numpy as np


def _orthogonal(rng, n):
    g = rng.standard_normal((n, n))
    q, r = np.linalg.qr(g)
    q = q * np.sign(np.diag(r))[None, :]
    return q


def standard(n: int = 412, seed: int = 0):
    """Config 1: returns (A, exact eigenvalues ascending)."""
    rng = np.random.default_rng(seed)
    q = _orthogonal(rng, n)
    ncl = min(8, n)
    lam = np.concatenate([rng.uniform(-1.2, 0.6, n - ncl), -0.25 + (np.arange(ncl) - 3.5) * 1e-6])
    a = (q * lam[None, :]) @ q.T
    a = 0.5 * (a + a.T)
    return np.asfortranarray(a), np.sort(lam)


def overlap(n: int, rng) -> np.ndarray:
    idx = np.arange(n)
    dist = np.abs(idx[:, None] - idx[None, :])
    u = rng.uniform(-1.0, 1.0, (n, n))
    g = 0.35 * np.exp(-dist / 12.0) * np.triu(u, 1)
    s = np.eye(n) + g + g.T
    lmin = np.linalg.eigvalsh(s)[0]
    if lmin < 0.05:
        s += (0.05 - lmin) * np.eye(n)
    return s


def generalized(n: int, seed: int):
    """Configs 2-5: returns (H, S, exact generalized eigenvalues ascending)."""
    rng = np.random.default_rng(seed)
    s = overlap(n, rng)
    lam = np.sort(rng.uniform(-1.0, 0.5, n))
    lam[n // 2:] += 0.05
    q = _orthogonal(rng, n)
    ws, vs = np.linalg.eigh(s)
    shalf = (vs * np.sqrt(ws)[None, :]) @ vs.T
    shalf = 0.5 * (shalf + shalf.T)
    m = (q * lam[None, :]) @ q.T
    h = shalf @ m @ shalf
    h = 0.5 * (h + h.T)
    return np.asfortranarray(h), np.asfortranarray(s), lam


def batch_sizes(count: int = 256, seed: int = 3, lo: int = 124, hi: int = 1788):
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(lo, hi + 1, count)]


def random_symmetric(n: int, seed: int):
    """The reference's ``random:N`` edge-case matrices (uniform [-1, 1], main.swift:151-158), seeded by numpy."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.0, (n, n))
    a = np.triu(u) + np.triu(u, 1).T
    return np.asfortranarray(a)


def random_tridiagonal(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, n), rng.uniform(-1.0, 1.0, max(n - 1, 0))
