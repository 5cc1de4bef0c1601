"""Fermi occupations, the density matrix and its FP64 Daleckii-Krein gradient (TEST INFRASTRUCTURE ONLY).

``fermi`` restates scripts/kernels/refine.f90:106-121 (bisection for mu over 200 halvings, f = 1/(1+exp(min(700,
(e-mu)/kT)))) and ``density`` refine.f90:124-135 (P = C diag(f) C^T); kB = 3.166808578545117e-6 Eh/K is refine.f90:30.
The closed-shell occupation used for the density/adjoint workload is 2 f (alpha and beta each f, refine.f90:96-103
with UHF = 0).

The reference has no adjoint.  ``dk_gradient`` is the Daleckii-Krein formula for L = sum(W o P), P = C f(e) C^T with
H C = S C diag(e), C^T S C = I:
    dL/dH =  C (W^ o D1) C^T,   dL/dS = -C (W^ o D2) C^T,   W^ = C^T W C,
    D1_ij = (f_i - f_j)/(e_i - e_j)          (f'(e_i) on the diagonal),
    D2_ij = (f_i e_i - f_j e_j)/(e_i - e_j)  = (f_i + f_j)/2 + (e_i + e_j)/2 D1_ij.
The divided difference of the logistic function is evaluated in a form without cancellation for near-degenerate
pairs:  (s(a) - s(b))/(a - b) = -sinhc((a-b)/2) / (4 cosh(a/2) cosh(b/2)),  s(x) = 1/(1+e^x).
Gradients are with respect to the symmetric matrices' entries as independent variables: for a symmetric perturbation
H + h (E_ab + E_ba), a != b, dL/dh = 2 G_ab.
"""
from __future__ import annotations

import numpy as np

KB = 3.166808578545117e-06  # Eh / K


def kt_of(temp_k: float) -> float:
    return KB * temp_k


def fermi_mu(e, ne, kt):
    """refine.f90:106-121: mu by bisection so that sum(f) = ne, f = 1/(1+exp((e-mu)/kT))."""
    lo, hi = float(np.min(e)) - 1.0, float(np.max(e)) + 1.0
    f = None
    for _ in range(200):
        mu = 0.5 * (lo + hi)
        f = 1.0 / (1.0 + np.exp(np.minimum(700.0, (e - mu) / kt)))
        if f.sum() > ne:
            hi = mu
        else:
            lo = mu
    return mu, f


def occupations(e, mu, kt):
    """Closed-shell Fermi occupations 2 / (1 + exp((e - mu)/kT))."""
    x = np.clip((np.asarray(e) - mu) / kt, -700.0, 700.0)
    return 2.0 / (1.0 + np.exp(x))


def density(c, e, mu, kt):
    f = occupations(e, mu, kt)
    return (c * f[None, :]) @ c.T


def _sigma(x):
    return 1.0 / (1.0 + np.exp(np.clip(x, -700.0, 700.0)))


def divided_differences(e, mu, kt):
    """D1 (divided differences of f = 2 s((e - mu)/kT)) and D2 (of e f), FP64, stable for near-degenerate pairs."""
    e = np.asarray(e, np.float64)
    x = (e - mu) / kt
    a = x[:, None]
    b = x[None, :]
    delta = 0.5 * (a - b)
    with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
        direct = (_sigma(a) - _sigma(b)) / (a - b)
        ch = np.cosh(np.clip(0.5 * a, -350, 350)) * np.cosh(np.clip(0.5 * b, -350, 350))
        small = np.abs(delta) < 1e-2
        d = np.where(small, 1.0 + delta * delta / 6.0 + delta ** 4 / 120.0, 1.0)
        stable = -d / (4.0 * ch)
    ds = np.where(np.abs(delta) < 1e-2, stable, direct)
    d1 = (2.0 / kt) * ds
    f = 2.0 * _sigma(x)
    d2 = 0.5 * (f[:, None] + f[None, :]) + 0.5 * (e[:, None] + e[None, :]) * d1
    return d1, d2


def dk_gradient(c, e, w, mu, kt):
    """FP64 Daleckii-Krein gradient (dL/dH, dL/dS) of L = sum(W o P)."""
    what = c.T @ w @ c
    d1, d2 = divided_differences(e, mu, kt)
    gh = c @ (what * d1) @ c.T
    gs = -(c @ (what * d2) @ c.T)
    return 0.5 * (gh + gh.T), 0.5 * (gs + gs.T)
