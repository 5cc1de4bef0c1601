"""Accuracy measures (TEST INFRASTRUCTURE ONLY).

``eigen_accuracy`` is the reference's EigenBench ``accuracy`` (Sources/EigenBench/main.swift:231-251): max |w - wRef|,
residual max |H X - X diag(w)| / max |wRef| and orthogonality max |X^T X - I|, all in FP64.  The generalized measures
(backward error ||HC - SC diag(e)|| / (||H|| n eps), S-orthogonality max |C^T S C - I|) and the density-matrix error
are the ones the eigensolve is judged on; the density error is invariant to column signs and to rotations inside
degenerate subspaces because it compares P = C f C^T, not C.
"""
from __future__ import annotations

import numpy as np

EPS = np.finfo(np.float64).eps


def eigen_accuracy(h, w_ref, w, z):
    h = np.asarray(h, np.float64)
    w = np.asarray(w, np.float64)
    z = np.asarray(z, np.float64)
    dw = float(np.max(np.abs(w - w_ref))) if w.size else 0.0
    scale = float(np.max(np.abs(w_ref))) if w.size else 1.0
    res = float(np.max(np.abs(h @ z - z * w[None, :]))) / max(scale, 1e-300) if w.size else 0.0
    m = z.shape[1]
    orth = float(np.max(np.abs(z.T @ z - np.eye(m)))) if m else 0.0
    return dw, res, orth


def backward_error(h, s, w, c):
    """||H C - S C diag(w)||_F / (||H||_F n eps)."""
    h = np.asarray(h, np.float64)
    n = h.shape[0]
    r = h @ c - (s @ c) * np.asarray(w)[None, :]
    return float(np.linalg.norm(r) / (np.linalg.norm(h) * n * EPS))


def s_orthogonality(s, c):
    m = c.shape[1]
    return float(np.max(np.abs(c.T @ s @ c - np.eye(m))))


def density(c, occ):
    c = np.asarray(c, np.float64)
    return (c * np.asarray(occ)[None, :]) @ c.T


def density_error(c, c_ref, occ, occ_ref=None):
    occ_ref = occ if occ_ref is None else occ_ref
    return float(np.max(np.abs(density(c, occ) - density(c_ref, occ_ref))))


def aufbau(n, nocc):
    f = np.zeros(n)
    f[:nocc] = 2.0
    return f


def fnv1a(*arrays) -> int:
    """FNV-1a over the bytes of the arrays (the reference's tridiagonal hash, main.swift:253-266)."""
    h = 0xCBF29CE484222325
    for a in arrays:
        for b in np.ascontiguousarray(a).tobytes():
            h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h
