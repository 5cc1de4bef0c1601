"""FP64 Ogita-Aishima refinement of an approximate generalized eigendecomposition (TEST INFRASTRUCTURE ONLY).

CPU restatement of the reference's refinement step, scripts/kernels/refine.f90:258-325 (method_oa_from), with the
identity inner product replaced by S (the library refines H C = S C diag(e), C^T S C = I on the FP64 pair directly):

    A = C^T H C,  B = C^T S C
    lam_i = A_ii / B_ii                                   (refine.f90: lam(i) = A(i,i) / (1 - R(i,i)), R = I - C^T C)
    delta = min(max(32 max_{i != j} |A_ij|, 1e-10), 1e-3) (refine.f90:276-283 uses 2; 32 keeps every first-order
                                                          correction below 1/32, so two steps from FP32 vectors
                                                          reach FP64 S-orthogonality)
    E_ij  = (A_ij - lam_j B_ij) / (lam_j - lam_i)          if |lam_j - lam_i| > delta
          = (delta_ij - B_ij) / 2                          otherwise
    clusters (runs of consecutive lam closer than delta, cut at 32): x = the B_cc-orthonormal eigenvectors of
    (A_cc, B_cc) (the reference diagonalises A_cc alone), lam_c their eigenvalues; the cluster's columns of I + E
    become [(I + E)_{i,c} x for rows i outside the cluster; x inside], i.e. the first-order corrections from the
    other vectors are applied to the cluster's own vectors before they are rotated by x.  (The reference writes x
    over the block alone, which pairs the outside corrections with the wrong columns whenever x permutes or
    flips a cluster's vectors.)
    C <- C (I + E)

After the last step C and lam are put in ascending order.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

MAX_CLUSTER = 32
DELTA_FACTOR = 32.0


def oa_step(h, s, c):
    """One refinement step; returns (C_new, lam) with lam not yet sorted."""
    a = c.T @ h @ c
    b = c.T @ s @ c
    a = 0.5 * (a + a.T)
    b = 0.5 * (b + b.T)
    n = a.shape[0]
    lam = np.diag(a) / np.diag(b)
    off = np.abs(a - np.diag(np.diag(a)))
    delta = min(max(DELTA_FACTOR * off.max() if n > 1 else 0.0, 1e-10), 1e-3)
    g = lam[None, :] - lam[:, None]  # g[i, j] = lam_j - lam_i
    sep = np.abs(g) > delta
    with np.errstate(divide="ignore", invalid="ignore"):
        e = np.where(sep, (a - lam[None, :] * b) / np.where(sep, g, 1.0), -0.5 * b)
    np.fill_diagonal(e, 0.5 * (1.0 - np.diag(b)))
    m = np.eye(n) + e
    lam_out = lam.copy()
    i = 0
    while i < n:
        j = i + 1
        while j < n and abs(lam[j] - lam[j - 1]) <= delta:
            j += 1
        for c0 in range(i, j, MAX_CLUSTER):
            c1 = min(c0 + MAX_CLUSTER, j)
            if c1 - c0 >= 2:
                try:
                    w, x = sla.eigh(a[c0:c1, c0:c1], b[c0:c1, c0:c1])
                except np.linalg.LinAlgError:
                    continue
                m[:, c0:c1] = m[:, c0:c1] @ x
                m[c0:c1, c0:c1] = x
                lam_out[c0:c1] = w
        i = j
    return c @ m, lam_out


def refine(h, s, c, iters=2):
    """`iters` steps from C (any column order); returns (eigenvalues ascending, C in the same order)."""
    for _ in range(iters):
        c, lam = oa_step(h, s, c)
    order = np.argsort(lam, kind="stable")
    return lam[order], c[:, order]
