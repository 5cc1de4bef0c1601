"""Emulation of the library's FP64-from-int8 GEMM (Ozaki splitting) in numpy (TEST INFRASTRUCTURE ONLY).

The reference has no such GEMM: it calls Accelerate dgemm for every FP64 GEMM-shaped step
(Sources/Diagonalization/Stages/WYTransform.swift:22-79), so its oracle is the plain FP64 product.  This module restates
the library's splitting step by step so that the GPU engine can also be checked BIT FOR BIT:

  - every row r of op(A) (column of op(B)) gets e_r = 1 + frexp-exponent of its largest |entry| (1 for a zero row),
    so |x| 2^-e_r < 1/2;
  - 8 slices by repeated rounding to nearest (half to even): y = 128 x, a_p = rint(y), x = y - a_p (|a_p| <= 64);
  - D_d = sum_{p+q=d} A_p B_q^T for d = 2..9, exact integers (here FP64 BLAS products of integer matrices, exact while
    every partial sum stays below 2^53: 8 pairs x 64^2 x K is, for K < 2^37);
  - T = sum_{d=6..9} D_d 2^(7(9-d)) and U = sum_{d=2..5} D_d 2^(7(5-d)), integers below 2^53 (exact in FP64);
    C = alpha 2^(e_i + f_j - 63) (U 2^28 + T) + beta C, the sum U 2^28 + T rounded once.

The emulation reproduces the device result exactly when beta * C is exact (beta 0 or a power of two).
"""
from __future__ import annotations

import numpy as np

SLICES = 8


def split_rows(x: np.ndarray, slices: int = SLICES):
    """x: R x K.  Returns (a, e): a[p] (R x K, integer-valued float64), e (R,) int, x ~ 2^e sum_p a[p] 2^-7(p+1)."""
    x = np.asarray(x, dtype=np.float64)
    m = np.abs(x).max(axis=1) if x.shape[1] else np.zeros(x.shape[0])
    _, ef = np.frexp(m)
    e = ef.astype(np.int64) + 1
    r = np.ldexp(x, -e[:, None])
    a = np.empty((slices,) + x.shape)
    for p in range(slices):
        y = r * 128.0
        a[p] = np.rint(y)
        r = y - a[p]
    return a, e


def gemm(opa: np.ndarray, opb: np.ndarray, alpha: float = 1.0, beta: float = 0.0, c: np.ndarray | None = None,
         slices: int = SLICES) -> np.ndarray:
    """alpha op(A) op(B) + beta C as the device engine forms it (op(A): M x K, op(B): K x N, given explicitly)."""
    assert slices == SLICES
    a, ea = split_rows(opa, slices)
    b, eb = split_rows(np.asarray(opb, dtype=np.float64).T, slices)
    m, n = opa.shape[0], opb.shape[1]

    def part(dlo):  # sum_{d=dlo..dlo+3} D_d 2^(7(dlo+3-d)), Horner in 2^7 (every step an exact integer)
        acc = np.zeros((m, n))
        for d in range(dlo, dlo + 4):
            dd = np.zeros((m, n))
            for p in range(max(1, d - slices), min(slices, d - 1) + 1):
                dd += a[p - 1] @ b[d - p - 1].T  # integer sums, exact
            acc = acc * 128.0 + dd
        return acc

    t, u = part(6), part(2)
    acc = u * 2.0 ** 28 + t  # one rounding
    out = alpha * np.ldexp(acc, ea[:, None] + eb[None, :] - 63)
    if beta != 0.0:
        out = beta * np.asarray(c, dtype=np.float64) + out
    return out


def error_bound(opa: np.ndarray, opb: np.ndarray) -> np.ndarray:
    """A bound on |engine - exact| per entry, in FP64 units of the row's and column's scale.

    With s_i = 2^e_i <= 4 max|op(A)(i,:)| and t_j <= 4 max|op(B)(:,j)|, each of the K products carries at most
    2^-58 (slicing remainders, |r| <= 2^-57 against slices of sum <= 1/2) + 7 x 64^2 x 2^-70 (< 2^-55.1, the dropped
    pairs p + q = 10, and a 2^-7 geometric tail beyond) < 2^-54.9 of s_i t_j, and the 8 FP64 additions of the
    accumulator round at most 8 x 2^-53 of |acc| <= K/4.  Together below K 2^-51 s_i t_j <= K 2^-47 max|row| max|col|.
    """
    k = opa.shape[1]
    ra = np.abs(opa).max(axis=1) if k else np.zeros(opa.shape[0])
    cb = np.abs(opb).max(axis=0) if k else np.zeros(opb.shape[1])
    return max(k, 1) * 2.0 ** -47 * np.outer(ra, cb)
