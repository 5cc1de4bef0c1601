"""Generate the golden fixtures in this folder (run from the repository root: python tests/golden/make_golden.py).

The reference itself cannot run here (Swift + Apple Accelerate; its xtb submodule is empty), and it commits no H/S
dumps or eigensolver golden vectors.  Its own check pins every variant at run time to LAPACK dsyevd on the same
matrix (Sources/EigenBench/main.swift:505-531).  These fixtures are therefore
  * known-answer problems whose spectra are exact by construction (A = Q diag(lam) Q^T, H = S^1/2 Q diag(lam) Q^T S^1/2,
    the tridiagonal Toeplitz matrix with eigenvalues a + 2 b cos(k pi/(n+1))), and
  * the outputs of the reference's LAPACK call chain (OpenBLAS 0.3.30 from scipy 1.18.1) on small seeded inputs,
    recorded with the library build string, so that a later change of the CPU oracle is detected.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import inputs, lapack  # noqa: E402


def main():
    out = {}
    # Dense symmetric (the reference's random:N edge cases, odd and small sizes).
    for n in (1, 2, 3, 5, 17, 33, 64):
        a = inputs.random_symmetric(n, seed=100 + n)
        ar, d, e, tau = lapack.sytrd_upper(a)
        w, z, info = lapack.stedc(d, e)
        out[f"sym{n}_a"] = a
        out[f"sym{n}_sytrd_a"] = ar
        out[f"sym{n}_d"] = d
        out[f"sym{n}_e"] = e
        out[f"sym{n}_tau"] = tau
        out[f"sym{n}_w"] = w
        out[f"sym{n}_evals"] = np.linalg.eigvalsh(a)
    # Known spectrum, standard problem (config-1 construction at a small size).
    a, lam = inputs.standard(48, seed=0)
    out["std48_a"] = a
    out["std48_lam"] = lam
    # Known spectrum, generalized problem (config-2 construction at a small size).
    h, s, lam = inputs.generalized(40, seed=1)
    w, c = lapack.sygvd_chain(h, s)
    out["gen40_h"] = h
    out["gen40_s"] = s
    out["gen40_lam"] = lam
    out["gen40_w"] = w
    # Tridiagonal Toeplitz: exact eigenvalues a + 2 b cos(k pi / (n + 1)).
    n = 25
    out["toe25_d"] = np.full(n, 0.3)
    out["toe25_e"] = np.full(n - 1, -0.7)
    k = np.arange(1, n + 1)
    out["toe25_lam"] = np.sort(0.3 + 2 * (-0.7) * np.cos(k * np.pi / (n + 1)))
    out["oracle_build"] = np.array(os.path.basename(lapack._load()._name))
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
