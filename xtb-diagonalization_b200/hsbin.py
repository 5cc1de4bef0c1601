"""Reader and writer of the reference's H/S matrix dumps, so that real GFN2 matrices can replace the synthetic inputs.

Format (reference Sources/EigenBench/main.swift:159-174 reads it; scripts/kernels/refine.f90:64-83 reads the SCC-cycle
variant): little-endian int32 n, then H (n x n float64, column-major), S (n x n float64, column-major), and in the
per-cycle files "<prefix>_<k>.bin" also the eigenvalues e (n float64) and eigenvectors C (n x n float64,
column-major) of that cycle.  H and S are full symmetric matrices.
"""
from __future__ import annotations

import os
import struct

import numpy as np


def read_hs_bin(path: str) -> dict:
    """Read a dump: {"n", "h", "s"} and, when present, {"e", "c"} (numpy float64, Fortran order)."""
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        (n,) = struct.unpack("<i", f.read(4))
        if n <= 0:
            raise ValueError(f"{path}: invalid n = {n}")
        nn = n * n
        base = 4 + 16 * nn
        if size not in (base, base + 8 * (n + nn)):
            raise ValueError(f"{path}: {size} bytes do not match n = {n} (expected {base} or {base + 8 * (n + nn)})")
        h = np.fromfile(f, dtype="<f8", count=nn).reshape((n, n), order="F")
        s = np.fromfile(f, dtype="<f8", count=nn).reshape((n, n), order="F")
        out = {"n": n, "h": np.asfortranarray(h), "s": np.asfortranarray(s)}
        if size > base:
            out["e"] = np.fromfile(f, dtype="<f8", count=n)
            out["c"] = np.asfortranarray(np.fromfile(f, dtype="<f8", count=nn).reshape((n, n), order="F"))
    return out


def write_hs_bin(path: str, h, s, e=None, c=None) -> None:
    """Write a dump in the same format (e and c together or neither)."""
    h = np.asarray(h, dtype="<f8")
    s = np.asarray(s, dtype="<f8")
    n = h.shape[0]
    if h.shape != (n, n) or s.shape != (n, n):
        raise ValueError("h and s must be n x n")
    if (e is None) != (c is None):
        raise ValueError("e and c are written together")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(np.asfortranarray(h).tobytes(order="F"))
        f.write(np.asfortranarray(s).tobytes(order="F"))
        if e is not None:
            f.write(np.asarray(e, dtype="<f8").tobytes())
            f.write(np.asfortranarray(np.asarray(c, dtype="<f8")).tobytes(order="F"))
