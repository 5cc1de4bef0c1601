"""The H/S dump format (reference Sources/EigenBench/main.swift:159-174, scripts/kernels/refine.f90:64-83): round trips
with and without the per-cycle eigenpairs, column-major layout, and rejection of truncated files."""
import os
import struct

import numpy as np
import pytest

import hsbin
from oracle import inputs


def test_round_trip_h_s(tmp_path):
    h, s, _ = inputs.generalized(37, seed=3)
    p = os.path.join(tmp_path, "HS.bin")
    hsbin.write_hs_bin(p, h, s)
    assert os.path.getsize(p) == 4 + 16 * 37 * 37
    d = hsbin.read_hs_bin(p)
    assert d["n"] == 37 and "e" not in d
    np.testing.assert_array_equal(d["h"], h)
    np.testing.assert_array_equal(d["s"], s)


def test_round_trip_cycle_file_and_layout(tmp_path):
    n = 5
    h = np.arange(n * n, dtype=float).reshape(n, n)
    h = h + h.T
    s = np.eye(n)
    e = np.linspace(-1, 1, n)
    c = np.arange(n * n, dtype=float).reshape(n, n, order="F")
    p = os.path.join(tmp_path, "cycle_3.bin")
    hsbin.write_hs_bin(p, h, s, e, c)
    raw = open(p, "rb").read()
    assert struct.unpack("<i", raw[:4])[0] == n
    # column-major: the second stored double of H is H[1, 0]
    assert struct.unpack("<d", raw[12:20])[0] == h[1, 0]
    d = hsbin.read_hs_bin(p)
    np.testing.assert_array_equal(d["e"], e)
    np.testing.assert_array_equal(d["c"], c)


def test_truncated_file_rejected(tmp_path):
    p = os.path.join(tmp_path, "bad.bin")
    with open(p, "wb") as f:
        f.write(struct.pack("<i", 4) + b"\0" * 100)
    with pytest.raises(ValueError):
        hsbin.read_hs_bin(p)
