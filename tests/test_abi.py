"""The C-ABI library loads and exports what include/xtb_eig.h declares (CPU only: no compute call is made)."""
import ctypes
import os
import re
import subprocess

import pytest

import xtbeig

# The eight symbols of xtb's src/mctc/lapack/sytrd.c that the reference re-exports
# (Sources/Diagonalization/Exports.swift:8-138).
XTB_SYTRD_ABI = [
    "xtb_dsytrd_upper", "xtb_ssytrd_upper", "xtb_dsytrd_full", "xtb_dormtr_upper", "xtb_sormtr_upper",
    "xtb_dstedc", "xtb_sstedc", "xtb_dsymmetrize_pad",
]


def test_library_built_in_tree():
    assert os.path.exists(xtbeig.LIB_PATH), "run xtb-diagonalization_b200/build.py"


def test_header_declares_xtb_abi():
    syms = xtbeig.header_symbols()
    for s in XTB_SYTRD_ABI:
        assert s in syms


def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(xtbeig.LIB_PATH)
    missing = [s for s in xtbeig.header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_exports_are_unmangled_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", xtbeig.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (xtb_\w+)$", out, flags=re.M))
    assert set(xtbeig.header_symbols()) <= exported


def test_fortran_signatures_match_reference_arity():
    # Arity of each reference export (Exports.swift): sytrd 7, ormtr 8, stedc 10, symmetrize_pad 5.
    text = open(xtbeig.HEADER).read()
    arity = {"xtb_dsytrd_upper": 7, "xtb_ssytrd_upper": 7, "xtb_dsytrd_full": 7, "xtb_dormtr_upper": 8,
             "xtb_sormtr_upper": 8, "xtb_dstedc": 10, "xtb_sstedc": 10, "xtb_dsymmetrize_pad": 5}
    for name, k in arity.items():
        m = re.search(name + r"\s*\(([^;]*)\);", text, flags=re.S)
        assert m, name
        assert len(m.group(1).split(",")) == k, name


def test_options_roundtrip_without_gpu():
    xtbeig.set_option("ormtr_nb", 96)
    assert xtbeig.get_option("ormtr_nb") == 96
    xtbeig.set_option("ormtr_nb", 128)
    with pytest.raises(KeyError):
        xtbeig.set_option("no_such_option", 1)
    assert "sm_100a" in xtbeig.version()


def test_wait_limit_and_test_hook_option_ranges_without_gpu():
    """"wait_limit_ms" takes 1 .. 600000: a wait that gives up at once or never would defeat the limit."""
    old = xtbeig.get_option("wait_limit_ms")
    try:
        for bad in (0, -1, -1000, 600001):
            with pytest.raises(ValueError):
                xtbeig.set_option("wait_limit_ms", bad)
        assert xtbeig.get_option("wait_limit_ms") == old
        xtbeig.set_option("wait_limit_ms", 1)
        assert xtbeig.get_option("wait_limit_ms") == 1
    finally:
        xtbeig.set_option("wait_limit_ms", old)
    assert xtbeig.get_option("test_barrier_stall") == 0
    with pytest.raises(ValueError):
        xtbeig.set_option("test_barrier_stall", 2)


def test_sytrd_tail_option_range_without_gpu():
    """Option "sytrd_tail": the order of the trailing block finished on one CTA, 0 (off) to 128 in steps of 16."""
    old = xtbeig.get_option("sytrd_tail")
    try:
        for good in (0, 16, 64, 128):
            xtbeig.set_option("sytrd_tail", good)
            assert xtbeig.get_option("sytrd_tail") == good
        for bad in (-16, 50, 144):
            with pytest.raises(ValueError):
                xtbeig.set_option("sytrd_tail", bad)
    finally:
        xtbeig.set_option("sytrd_tail", old)
