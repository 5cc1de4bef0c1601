"""Test configuration: the `gpu` marker and import paths.

CPU tests (`-m "not gpu"`) check the oracle against known-answer spectra and the golden fixtures, and that the C-ABI
library loads and exports every symbol include/xtb_eig.h declares.  GPU tests (`-m gpu`) call the library through its
C ABI and compare with the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "xtb-diagonalization_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); calls the library through its C ABI")


@pytest.fixture(scope="session")
def xe():
    import xtbeig

    xtbeig.lib()
    return xtbeig
