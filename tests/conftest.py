"""Shared test setup.

``-m "not gpu"``: oracle vs golden fixtures, host helpers, ABI exports (no GPU).
``-m gpu``: parity of the CUDA path (through the C ABI) with the oracle and the
golden fixtures on a B200.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def native_lib():
    """Build (if needed) and load liblfts_b200.so."""
    from lfts_cpu_b200 import build, capi
    build.build()
    return capi.lib()


@pytest.fixture(scope="session")
def oracle_built():
    from pyoracle import build_oracle
    build_oracle(ref=False)
    return True


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
