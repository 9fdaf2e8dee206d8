"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The oracle (``oracle/``) is the checker only; the module under test is the
compiled ``doki_b200.doki`` extension, which has no CPU fallback.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_cases.npz")

# Tolerances: the reference checks amplitudes at atol 1e-13 (reference
# tests/one_gate_tests.py:76-77); the engine must match the reference CPU path
# to 1e-12 absolute for complex128.
ATOL_C128 = 1e-12
# complex64 storage: amplitudes carry ~6e-8 relative rounding per gate.
ATOL_C64 = 5e-5


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    lib = os.path.join(ROOT, "oracle", "_build", "libdkoracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"],
                       check=True, capture_output=True)
    return O


@pytest.fixture(scope="session")
def orc(oracle_mod):
    return oracle_mod.OracleDoki()


@pytest.fixture(scope="session")
def ref(oracle_mod):
    if not oracle_mod.have_reference():
        pytest.skip("reference module not built (oracle/_ref)")
    return oracle_mod.reference_module()


@pytest.fixture(scope="session")
def dk():
    """The engine under test (compiled extension; fails loudly if absent)."""
    import doki_b200
    return doki_b200.load()


@pytest.fixture(scope="session")
def dk_gpu(dk):
    """The engine on a live device: a registry must be creatable."""
    r = dk.registry_new(1, False)
    del r
    return dk
