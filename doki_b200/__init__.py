"""B200 state-vector engine behind the `doki` module API.

``doki_b200.doki`` is a CPython extension with the reference ``doki`` module's
functions (registry_*, gate_*, funmatrix_*), backed by ``libdokigpu.so``
(C ABI in ``include/dokigpu.h``): hand-written sm_100a kernels with the state
vector resident in device memory.  There is no CPU fallback: importing the
module fails when the compiled library is missing.

To use it as a drop-in for ``import doki``, put this package directory on
``sys.path`` (see :func:`install_as_doki`).
"""
from __future__ import annotations

import importlib
import os
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    """Import and return the compiled ``doki`` extension of this package."""
    try:
        return importlib.import_module("doki_b200.doki")
    except ImportError as e:  # pragma: no cover - message only
        raise ImportError(
            "doki_b200: compiled extension missing; run `python -m doki_b200.build`"
        ) from e


def install_as_doki():
    """Make ``import doki`` resolve to this engine; returns the module."""
    mod = load()
    sys.modules["doki"] = mod
    return mod


def lib_path() -> str:
    return os.path.join(_HERE, "libdokigpu.so")
