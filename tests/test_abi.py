"""The drop-in boundary on CPU: the C-ABI library loads and exports every
symbol the public headers declare, and the `doki` module exposes the
reference module's API with the same host-side behaviour."""
from __future__ import annotations

import ctypes
import glob
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT

REFERENCE_API = [
    "gate_new", "gate_get", "registry_new", "registry_new_data", "registry_clone",
    "registry_del", "registry_get", "registry_apply", "registry_join",
    "registry_measure", "registry_prob", "registry_density", "registry_mem",
    "funmatrix_create", "funmatrix_identity", "funmatrix_statezero",
    "funmatrix_densityzero", "funmatrix_hadamard", "funmatrix_addcontrol",
    "funmatrix_get", "funmatrix_add", "funmatrix_sub", "funmatrix_scalar_mul",
    "funmatrix_scalar_div", "funmatrix_matmul", "funmatrix_ewmul", "funmatrix_kron",
    "funmatrix_eyekron", "funmatrix_transpose", "funmatrix_dagger",
    "funmatrix_projection", "funmatrix_shape", "funmatrix_partialtrace",
    "funmatrix_trace", "funmatrix_apply", "funmatrix_mem",
]


def header_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(dk_\w+)\s*\(", text))
    return sorted(syms)


def test_library_exports_header_symbols():
    lib = ctypes.CDLL(os.path.join(ROOT, "doki_b200", "libdokigpu.so"))
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_strerror_without_device():
    lib = ctypes.CDLL(os.path.join(ROOT, "doki_b200", "libdokigpu.so"))
    lib.dk_strerror.restype = ctypes.c_char_p
    assert lib.dk_strerror(0) == b"ok"
    assert b"maximum" in lib.dk_strerror(3)


def test_module_api_surface(dk):
    for name in REFERENCE_API:
        assert callable(getattr(dk, name)), name
    assert dk.error.__module__ == "qsimov.doki" and dk.error.__name__ == "error"


def err(f):
    try:
        f()
    except Exception as e:  # noqa: BLE001
        return type(e).__module__ + "." + type(e).__name__, str(e)
    return None


@pytest.mark.parametrize("call", [
    lambda d: d.registry_new(0, False),
    lambda d: d.registry_new(3),
    lambda d: d.gate_new(0, [[0, 1], [1, 0]], False),
    lambda d: d.gate_new(2, [[0, 1], [1, 0]], False),
    lambda d: d.gate_new(1, [[0, 1], [1]], False),
    lambda d: d.gate_new(1, [[0, 1], [1, "a"]], False),
    lambda d: d.gate_new(1, ((0, 1), (1, 0)), False),
    lambda d: d.registry_new_data(2, (1, 0, 0, 0), False),
    lambda d: d.registry_new_data(2, [1, 0, 0], False),
    lambda d: d.registry_get(None, 0, False, False),
    lambda d: d.registry_prob(None, 0, 0, False),
    lambda d: d.registry_measure(None, 0, [], 1, False),
    lambda d: d.funmatrix_get(d.funmatrix_identity(2, False), 4, 0, False),
    lambda d: d.funmatrix_partialtrace(d.funmatrix_identity(2, False), -1, False),
    lambda d: d.funmatrix_create([], False),
    lambda d: d.funmatrix_create([[1, 2], [3]], False),
])
def test_host_side_errors_match_reference(dk, ref, call):
    assert err(lambda: call(dk)) == err(lambda: call(ref))


def test_gate_roundtrip_matches_reference(dk, ref):
    m = [[0.5, 1j], [2, -0.25 + 0.5j]]
    assert dk.gate_get(dk.gate_new(1, m, False), False) == \
        ref.gate_get(ref.gate_new(1, m, False), False)


@pytest.mark.parametrize("ctor,n", [("funmatrix_identity", 3), ("funmatrix_hadamard", 3),
                                    ("funmatrix_statezero", 2),
                                    ("funmatrix_densityzero", 2)])
def test_host_funmatrix_constructors(dk, ref, ctor, n):
    a = getattr(dk, ctor)(n, False)
    b = getattr(ref, ctor)(n, False)
    assert dk.funmatrix_shape(a, False) == ref.funmatrix_shape(b, False)
    r, c = dk.funmatrix_shape(a, False)
    va = np.array([[dk.funmatrix_get(a, i, j, False) for j in range(c)] for i in range(r)])
    vb = np.array([[ref.funmatrix_get(b, i, j, False) for j in range(c)] for i in range(r)])
    assert np.array_equal(va, vb)
    assert dk.funmatrix_trace(a, False) == ref.funmatrix_trace(b, False)


def test_host_funmatrix_custom_cu_ptrace(dk, ref):
    m = [[1, 2j, 0, 1], [3, 4, 5, 6], [0.5, -1, 2, 2], [7, 8, 9, 1j]]
    for mod in (dk, ref):
        pass
    a = dk.funmatrix_addcontrol(dk.funmatrix_create(m, False), False)
    b = ref.funmatrix_addcontrol(ref.funmatrix_create(m, False), False)
    va = np.array([[dk.funmatrix_get(a, i, j, False) for j in range(8)] for i in range(8)])
    vb = np.array([[ref.funmatrix_get(b, i, j, False) for j in range(8)] for i in range(8)])
    assert np.array_equal(va, vb)
    pa = dk.funmatrix_partialtrace(a, 1, False)
    pb = ref.funmatrix_partialtrace(b, 1, False)
    va = np.array([[dk.funmatrix_get(pa, i, j, False) for j in range(4)] for i in range(4)])
    vb = np.array([[ref.funmatrix_get(pb, i, j, False) for j in range(4)] for i in range(4)])
    assert np.array_equal(va, vb)
    assert dk.funmatrix_trace(pa, False) == ref.funmatrix_trace(pb, False)


def test_device_ops_fail_loudly_without_gpu(dk):
    """No CPU fallback: without a device, creating a registry raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    e = err(lambda: dk.registry_new(3, False))
    assert e is not None and e[0] == "qsimov.doki.error"
