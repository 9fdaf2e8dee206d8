"""Allocation-free marginals (dk_marginals_noalloc), on the GPU.

This entry point exists for callers that cannot let the library allocate
device memory -- a framework that owns every device byte through its own
allocator or an HBM-budget arena, or a latency-critical loop where a
cudaMalloc / cudaFree would synchronise the device.  The caller owns the
amplitude array and the output array; the scratch is a fixed device array
inside the library.  Its results must agree with the allocating
dk_marginals on the same amplitudes, call after call (the fixed scratch keeps
the previous call's contents).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from tests.conftest import ATOL_C128, ROOT

pytestmark = pytest.mark.gpu

DK_ERR_NOALLOC_LIMIT = 28


def noalloc_lib():
    lib = ctypes.CDLL(os.path.join(ROOT, "doki_b200", "libdokigpu.so"))
    lib.dk_marginals_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]
    lib.dk_marginals_noalloc.restype = ctypes.c_int
    return lib


def random_state(rng, n):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def torch_marginals(amps, n):
    """Plain PyTorch FP64 restatement of the reduction: out[q] = sum of
    |a_i|^2 over i with bit q set, out[n] = the total."""
    import torch
    p = amps.to(torch.complex128).abs().pow(2)
    out = [p.view(1 << (n - 1 - q), 2, 1 << q)[:, 1, :].sum().item() for q in range(n)]
    return np.array(out + [p.sum().item()])


@pytest.mark.parametrize("precision", [2, 1])
def test_noalloc_marginals_match_allocating_entry_point(dk_gpu, precision):
    import torch

    d = dk_gpu
    lib = noalloc_lib()
    rng = np.random.default_rng(2024 + precision)
    host_dtype = np.complex128 if precision == 2 else np.complex64
    stream = torch.cuda.current_stream().cuda_stream
    tol = ATOL_C128 if precision == 2 else 1e-6
    # calls in a row, different sizes: leftover scratch must not leak in.
    # n = 3 and 6 run one warp with idle lanes; 17 and 20 the block-limited
    # grid with 12 accumulated bits per thread.
    for n in (20, 3, 17, 6):
        v = random_state(rng, n)
        host = np.ascontiguousarray(v.astype(host_dtype))
        amps = torch.from_numpy(host.view(np.float64 if precision == 2 else np.float32)).cuda()
        out = torch.full((n + 1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.dk_marginals_noalloc(amps.data_ptr(), n, precision, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # the allocating entry point on a register holding the same values
        reg = d.registry_new_data(n, host.astype(np.complex128), False, precision)
        want = np.array(d.registry_probs(reg))  # norm = 1: raw sums, as the reference
        assert np.allclose(got[:n], want, atol=tol, rtol=0)
        # and numpy on the stored values, qubit by qubit
        stored = np.abs(host.astype(np.complex128)) ** 2
        idx = np.arange(1 << n)
        for q in range(n):
            assert abs(got[q] - stored[(idx >> q) & 1 == 1].sum()) < tol, (n, q)
        assert abs(got[n] - stored.sum()) < tol


def test_noalloc_marginals_wide_accumulators(dk_gpu):
    """29 qubits complex64 (4 GiB): 256 blocks of 256 threads leave 13 bits
    per thread, the kernel variant with 16 accumulators.  Checked against a
    plain PyTorch FP64 reduction of the same device array, twice in a row."""
    import torch

    lib = noalloc_lib()
    n = 29
    gen = torch.Generator(device="cuda").manual_seed(29)
    amps = torch.randn(1 << n, dtype=torch.complex64, device="cuda", generator=gen)
    amps /= amps.abs().pow(2).sum().sqrt()
    want = torch_marginals(amps, n)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((n + 1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.dk_marginals_noalloc(amps.data_ptr(), n, 1, out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.allclose(out.cpu().numpy(), want, atol=1e-9, rtol=0)
    del amps
    torch.cuda.empty_cache()


def test_noalloc_rejects_oversized_registers():
    lib = noalloc_lib()
    out = ctypes.c_double * 64
    buf = out()
    # rejected before any device work: the pointers are never dereferenced
    rc = lib.dk_marginals_noalloc(ctypes.addressof(buf), 41, 2, ctypes.addressof(buf), None)
    assert rc == DK_ERR_NOALLOC_LIMIT
