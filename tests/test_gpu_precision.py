"""Precision form on the GPU: complex64 registers with FP64 reductions track
the complex128 path layer by layer (fidelity >= 1 - 1e-6)."""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import precision as P
from doki_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_per_layer_fidelity(dk_gpu):
    out = P.run(dk_gpu, n=16, depth=12, seed=3)
    assert len(out["layers"]) == 12
    assert out["worst"]["min_fidelity"] > 1 - 1e-6
    assert out["worst"]["max_amp_err"] < 5e-5
    assert out["worst"]["max_prob_err"] < 5e-6
    # the fused whole-circuit runs (no per-layer flush) agree as well
    assert out["fused_final"]["fidelity"] > 1 - 1e-6
    assert out["c64_layers_per_s_fused"] > 0 and out["c128_layers_per_s_fused"] > 0


def test_compare_matches_host_computation(dk_gpu):
    d = dk_gpu
    c = W.small_circuit(seed=8, n=12, depth=6)
    a = W.run_ops(d, d.registry_new(12, False, 1), c.ops)
    b = W.run_ops(d, d.registry_new(12, False, 2), c.ops)
    fid, err = d.registry_compare(a, b)
    va, vb = d.registry_get_all(a), d.registry_get_all(b)
    assert abs(fid - abs(np.vdot(va, vb)) ** 2) < 1e-12
    assert abs(err - np.max(np.abs(va - vb))) < 1e-12
    same, zero = d.registry_compare(b, b)
    assert abs(same - 1) < 1e-12 and zero == 0
