"""Host-side pieces of bench.py that need no GPU: the reference CPU baseline
(a measured full workload layer through the reference module) and the
kind-mixing order the reference arm walks."""
from __future__ import annotations

import os
import sys

import pytest

from doki_b200 import workloads as W
from tests.conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_gate_kinds_and_stratified_order():
    c = W.scale_circuit(seed=2, n=30, depth=40, keep=10)
    ops = bench.layer_ops(c)
    kinds = [bench.gate_kind(op) for op in ops]
    assert kinds.count("cond") == 2 and kinds.count("pair") == 15 and kinds.count("u3") == 28
    order = bench.stratified_order(ops)
    assert sorted(order) == list(range(len(ops)))
    # the conditioned gates lead, then pairs and U3s alternate
    assert [kinds[i] for i in order[:6]] == ["cond", "cond", "pair", "u3", "pair", "u3"]


def test_cpu_baseline_measures_a_whole_layer():
    from oracle import oracle as O
    if not O.have_reference():
        pytest.skip("reference module not built (oracle/_ref)")
    c = W.scale_circuit(seed=2, n=12, depth=3, keep=10)
    cb = bench.cpu_baseline(12, c)
    assert cb["kind"] == "reference" and cb["cores"] == (os.cpu_count() or 1)
    assert cb["layer"]["gates"] == len(bench.layer_ops(c))
    assert cb["value"] > 0 and cb["one_thread"]["cores"] == 1
    assert "measured whole" in cb["sample"]


def test_plain_rate_scales_by_qubit_count():
    """One-at-a-time throughput from per-size means: 3 requests of 10 qubits
    at 1 s and 1 of 20 qubits at 5 s take 8 s for 4 requests."""
    per_n = {10: [0.5, 1.5], 20: [5.0]}
    assert abs(bench.plain_rate(per_n, {10: 3, 20: 1}) - 4 / 8.0) < 1e-12
    # a size without a sample borrows the nearest measured size
    assert abs(bench.plain_rate(per_n, {11: 2}) - 2 / 2.0) < 1e-12
