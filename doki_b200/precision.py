"""Precision form: complex64 amplitudes with FP64 norms, reductions and
collapse renormalisation, checked layer by layer against a complex128
register running the same circuit on the same device.

For every layer the fidelity |<psi64|psi128>|^2 of the logical states, the
largest amplitude error and the largest single-qubit probability error are
recorded (all computed on the device in FP64)."""
from __future__ import annotations

import time
from typing import Dict, List

import numpy as np

from . import workloads as W


def run(d, n: int = 32, depth: int = 60, seed: int = 1, per_layer: bool = True,
        fused: bool = True) -> Dict:
    """The circuit layer by layer on both registers (each layer flushed and
    synchronised so it can be compared: `*_layers_per_s_flushed_each_layer`
    counts that serialised run), then, when `fused`, the whole circuit once
    per precision with no intermediate read, so the planner fuses across
    layers as a plain run does (`*_layers_per_s_fused`, host time from the
    first queued gate to the flushed register), and the fidelity of those two
    final states."""
    c = W.small_circuit(seed=seed, n=n, depth=depth)
    starts = list(c.layer_starts) + [len(c.ops)]
    r64 = d.registry_new(n, False, 1)
    r128 = d.registry_new(n, False, 2)
    layers: List[Dict] = []
    t64 = t128 = 0.0
    for layer in range(depth):
        ops = c.ops[starts[layer]:starts[layer + 1]]
        t0 = time.perf_counter()
        r64 = W.run_ops(d, r64, ops)
        d.registry_flush(r64)
        d.engine_sync()
        t1 = time.perf_counter()
        r128 = W.run_ops(d, r128, ops)
        d.registry_flush(r128)
        d.engine_sync()
        t2 = time.perf_counter()
        t64 += t1 - t0
        t128 += t2 - t1
        if per_layer or layer == depth - 1:
            fid, err = d.registry_compare(r64, r128)
            p64 = np.array(d.registry_probs(r64))
            p128 = np.array(d.registry_probs(r128))
            layers.append({"layer": layer, "fidelity": fid, "max_amp_err": err,
                           "max_prob_err": float(np.max(np.abs(p64 - p128)))})
    worst = {"min_fidelity": min(x["fidelity"] for x in layers),
             "max_amp_err": max(x["max_amp_err"] for x in layers),
             "max_prob_err": max(x["max_prob_err"] for x in layers)}
    out = {"qubits": n, "depth": depth, "gates": len(c.ops), "layers": layers,
           "worst": worst, "c64_layers_per_s_flushed_each_layer": depth / t64,
           "c128_layers_per_s_flushed_each_layer": depth / t128}
    if fused:
        del r64, r128
        regs, rate = {}, {}
        for prec, name in ((1, "c64"), (2, "c128")):
            d.engine_sync()
            t0 = time.perf_counter()
            r = W.run_ops(d, d.registry_new(n, False, prec), c.ops)
            d.registry_flush(r)
            d.engine_sync()
            rate[name] = depth / (time.perf_counter() - t0)
            regs[name] = r
        fid, err = d.registry_compare(regs["c64"], regs["c128"])
        out.update({"c64_layers_per_s_fused": rate["c64"],
                    "c128_layers_per_s_fused": rate["c128"],
                    "fused_final": {"fidelity": fid, "max_amp_err": err}})
    return out
