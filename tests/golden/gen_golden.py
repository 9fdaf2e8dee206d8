"""Generate the golden fixtures in this directory from the reference module.

The reference Doki extension is compiled from its own sources into
oracle/_ref/ (``make -C oracle ref``, needs the reference tree mounted).  This
script replays seeded workloads through it and stores inputs + outputs as
compressed .npz files, so the tests can pin both the CPU oracle and the CUDA
engine against reference outputs on machines where the reference is absent.

Run from the repository root:  python tests/golden/gen_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from doki_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ops_digest(ops) -> str:
    h = hashlib.sha256()
    for op in ops:
        h.update(np.ascontiguousarray(op.gate).tobytes())
        h.update(repr((list(op.targets), sorted(op.controls),
                       sorted(op.anticontrols))).encode())
    return h.hexdigest()


def get_all(d, reg, n, canonical=False):
    return np.array([d.registry_get(reg, i, canonical, False)
                     for i in range(1 << n)], dtype=np.complex128)


def random_unitary(rng, k):
    z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def main():
    d = O.reference_module()
    out = {}

    # 1. the CPU-runnable plain-method workload (12 qubits, depth 20)
    c = W.small_circuit(seed=1, n=12, depth=20)
    reg = W.run_ops(d, d.registry_new(12, False), c.ops)
    out["small12_digest"] = np.frombuffer(ops_digest(c.ops).encode(), dtype=np.uint8)
    out["small12_amps"] = get_all(d, reg, 12)
    out["small12_probs"] = np.array([d.registry_prob(reg, q, 1, False)
                                     for q in range(12)])
    out["small12_rolls"] = c.rolls
    _, res = d.registry_measure(reg, (1 << 12) - 1, c.rolls.tolist(), 1, False)
    out["small12_measure_all"] = np.array([-1 if v is None else int(v) for v in res])
    half_mask = 0b101100100110
    half_rolls = c.rolls[:bin(half_mask).count("1")]
    r2, res2 = d.registry_measure(reg, half_mask, half_rolls.tolist(), 1, False)
    out["small12_half_mask"] = np.array([half_mask])
    out["small12_half_rolls"] = half_rolls
    out["small12_half_res"] = np.array([-1 if v is None else int(v) for v in res2])
    out["small12_half_amps"] = get_all(d, r2, 12 - bin(half_mask).count("1"), True)

    # 2. one-qubit U3 on every qubit in turn (one_gate_tests.py pattern)
    rng = W.rng_for(11)
    for n in range(1, 7):
        reg = d.registry_new(n, False)
        angs = []
        for q in range(n):
            a = np.pi * (rng.random(3) * 2 - 1)
            angs.append(a)
            reg = d.registry_apply(reg, d.gate_new(1, W.u3(*a).tolist(), False),
                                   [q], None, None, 1, False)
        out[f"one_{n}_angles"] = np.array(angs)
        out[f"one_{n}_amps"] = get_all(d, reg, n)

    # 3. growing alternating control / anticontrol sets (multiple_gate_tests.py)
    rng = W.rng_for(12)
    n = 7
    order = [int(x) for x in rng.permutation(n)]
    ang = rng.random(3)
    g = d.gate_new(1, W.u3(*ang).tolist(), False)
    reg = d.registry_apply(d.registry_new(n, False), g, [order[0]], None, None, 1, False)
    ctl, act = [], []
    is_c = True
    for prev, q in zip(order, order[1:]):
        (ctl if is_c else act).append(prev)
        reg = d.registry_apply(reg, g, [q], set(ctl), set(act), 1, False)
        is_c = not is_c
    out["ctrl_order"] = np.array(order)
    out["ctrl_angles"] = ang
    out["ctrl_amps"] = get_all(d, reg, n)

    # 4. dense two-qubit gate on every ordered pair, each from a random state
    rng = W.rng_for(13)
    n = 5
    base_ops = [W.Op(W.u3(*(rng.random(3) * 2 * np.pi)), [q]) for q in range(n)]
    u2 = random_unitary(rng, 2)
    out["pair_base"] = np.array([op.gate for op in base_ops])
    out["pair_u"] = u2
    start = W.run_ops(d, d.registry_new(n, False), base_ops)
    amps = []
    for a in range(n):
        for b in range(n):
            if a != b:
                r = d.registry_apply(start, d.gate_new(2, u2.tolist(), False), [a, b],
                                     None, None, 1, False)
                amps.append(get_all(d, r, n))
    out["pair_amps"] = np.array(amps)

    # 5. three-qubit dense gates, a diagonal two-qubit gate, controls on them
    rng = W.rng_for(14)
    n = 6
    u3q = random_unitary(rng, 3)
    diag2 = np.diag(np.exp(1j * rng.random(4) * 2 * np.pi))
    reg = W.run_ops(d, d.registry_new(n, False),
                    [W.Op(W.u3(*(rng.random(3) * 2 * np.pi)), [q]) for q in range(n)])
    seq = [(u3q, [4, 0, 2], set(), set()), (diag2, [1, 5], {3}, set()),
           (u3q, [5, 3, 1], set(), {0}), (u3q, [0, 1, 2], {5}, {4})]
    for m, tg, cs, acs in seq:
        reg = d.registry_apply(reg, d.gate_new(len(tg), m.tolist(), False), tg,
                               cs if (cs or acs) else None, acs or None, 1, False)
    out["k3_u"] = u3q
    out["k3_diag2"] = diag2
    out["k3_base_seed"] = np.array([14])
    out["k3_amps"] = get_all(d, reg, n)

    # 6. join (join_regs_tests.py): one-qubit registers joined left to right
    rng = W.rng_for(15)
    n = 5
    gates = [W.u3(*(np.pi * (rng.random(3) * 2 - 1))) for _ in range(n)]
    regs = [d.registry_apply(d.registry_new(1, False), d.gate_new(1, gm.tolist(), False),
                             [0], None, None, 1, False) for gm in gates]
    res = regs[0]
    for r in regs[1:]:
        res = d.registry_join(res, r, 1, False)
    out["join_gates"] = np.array(gates)
    out["join_amps"] = get_all(d, res, n)

    # 7. density matrix and chained partial traces of an 8-qubit state
    c8 = W.small_circuit(seed=16, n=8, depth=6)
    reg = W.run_ops(d, d.registry_new(8, False), c8.ops)
    rho = d.registry_density(reg, False)
    out["rho8_digest"] = np.frombuffer(ops_digest(c8.ops).encode(), dtype=np.uint8)
    out["rho8_diag"] = np.array([d.funmatrix_get(rho, i, i, False) for i in range(256)])
    out["rho8_row5"] = np.array([d.funmatrix_get(rho, 5, j, False) for j in range(256)])
    pt = rho
    elems = [7, 3, 0]
    for e in elems:
        pt = d.funmatrix_partialtrace(pt, e, False)
    out["rho8_elems"] = np.array(elems)
    out["rho8_ptrace"] = np.array([[d.funmatrix_get(pt, i, j, False) for j in range(32)]
                                   for i in range(32)])
    out["rho8_ptrace_trace"] = np.array([d.funmatrix_trace(pt, False)])
    pt2 = rho
    for _ in range(5):
        pt2 = d.funmatrix_partialtrace(pt2, 3, False)
    out["rho8_low3"] = np.array([[d.funmatrix_get(pt2, i, j, False) for j in range(8)]
                                 for i in range(8)])

    # 8. canonical form after phase gates and a measurement
    rng = W.rng_for(17)
    n = 4
    reg = d.registry_new(n, False)
    h = W.H
    for q in range(n):
        ph = np.exp(1j * np.pi * (rng.random() * 2 - 1)) * h
        reg = d.registry_apply(reg, d.gate_new(1, ph.tolist(), False), [q], None, None,
                               1, False)
    out["canon_seed"] = np.array([17])
    out["canon_raw"] = get_all(d, reg, n, False)
    out["canon_amps"] = get_all(d, reg, n, True)
    roll = float(rng.random())
    r2, res = d.registry_measure(reg, 1, [roll], 1, False)
    out["canon_roll"] = np.array([roll])
    out["canon_meas_res"] = np.array([-1 if v is None else int(v) for v in res])
    out["canon_meas_amps"] = get_all(d, r2, n - 1, True)

    # 9. unnormalised data: read back raw, then renormalised by a gate
    vals = np.array([2.0, 1j, -1.0, 0.5 + 0.5j, 0, 0, 3.0, -2j], dtype=np.complex128)
    reg = d.registry_new_data(3, vals, False)
    out["data_vals"] = vals
    out["data_raw"] = get_all(d, reg, 3)
    reg2 = d.registry_apply(reg, d.gate_new(1, W.H.tolist(), False), [1], None, None, 1,
                            False)
    out["data_after_h"] = get_all(d, reg2, 3)
    out["data_prob"] = np.array([d.registry_prob(reg, q, 1, False) for q in range(3)])

    np.savez_compressed(os.path.join(OUT, "reference_cases.npz"), **out)
    print("wrote", os.path.join(OUT, "reference_cases.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
