"""Seeded synthetic circuits for the Doki state-vector engine.

Every workload is drawn from ``numpy.random.default_rng(SeedSequence(seed))``,
the generator the reference tests use (reference ``tests/timed_test.py:69-71``),
so any doki-API engine can replay identical gates, qubit choices and
measurement rolls.

A circuit is a list of :class:`Op` (a dense 2^k x 2^k gate, its targets with
``targets[0]`` the least significant bit of the gate index, and the control /
anticontrol sets), exactly the arguments of ``registry_apply``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
from numpy.random import SeedSequence

X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
H = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2.0)


def u3(theta: float, phi: float, lam: float) -> np.ndarray:
    """IBM U3(theta, phi, lambda)."""
    c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
    return np.array([[c, -np.exp(1j * lam) * s],
                     [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]],
                    dtype=np.complex128)


@dataclass
class Op:
    gate: np.ndarray
    targets: List[int]
    controls: set = field(default_factory=set)
    anticontrols: set = field(default_factory=set)

    @property
    def k(self) -> int:
        return len(self.targets)


@dataclass
class Circuit:
    num_qubits: int
    ops: List[Op]
    layer_starts: List[int]  # index into ops where each layer begins
    rolls: np.ndarray  # measurement draws in [0, 1)
    measure_mask: int = 0
    keep_qubits: Optional[Sequence[int]] = None  # partial-trace survivors

    @property
    def depth(self) -> int:
        return len(self.layer_starts)


def rng_for(seed: int) -> np.random.Generator:
    return np.random.default_rng(SeedSequence(seed))


def _random_u3(rng) -> np.ndarray:
    return u3(*(rng.random(3) * 2.0 * np.pi))


def small_circuit(seed: int = 1, n: int = 12, depth: int = 20) -> Circuit:
    """Plain method, CPU-runnable case: each layer is U3(theta, phi, lambda ~
    U[0, 2pi)) on every qubit, CNOT on a random disjoint pairing, and one
    Toffoli (X target, two random controls, one of them an anticontrol).
    Followed by all single-qubit probabilities and a full measurement."""
    rng = rng_for(seed)
    ops: List[Op] = []
    starts = []
    for _ in range(depth):
        starts.append(len(ops))
        for q in range(n):
            ops.append(Op(_random_u3(rng), [q]))
        perm = [int(x) for x in rng.permutation(n)]
        for a in range(0, n - 1, 2):
            ops.append(Op(X.copy(), [perm[a + 1]], {perm[a]}))
        if n >= 3:
            t, c, ac = (int(x) for x in rng.choice(n, size=3, replace=False))
            ops.append(Op(X.copy(), [t], {c}, {ac}))
    rolls = rng.random(n)
    return Circuit(n, ops, starts, rolls, measure_mask=(1 << n) - 1)


def scale_circuit(seed: int = 2, n: int = 30, depth: int = 40,
                  ctrl_frac: float = 0.05, n_measure: int = 4,
                  keep: int = 10) -> Circuit:
    """Plain method at scale: per layer U3 on all qubits (angles ~ U[0, 2pi)),
    then a CZ/CNOT brickwork on (q, q+1) pairs starting at offset layer % 2;
    a fraction ``ctrl_frac`` of the gates gain 1-3 random extra controls /
    anticontrols.  Ends with all marginals, measurement of ``n_measure``
    random qubits and a partial trace down to qubits 0..keep-1."""
    rng = rng_for(seed)
    ops: List[Op] = []
    starts = []
    for layer in range(depth):
        starts.append(len(ops))
        layer_ops: List[Op] = []
        for q in range(n):
            layer_ops.append(Op(_random_u3(rng), [q]))
        for a in range(layer % 2, n - 1, 2):
            g = X if rng.random() < 0.5 else Z
            t, c = (a, a + 1) if rng.random() < 0.5 else (a + 1, a)
            layer_ops.append(Op(g.copy(), [t], {c}))
        for op in layer_ops:
            if rng.random() < ctrl_frac:
                used = set(op.targets) | op.controls | op.anticontrols
                free = [q for q in range(n) if q not in used]
                extra = int(rng.integers(1, 4))
                for q in rng.choice(free, size=min(extra, len(free)),
                                    replace=False):
                    (op.controls if rng.random() < 0.5
                     else op.anticontrols).add(int(q))
            ops.append(op)
    mq = rng.choice(n, size=n_measure, replace=False)
    mask = 0
    for q in mq:
        mask |= 1 << int(q)
    rolls = rng.random(n_measure)
    return Circuit(n, ops, starts, rolls, measure_mask=mask,
                   keep_qubits=list(range(keep)))


def batch_circuits(seed: int = 4, count: int = 4096, qmin: int = 4,
                   qmax: int = 16, dmin: int = 10, dmax: int = 50) -> List[Circuit]:
    """Batching form: independent registers with n ~ U[qmin, qmax] and depth
    ~ U[dmin, dmax]; each layer is U3 on every qubit, then CNOTs and
    controlled-U3s on a random disjoint pairing."""
    rng = rng_for(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(qmin, qmax + 1))
        depth = int(rng.integers(dmin, dmax + 1))
        ops: List[Op] = []
        starts = []
        for _layer in range(depth):
            starts.append(len(ops))
            for q in range(n):
                ops.append(Op(_random_u3(rng), [q]))
            perm = [int(x) for x in rng.permutation(n)]
            for a in range(0, n - 1, 2):
                if rng.random() < 0.5:
                    ops.append(Op(X.copy(), [perm[a + 1]], {perm[a]}))
                else:
                    ops.append(Op(_random_u3(rng), [perm[a + 1]], {perm[a]}))
        out.append(Circuit(n, ops, starts, np.zeros(0),
                           keep_qubits=list(range(n // 2))))
    return out


def run_ops(mod, reg, ops: Sequence[Op], gate_cache=None, num_threads=-1):
    """Replay ``ops`` through any doki-API module; returns the last register.
    Intermediate registers are released as soon as they are replaced."""
    for op in ops:
        g = mod.gate_new(op.k, op.gate.tolist(), False)
        # the reference rejects anticontrols when the control set is None
        ctl = set(op.controls) if (op.controls or op.anticontrols) else None
        new = mod.registry_apply(reg, g, list(op.targets), ctl,
                                 set(op.anticontrols) or None,
                                 num_threads, False)
        reg = new
    return reg
