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


@dataclass
class FlatBatch:
    """A batch of circuits as flat arrays (the layout of dk_batch_build)."""
    num_qubits: np.ndarray  # uint32 [C]
    keep: np.ndarray  # uint32 [C]
    op_start: np.ndarray  # uint64 [C + 1]
    op_k: np.ndarray  # uint32 [N]
    op_targets: np.ndarray  # uint32 [N, 3]
    op_controls: np.ndarray  # uint64 [N]
    op_anticontrols: np.ndarray  # uint64 [N]
    op_matrix: np.ndarray  # uint64 [N]: first complex entry of the op's matrix
    matrices: np.ndarray  # complex128 [M]

    @property
    def count(self) -> int:
        return int(self.num_qubits.size)

    def ops(self, c: int) -> List[Op]:
        """Circuit c as a list of Op (for the oracle and the plain path)."""
        out = []
        for i in range(int(self.op_start[c]), int(self.op_start[c + 1])):
            k = int(self.op_k[i])
            m0 = int(self.op_matrix[i])
            mat = self.matrices[m0:m0 + (1 << (2 * k))].reshape(1 << k, 1 << k).copy()
            cm, am = int(self.op_controls[i]), int(self.op_anticontrols[i])
            out.append(Op(mat, [int(t) for t in self.op_targets[i, :k]],
                          {q for q in range(64) if (cm >> q) & 1},
                          {q for q in range(64) if (am >> q) & 1}))
        return out

    def subset(self, idx: Sequence[int]) -> "FlatBatch":
        """The circuits idx as a batch of their own (shares matrices)."""
        starts = [0]
        sel = []
        for c in idx:
            a, b = int(self.op_start[c]), int(self.op_start[c + 1])
            sel.append(np.arange(a, b))
            starts.append(starts[-1] + (b - a))
        ops = np.concatenate(sel) if sel else np.zeros(0, dtype=np.int64)
        return FlatBatch(self.num_qubits[list(idx)].copy(), self.keep[list(idx)].copy(),
                         np.array(starts, dtype=np.uint64), self.op_k[ops].copy(),
                         self.op_targets[ops].copy(), self.op_controls[ops].copy(),
                         self.op_anticontrols[ops].copy(), self.op_matrix[ops].copy(),
                         self.matrices)


def _u3_many(angles: np.ndarray) -> np.ndarray:
    th, ph, la = angles[:, 0], angles[:, 1], angles[:, 2]
    c, s = np.cos(th / 2.0), np.sin(th / 2.0)
    m = np.empty((angles.shape[0], 2, 2), dtype=np.complex128)
    m[:, 0, 0] = c
    m[:, 0, 1] = -np.exp(1j * la) * s
    m[:, 1, 0] = np.exp(1j * ph) * s
    m[:, 1, 1] = np.exp(1j * (ph + la)) * c
    return m


def batch_arrays(seed: int = 4, count: int = 4096, qmin: int = 4, qmax: int = 16,
                 dmin: int = 10, dmax: int = 50) -> FlatBatch:
    """Batching form: `count` independent registers with n ~ U[qmin, qmax] and
    depth ~ U[dmin, dmax]; each layer is U3(theta, phi, lambda ~ U[0, 2pi)) on
    every qubit, then, on a random disjoint pairing, a CNOT or a controlled
    U3 (probability 1/2 each).  The reduced density matrix is taken over the
    lower floor(n / 2) qubits."""
    rng = rng_for(seed)
    ns = rng.integers(qmin, qmax + 1, size=count)
    depths = rng.integers(dmin, dmax + 1, size=count)
    mats = [X.reshape(-1)]  # entry 0..3: the shared X matrix
    moff = 4
    ks, tgs, cms, mat_idx, starts = [], [], [], [], [0]
    for c in range(count):
        n, d = int(ns[c]), int(depths[c])
        npairs = n // 2
        # per layer: n U3 on qubits 0..n-1, then npairs controlled ops
        u3s = _u3_many(rng.random((d * n, 3)) * 2.0 * np.pi)
        perms = np.argsort(rng.random((d, n)), axis=1)
        coin = rng.random((d, npairs)) < 0.5
        cu = _u3_many(rng.random((d * npairs, 3)) * 2.0 * np.pi)
        layer_ops = n + npairs
        tot = d * layer_ops
        tg = np.zeros((tot, 3), dtype=np.uint32)
        cm = np.zeros(tot, dtype=np.uint64)
        mi = np.zeros(tot, dtype=np.uint64)
        base = np.arange(d) * layer_ops
        # U3 on every qubit
        u_idx = (base[:, None] + np.arange(n)[None, :]).reshape(-1)
        tg[u_idx, 0] = np.tile(np.arange(n, dtype=np.uint32), d)
        mi[u_idx] = moff + 4 * np.arange(d * n, dtype=np.uint64)
        mats.append(u3s.reshape(-1))
        moff += 4 * d * n
        # controlled ops on the pairing (control perm[2a], target perm[2a+1])
        p_idx = (base[:, None] + n + np.arange(npairs)[None, :]).reshape(-1)
        ctl = perms[:, 0:2 * npairs:2].reshape(-1)
        tgt = perms[:, 1:2 * npairs:2].reshape(-1)
        tg[p_idx, 0] = tgt.astype(np.uint32)
        cm[p_idx] = (np.uint64(1) << ctl.astype(np.uint64))
        flat_coin = coin.reshape(-1)
        mi[p_idx] = np.where(flat_coin, 0,
                             moff + 4 * np.arange(d * npairs, dtype=np.uint64)).astype(np.uint64)
        mats.append(cu.reshape(-1))
        moff += 4 * d * npairs
        ks.append(np.ones(tot, dtype=np.uint32))
        tgs.append(tg)
        cms.append(cm)
        mat_idx.append(mi)
        starts.append(starts[-1] + tot)
    n_ops = starts[-1]
    return FlatBatch(ns.astype(np.uint32), (ns // 2).astype(np.uint32),
                     np.array(starts, dtype=np.uint64), np.concatenate(ks),
                     np.concatenate(tgs), np.concatenate(cms), np.zeros(n_ops, dtype=np.uint64),
                     np.concatenate(mat_idx), np.concatenate(mats).astype(np.complex128))


@dataclass
class FlatCircuit:
    """One circuit as the flat arrays of registry_apply_many / dk_apply_gates."""
    num_qubits: int
    op_k: np.ndarray  # uint32 [N]
    op_targets: np.ndarray  # uint32 [N, 3]
    op_controls: np.ndarray  # uint64 [N]
    op_anticontrols: np.ndarray  # uint64 [N]
    op_matrix: np.ndarray  # uint64 [N]
    matrices: np.ndarray  # complex128 [M]
    rolls: np.ndarray

    def arrays(self):
        return (self.op_k, self.op_targets, self.op_controls, self.op_anticontrols,
                self.op_matrix, self.matrices)

    @property
    def count(self) -> int:
        return int(self.op_k.size)


def small_circuit_flat(seed: int = 1, n: int = 12, depth: int = 20) -> FlatCircuit:
    """small_circuit(seed, n, depth) as flat arrays, drawn from the same
    seeded stream (three generator calls per layer instead of n + 2, so
    thousands of circuits can be prepared ahead of a serving run): the gates,
    qubit choices and rolls are the same; the U3 matrices are computed in
    one vectorised pass (equal to u3() up to the last bit of the libm
    functions)."""
    rng = rng_for(seed)
    npairs = n // 2
    per_layer = n + npairs + (1 if n >= 3 else 0)
    tot = depth * per_layer
    k = np.ones(tot, dtype=np.uint32)
    tg = np.zeros((tot, 3), dtype=np.uint32)
    cm = np.zeros(tot, dtype=np.uint64)
    am = np.zeros(tot, dtype=np.uint64)
    mi = np.zeros(tot, dtype=np.uint64)
    angles = np.empty((depth, n, 3))
    one = np.uint64(1)
    for layer in range(depth):
        angles[layer] = rng.random(3 * n).reshape(n, 3) * 2.0 * np.pi
        b = layer * per_layer
        tg[b:b + n, 0] = np.arange(n, dtype=np.uint32)
        mi[b:b + n] = 4 + 4 * (layer * n + np.arange(n, dtype=np.uint64))
        perm = rng.permutation(n)
        p = b + n
        tg[p:p + npairs, 0] = perm[1:2 * npairs:2]
        cm[p:p + npairs] = one << perm[0:2 * npairs:2].astype(np.uint64)
        if n >= 3:
            t, c, ac = (int(x) for x in rng.choice(n, size=3, replace=False))
            i = b + n + npairs
            tg[i, 0] = t
            cm[i] = one << np.uint64(c)
            am[i] = one << np.uint64(ac)
    rolls = rng.random(n)
    mats = np.concatenate([X.reshape(-1), _u3_many(angles.reshape(-1, 3)).reshape(-1)])
    return FlatCircuit(n, k, tg, cm, am, mi, mats.astype(np.complex128), rolls)
