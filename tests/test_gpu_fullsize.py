"""Full-size checks at 30 qubits (16 GiB complex128 registers), where a
whole-circuit oracle run is too slow: the sizes of the benchmark workload,
with the qubits 26-29 that the oracle-parity tests (26 qubits and below,
``test_gpu_config2.py`` and ``test_gpu_parity.py``) never reach; the one
30-qubit comparison with the reference itself is the benchmark's first
layer (``test_gpu_config2.py``).  Each test here checks a property that holds
exactly for any correct state-vector engine, to the complex128 tolerance of
the parity tests:

- a product state after permutation and phase gates against its closed form,
  amplitude by amplitude at sampled indices (reference qops.c:176-261);
- the benchmark circuit followed by its inverse returns |0...0>;
- measuring four qubits in one call gives the outcomes and the collapsed
  register of measuring them one at a time (reference doki.c:1097-1157);
- the reduced density matrix of qubits 0-9 is Hermitian, positive, of trace
  one, and its diagonal gives the marginals (funmatrix.c:905-1037 and
  qops.c:72-95 evaluated on the same register);
- joins whose least register exceeds the L2 give the products of the inputs'
  amplitudes and the inputs' marginals (qops.c:97-122).
"""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import ATOL_C128

pytestmark = pytest.mark.gpu

N = 30


def _sample_indices(rng, n, count=2048):
    idx = set(int(i) for i in rng.integers(0, 1 << n, size=count))
    idx |= {0, (1 << n) - 1}
    idx |= {1 << q for q in range(n)}
    idx |= {((1 << n) - 1) ^ (1 << q) for q in range(n)}
    return sorted(idx)


def _permutation_phase_ops(n, rng):
    """CZ and CNOT brickworks, long-range CZs and anticontrolled X gates on the
    high qubits: every gate maps basis states to basis states."""
    ops = []
    for a in range(0, n - 1, 2):
        ops.append(W.Op(W.Z.copy(), [a + 1], {a}))
    for a in range(1, n - 1, 2):
        t, c = (a, a + 1) if rng.random() < 0.5 else (a + 1, a)
        ops.append(W.Op(W.X.copy(), [t], {c}))
    for a, b in ((0, n - 1), (3, n - 3), (n - 2, 5)):
        ops.append(W.Op(W.Z.copy(), [a], {b}))
    ops.append(W.Op(W.X.copy(), [n - 2], set(), {n - 1}))
    ops.append(W.Op(W.X.copy(), [n - 4], {1}, {n - 3}))
    return ops


def _closed_form(us, ops, i):
    """Amplitude i of (ops) (x)_q u_q |0>, walking the basis-state gates back."""
    phase = 1.0
    for op in reversed(ops):
        ok = all((i >> c) & 1 for c in op.controls) and \
            not any((i >> c) & 1 for c in op.anticontrols)
        if not ok:
            continue
        t = op.targets[0]
        if op.gate[0, 0] == 0:  # X: the amplitude comes from the flipped index
            i ^= 1 << t
        elif (i >> t) & 1:  # Z: -1 on the target's 1 half
            phase = -phase
    amp = complex(phase)
    for q, u in enumerate(us):
        amp *= u[(i >> q) & 1, 0]
    return amp


def test_30q_product_state_against_closed_form(dk_gpu):
    d = dk_gpu
    rng = W.rng_for(301)
    us = [W.u3(*rng.uniform(0, 2 * np.pi, 3)) for _ in range(N)]
    layer = [W.Op(u, [q]) for q, u in enumerate(us)]
    # marginals of the product state are untouched by the CZ brickwork
    czs = [W.Op(W.Z.copy(), [a + 1], {a}) for a in range(0, N - 1, 2)]
    r = W.run_ops(d, d.registry_new(N, False), layer + czs)
    want = [abs(u[1, 0]) ** 2 for u in us]
    assert np.allclose(d.registry_probs(r), want, atol=ATOL_C128, rtol=0)
    del r
    perm = _permutation_phase_ops(N, rng)
    r = W.run_ops(d, d.registry_new(N, False), layer + perm)
    for i in _sample_indices(rng, N):
        got = d.registry_get(r, i, False, False)
        assert abs(got - _closed_form(us, perm, i)) < ATOL_C128, i


def test_30q_benchmark_circuit_inverse_returns_zero_state(dk_gpu):
    d = dk_gpu
    c = W.scale_circuit(seed=2, n=N, depth=6, keep=10)
    inv = [W.Op(op.gate.conj().T, op.targets, op.controls, op.anticontrols)
           for op in reversed(c.ops)]
    r = W.run_ops(d, d.registry_new(N, False), c.ops + inv)
    assert abs(d.registry_get(r, 0, False, False) - 1) < ATOL_C128
    assert max(d.registry_probs(r)) < ATOL_C128


def test_30q_joint_measurement_equals_one_qubit_at_a_time(dk_gpu):
    d = dk_gpu
    c = W.scale_circuit(seed=2, n=N, depth=4, keep=10)
    r = W.run_ops(d, d.registry_new(N, False), c.ops)
    rolls = [float(x) for x in c.rolls]
    qubits = sorted((q for q in range(N) if (c.measure_mask >> q) & 1), reverse=True)
    joint, res = d.registry_measure(r, c.measure_mask, rolls, -1, False)
    seq = r
    for k, q in enumerate(qubits):
        n_now = N - k
        seq, one = d.registry_measure(seq, 1 << q, [rolls[k]], -1, False)
        assert one[n_now - 1 - q] == res[N - 1 - q], q
    rng = W.rng_for(302)
    for i in _sample_indices(rng, N - len(qubits), 1024):
        assert abs(d.registry_get(joint, i, False, False) -
                   d.registry_get(seq, i, False, False)) < ATOL_C128, i


def test_30q_reduced_density_properties(dk_gpu):
    d = dk_gpu
    c = W.scale_circuit(seed=2, n=N, depth=4, keep=10)
    r = W.run_ops(d, d.registry_new(N, False), c.ops)
    probs = d.registry_probs(r)
    rho = d.registry_density(r, False)
    for e in range(N - 1, 9, -1):
        rho = d.funmatrix_partialtrace(rho, e, False)
    m = d.funmatrix_numpy(rho)
    assert m.shape == (1024, 1024)
    assert abs(np.trace(m) - 1) < 1e-11
    assert np.abs(m - m.conj().T).max() < 1e-14
    assert np.linalg.eigvalsh(m).min() > -1e-12
    diag = np.diag(m).real
    a = np.arange(1024)
    for q in range(10):
        assert abs(diag[(a >> q) & 1 == 1].sum() - probs[q]) < ATOL_C128, q


@pytest.mark.parametrize("n1,n2,prec,tol", [(3, 24, 2, ATOL_C128), (1, 29, 2, ATOL_C128),
                                            (2, 26, 1, 1e-7)])
def test_join_with_a_large_least_register(dk_gpu, n1, n2, prec, tol):
    """registry_join where the least register exceeds the L2 (read once per
    amplitude, reference qops.c:97-122): every sampled amplitude is the
    product of the inputs' amplitudes and the result is normalised."""
    d = dk_gpu
    rng = W.rng_for(303 + n2)

    def reg(n):
        r = d.registry_new(n, False, prec)
        for q in range(n):
            r = d.registry_apply(r, d.gate_new(1, W._random_u3(rng).tolist(), False), [q],
                                 None, None, -1, False)
        return r

    most, least = reg(n1), reg(n2)
    j = d.registry_join(most, least, -1, False)
    for i in _sample_indices(rng, n1 + n2, 512):
        want = d.registry_get(most, i >> n2, False, False) * \
            d.registry_get(least, i & ((1 << n2) - 1), False, False)
        assert abs(d.registry_get(j, i, False, False) - want) < tol, i
    p = d.registry_probs(j)
    pm, pl = d.registry_probs(most), d.registry_probs(least)
    assert np.allclose(p, list(pl) + list(pm), atol=tol * 10, rtol=0)
