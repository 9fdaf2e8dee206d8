"""Parity of the benchmark workload's circuit family in complex128.

The 30-qubit benchmark circuit (``workloads.scale_circuit``: U3 on every qubit,
CZ / CNOT brickwork, 5 % of the gates with 1-3 extra controls or
anticontrols) runs through the default planner: 12-bit tensor-core tiles,
2 pinned low qubits, chained pass pairs, and tile-condition variants
(``DK_GC_DENSE3V``) for the conditioned gates whose extra qubits lie outside
the tile.  These tests pin that exact path against the references:

- at 24 and 26 qubits, depth 8, against the CPU oracle: every amplitude,
  every marginal, the reduced density matrix of qubits 0-9, the outcomes of
  the benchmark's 4-qubit measurement and the collapsed register (reference
  qops.c:176-261, qops.c:72-95, funmatrix.c:905-1037, doki.c:1023-1192);
- at 30 qubits, the benchmark's own first layer (45 gates, two of them
  conditioned, one on qubits 25 and 27 outside every tile) against the
  reference module itself, compiled from its sources: sampled amplitudes,
  all 30 probabilities (the engine's checked against an independent sum of
  its own amplitudes at 1e-13, the reference's within the 2e-11 relative
  rounding of its own sums of 2^29-2^30 terms), and the benchmark mask's
  outcomes and collapsed register.
"""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import ATOL_C128, TIE_C128, compare_outcomes

pytestmark = pytest.mark.gpu


def _conditioned(op):
    """A gate the generator gave extra controls or anticontrols."""
    return bool(op.anticontrols) or len(op.controls) > 1 or \
        (bool(op.controls) and abs(op.gate[0, 0]) not in (0.0, 1.0))


def _res(res):
    return [-1 if v is None else int(v) for v in res]


def _rho_low(vec, n, keep):
    """Reduced density matrix of qubits 0..keep-1 as a plain product:
    rho = M^T conj(M) for the (2^(n-keep) x 2^keep) row-major view M of the
    state (the traced qubits are the high ones)."""
    m = vec.reshape(1 << (n - keep), 1 << keep)
    return m.T @ m.conj()


@pytest.mark.parametrize("n", [24, 26])
def test_benchmark_circuit_family_vs_oracle(dk_gpu, orc, n):
    d = dk_gpu
    c = W.scale_circuit(seed=2, n=n, depth=8, keep=10)
    assert sum(_conditioned(op) for op in c.ops) >= 10
    a = W.run_ops(d, d.registry_new(n, False), c.ops)
    b = W.run_ops(orc, orc.registry_new(n), c.ops)
    va, vb = d.registry_get_all(a, False), orc.registry_get_all(b)
    assert np.abs(va - vb).max() < ATOL_C128
    assert np.allclose(d.registry_probs(a), orc.registry_probs(b), atol=ATOL_C128, rtol=0)

    rho = d.registry_density(a, False)
    for e in range(n - 1, 9, -1):
        rho = d.funmatrix_partialtrace(rho, e, False)
    assert np.abs(d.funmatrix_numpy(rho) - _rho_low(vb, n, 10)).max() < ATOL_C128

    rolls = c.rolls.tolist()
    ra, resa = d.registry_measure(a, c.measure_mask, rolls, 1, False)
    rb, resb = orc.registry_measure(b, c.measure_mask, rolls)
    tie = compare_outcomes(_res(resa), _res(resb), orc.last_margins, TIE_C128)
    if tie:
        pytest.xfail(tie)
    assert np.abs(d.registry_get_all(ra, False) - orc.registry_get_all(rb)).max() < ATOL_C128


def test_30q_first_benchmark_layer_vs_reference_module(dk_gpu, ref):
    """About a minute of reference CPU time (16 GiB registers, one OpenMP
    sweep per gate on the host)."""
    d = dk_gpu
    n = 30
    c = W.scale_circuit(seed=2, n=n, depth=40, keep=10)
    ops = c.ops[c.layer_starts[0]:c.layer_starts[1]]
    assert sum(_conditioned(op) for op in ops) == 2
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(ref, ref.registry_new(n, False), ops)

    rng = W.rng_for(3030)
    idx = sorted(set(int(i) for i in rng.integers(0, 1 << n, size=2000)) |
                 {0, (1 << n) - 1} | {1 << q for q in range(n)})
    for i in idx:
        assert abs(d.registry_get(a, i, False, False) -
                   ref.registry_get(b, i, False, False)) < ATOL_C128, i
    # The engine's marginals against an independent sum of its own
    # amplitudes (numpy's pairwise summation over contiguous halves, error
    # near 1e-16 relative), for low, middle and high qubits.
    got = np.array(d.registry_probs(a))
    amps = d.registry_get_all(a, False)
    p = (amps.real ** 2 + amps.imag ** 2).reshape(-1)
    del amps
    for q in (0, 13, 25, n - 1):
        half = np.ascontiguousarray(p.reshape(1 << (n - 1 - q), 2, 1 << q)[:, 1, :])
        assert abs(float(half.sum()) - got[q]) < 1e-13, q
    del p, half
    # The reference's probabilities at 30 qubits carry the rounding of its
    # own OpenMP sums (each one 2^29 squared amplitudes in partial sums of
    # 2^25 per thread, and its norm constant one of 2^30): a few 1e-12
    # relative here, above the 1e-12 of the smaller registers.  They agree
    # with the engine's within 2e-11 relative.
    want = np.array([ref.registry_prob(b, q, -1, False) for q in range(n)])
    assert np.allclose(got, want, rtol=2e-11, atol=0)
    rolls = c.rolls.tolist()
    ra, resa = d.registry_measure(a, c.measure_mask, rolls, -1, False)
    del a
    rb, resb = ref.registry_measure(b, c.measure_mask, rolls, -1, False)
    del b
    assert _res(resa) == _res(resb)
    m = n - bin(c.measure_mask).count("1")
    for i in sorted(set(int(i) for i in rng.integers(0, 1 << m, size=1000)) | {0}):
        assert abs(d.registry_get(ra, i, False, False) -
                   ref.registry_get(rb, i, False, False)) < ATOL_C128, i
