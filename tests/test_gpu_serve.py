"""Serving form on the GPU: requests served concurrently on several stream
slots must give the same results as each request run alone, and registers of
different slots must stay independent (including a join across slots)."""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import serve as S
from doki_b200 import workloads as W
from tests.conftest import ATOL_C128

pytestmark = pytest.mark.gpu


def compare(a, b, atol):
    assert a[0] == b[0]
    if a[0] == "probs":
        assert np.allclose(a[1], b[1], atol=atol, rtol=0)
    else:
        assert a[1] == b[1]


@pytest.mark.parametrize("precision", [2, 1])
def test_served_equals_alone(dk_gpu, precision):
    d = dk_gpu
    reqs = S.request_stream(seed=33, count=40, qmin=6, qmax=16, dmin=2, dmax=8, rate=400.0)
    srv = S.Server(d, workers=6, budget_bytes=2e9, precision=precision)
    mix = srv.run(reqs, keep_results=True)
    assert mix["requests"] == 40 and mix["p99_ms"] >= mix["p50_ms"] > 0
    atol = ATOL_C128 if precision == 2 else 1e-6
    for r in reqs:
        alone = S.execute(d, r, precision)
        compare(mix["results"][r.rid], alone, atol)


def test_served_matches_oracle(dk_gpu, orc):
    d = dk_gpu
    reqs = S.request_stream(seed=34, count=12, qmin=5, qmax=12, dmin=2, dmax=6, rate=1000.0)
    srv = S.Server(d, workers=4, budget_bytes=1e9, precision=2)
    out = srv.run(reqs, keep_results=True)
    for r in reqs:
        c = r.circuit()
        reg = W.run_ops(orc, orc.registry_new(r.n), c.ops)
        got = out["results"][r.rid]
        if r.terminal == "probs":
            assert np.allclose(got[1], orc.registry_probs(reg), atol=ATOL_C128)
        else:
            _, res = orc.registry_measure(reg, r.mask, r.rolls)
            assert got[1] == res


def test_budget_limits_concurrency(dk_gpu):
    """With a budget for one register at a time, requests run one by one."""
    d = dk_gpu
    reqs = S.request_stream(seed=35, count=6, qmin=14, qmax=14, dmin=2, dmax=3, rate=1e4)
    one = 2 * reqs[0].state_bytes(2)
    srv = S.Server(d, workers=4, budget_bytes=one, precision=2)
    out = srv.run(reqs)
    assert out["requests"] == 6


def test_join_across_slots(dk_gpu, orc):
    d = dk_gpu
    s1 = d.engine_new_slot()
    s2 = d.engine_new_slot()
    d.engine_set_slot(s1)
    a = W.run_ops(d, d.registry_new(6, False), W.small_circuit(seed=40, n=6, depth=3).ops)
    d.engine_set_slot(s2)
    b = W.run_ops(d, d.registry_new(5, False), W.small_circuit(seed=41, n=5, depth=3).ops)
    d.engine_set_slot(0)
    j = d.registry_join(a, b, 1, False)
    oa = W.run_ops(orc, orc.registry_new(6), W.small_circuit(seed=40, n=6, depth=3).ops)
    ob = W.run_ops(orc, orc.registry_new(5), W.small_circuit(seed=41, n=5, depth=3).ops)
    assert np.allclose(d.registry_get_all(j), orc.registry_get_all(orc.registry_join(oa, ob)),
                       atol=ATOL_C128)


@pytest.mark.parametrize("after", ["del", "overwrite"])
def test_join_across_slots_then_reuse_least(dk_gpu, after):
    """A join reads the least register's storage on the most register's
    stream.  Work that least's slot queues right after the join -- freeing
    that storage (and a new register reusing the pool block), or a register
    derived from least flushed in place over it -- must wait for that read."""
    d = dk_gpu
    s1, s2 = d.engine_new_slot(), d.engine_new_slot()
    d.engine_set_slot(s1)
    a = W.run_ops(d, d.registry_new(2, False), W.small_circuit(seed=42, n=2, depth=2).ops)
    d.engine_set_slot(s2)
    b = W.run_ops(d, d.registry_new(24, False), W.small_circuit(seed=43, n=24, depth=1).ops)
    d.engine_set_slot(0)
    va, vb = d.registry_get_all(a, False), d.registry_get_all(b, False)
    j = d.registry_join(a, b, 1, False)
    if after == "del":
        d.registry_del(b, False)
        d.engine_set_slot(s2)
        reuse = d.registry_new(24, False)
        d.engine_set_slot(0)
        assert d.registry_prob(reuse, 0, 1, False) == 0.0
    else:
        g = d.gate_new(1, W.u3(0.3, 0.2, 0.1).tolist(), False)
        b2 = d.registry_apply(b, g, [0], None, None, 1, False)
        del b  # b2 alone holds the storage: its sweep runs in place
        d.registry_prob(b2, 0, 1, False)
    assert np.allclose(d.registry_get_all(j, False), np.kron(va, vb), atol=ATOL_C128, rtol=0)


def _flat(ops):
    """ops as the flat arrays registry_apply_many takes."""
    n = len(ops)
    k = np.array([op.k for op in ops], dtype=np.uint32)
    tg = np.zeros((n, 3), dtype=np.uint32)
    cm = np.zeros(n, dtype=np.uint64)
    am = np.zeros(n, dtype=np.uint64)
    mi = np.zeros(n, dtype=np.uint64)
    mats, off = [], 0
    for i, op in enumerate(ops):
        tg[i, :op.k] = op.targets
        cm[i] = sum(1 << c for c in op.controls)
        am[i] = sum(1 << c for c in op.anticontrols)
        mi[i] = off
        mats.append(np.ascontiguousarray(op.gate, dtype=np.complex128).reshape(-1))
        off += op.gate.size
    return k, tg, cm, am, mi, np.concatenate(mats)


@pytest.mark.parametrize("precision", [2, 1])
def test_apply_many_equals_one_call_per_gate(dk_gpu, precision):
    """registry_apply_many queues the same gates as one registry_apply call
    per gate: the flushed registers are identical."""
    d = dk_gpu
    c = W.small_circuit(seed=44, n=15, depth=6)
    ops = c.ops + [W.Op(W.u3(0.1, 0.2, 0.3), [3], {7}, {11})]
    a = W.run_ops(d, d.registry_new(15, False, precision), ops)
    b = d.registry_apply_many(d.registry_new(15, False, precision), *_flat(ops))
    assert np.array_equal(d.registry_get_all(a, False), d.registry_get_all(b, False))
    # rejected as a whole: a target out of range queues nothing
    bad = list(_flat(ops[:3]))
    bad[1] = bad[1].copy()
    bad[1][2, 0] = 15
    with pytest.raises(d.error):
        d.registry_apply_many(b, *bad)
