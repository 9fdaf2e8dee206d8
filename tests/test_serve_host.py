"""Host logic of the serving form on CPU, with a fake engine: admission in
arrival order under the HBM budget and the slot count, and errors that
surface instead of hanging the dispatcher."""
from __future__ import annotations

import threading
import time

import pytest

from doki_b200 import serve as S


class FakeDoki:
    """Stands in for the engine: records how many registers are alive."""

    def __init__(self, fail_on=None, delay=0.002):
        self.lock = threading.Lock()
        self.live = 0
        self.max_live = 0
        self.nslots = 1
        self.fail_on = fail_on
        self.delay = delay
        self.mem = 0
        self.max_mem = 0

    def engine_new_slot(self):
        self.nslots += 1
        return self.nslots - 1

    def engine_set_slot(self, slot):
        assert 0 <= slot < self.nslots

    def gate_new(self, k, m, verbose):
        return (k, m)

    def registry_new(self, n, verbose, precision=2):
        if self.fail_on is not None and n == self.fail_on:
            raise RuntimeError("planted failure")
        with self.lock:
            self.live += 1
            self.max_live = max(self.max_live, self.live)
            self.mem += (8 if precision == 1 else 16) << n
            self.max_mem = max(self.max_mem, self.mem)
        return {"n": n, "precision": precision}

    def registry_apply(self, reg, g, targets, c, a, threads, verbose):
        return reg

    def registry_apply_many(self, reg, *arrays):
        assert len(arrays) == 6
        return reg

    def _finish(self, reg):
        time.sleep(self.delay)
        with self.lock:
            self.live -= 1
            self.mem -= (8 if reg["precision"] == 1 else 16) << reg["n"]

    def registry_probs(self, reg):
        self._finish(reg)
        return [0.5] * reg["n"]

    def registry_measure(self, reg, mask, rolls, threads, verbose):
        self._finish(reg)
        return None, [None] * reg["n"]


def small_stream(count, n=10):
    reqs = S.request_stream(seed=3, count=count, qmin=n, qmax=n, dmin=1, dmax=2, rate=1e6)
    return reqs


def test_slot_count_bounds_concurrency():
    d = FakeDoki()
    out = S.Server(d, workers=3, budget_bytes=1e12, precision=1).run(small_stream(24))
    assert out["requests"] == 24
    assert d.max_live <= 3


def test_budget_bounds_resident_registers():
    d = FakeDoki()
    reqs = small_stream(20, n=12)
    two = 2 * 2 * reqs[0].state_bytes(1)  # room for two reservations
    S.Server(d, workers=6, budget_bytes=two, precision=1).run(reqs)
    assert d.max_live <= 2


def test_worker_error_surfaces():
    d = FakeDoki(fail_on=11)
    reqs = S.request_stream(seed=4, count=10, qmin=10, qmax=12, dmin=1, dmax=2, rate=1e6)
    assert any(r.n == 11 for r in reqs)
    with pytest.raises(RuntimeError, match="planted failure"):
        S.Server(d, workers=2, precision=1, deadline_s=30).run(reqs)


def test_request_stream_is_seeded():
    a = S.request_stream(seed=9, count=50)
    b = S.request_stream(seed=9, count=50)
    assert [(r.n, r.depth, r.terminal, r.mask) for r in a] == \
        [(r.n, r.depth, r.terminal, r.mask) for r in b]
    assert all(8 <= r.n <= 28 and 10 <= r.depth <= 100 for r in a)
    assert all(r.arrival >= 0 for r in a)


def test_plain_path_runs_one_request_at_a_time_gate_by_gate():
    d = FakeDoki()
    calls = []
    d.registry_apply = lambda reg, g, t, c, a, th, v: calls.append(t) or reg
    reqs = S.request_stream(seed=3, count=5, qmin=4, qmax=6, dmin=2, dmax=3)
    out = S.run_plain(d, reqs, precision=2)
    assert out["requests"] == 5 and len(out["seconds"]) == 5
    assert d.max_live == 1
    assert len(calls) == sum(r.flat().count for r in reqs)


class SizedDelay(FakeDoki):
    """Requests of more than 20 qubits take long on the fake device."""

    def _finish(self, reg):
        time.sleep(0.3 if reg["n"] > 20 else 0.002)
        with self.lock:
            self.live -= 1
            self.mem -= (8 if reg["precision"] == 1 else 16) << reg["n"]


def mixed_stream():
    # two large requests first, then small ones arriving right behind them
    reqs = []
    for i, n in enumerate([24, 24] + [10] * 12):
        reqs.append(S.Request(rid=i, arrival=0.001 * i, n=n, depth=1, seed=i,
                              terminal="probs"))
    return reqs


def test_express_slots_let_small_requests_pass_large_ones():
    """With 2 slots both held by large requests, small requests queue behind
    them (plain arrival order); with one express slot they run meanwhile,
    while the large ones keep their order on the general slot."""
    plain = S.Server(SizedDelay(), workers=2, budget_bytes=1e12, precision=1)
    out = plain.run(mixed_stream(), keep_results=False)
    fast = S.Server(SizedDelay(), workers=2, budget_bytes=1e12, precision=1, express=1)
    out2 = fast.run(mixed_stream(), keep_results=False)
    assert out["requests"] == out2["requests"] == 14
    # the small requests' median latency: behind the large ones vs not
    assert out["p50_ms"] > 250
    assert out2["p50_ms"] < 100


def test_express_slots_leave_a_general_slot():
    with pytest.raises(ValueError):
        S.Server(FakeDoki(), workers=2, express=2)
