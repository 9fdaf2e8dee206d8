"""Serving form: continuous batching of circuit requests under an HBM budget.

Requests arrive as a Poisson stream.  Each carries a circuit of n qubits
(log-uniform in [qmin, qmax]) and depth d (uniform in [dmin, dmax]) drawn
from the plain method's CPU-runnable generator (U3 on every qubit, CNOT on a
random pairing, one Toffoli with an anticontrol per layer), and a terminal
operation: all single-qubit probabilities, or the measurement of k in [1, 8]
random qubits with seeded draws.  A request arrives with its circuit as
data (the flat gate arrays of ``registry_apply_many``, built by the client
before the stream starts: :func:`prepare`), as a request to a server does.

The server keeps `workers` requests in flight, each on its own stream slot of
the engine (so their kernels overlap on the device), admits the next request
in arrival order as soon as a slot is free and its register fits in the HBM
budget, queues the whole circuit with one ``registry_apply_many`` call (no
Python work per gate, the interpreter lock released), keeps every register
resident on the device from its first gate to its result, and records
per-request latency from arrival to result on the host.

The plain path (:func:`run_plain`) is the reference's way of using the
module: one request at a time, one ``registry_apply`` call per gate.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional, Sequence

import numpy as np

from . import workloads as W


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the stream starts
    n: int
    depth: int
    seed: int
    terminal: str  # "probs" or "measure"
    mask: int = 0
    rolls: List[float] = field(default_factory=list)

    def circuit(self) -> W.Circuit:
        return W.small_circuit(seed=self.seed, n=self.n, depth=self.depth)

    def flat(self) -> W.FlatCircuit:
        """The circuit as flat gate arrays (built once, kept)."""
        f = self.__dict__.get("_flat")
        if f is None:
            f = W.small_circuit_flat(seed=self.seed, n=self.n, depth=self.depth)
            self.__dict__["_flat"] = f
        return f

    def state_bytes(self, precision: int) -> int:
        return (16 if precision == 2 else 8) << self.n


def request_stream(seed: int = 5, count: int = 20000, qmin: int = 8, qmax: int = 28,
                   dmin: int = 10, dmax: int = 100, rate: float = 1.0) -> List[Request]:
    """`count` requests; inter-arrival times ~ Exp(rate) (requests / s)."""
    rng = W.rng_for(seed)
    ns = np.floor(np.exp(rng.uniform(np.log(qmin), np.log(qmax + 1), size=count))).astype(int)
    ns = np.clip(ns, qmin, qmax)
    depths = rng.integers(dmin, dmax + 1, size=count)
    gaps = rng.exponential(1.0 / rate, size=count) if rate > 0 else np.zeros(count)
    arrivals = np.cumsum(gaps) - (gaps[0] if count else 0.0)
    out = []
    for i in range(count):
        n = int(ns[i])
        if rng.random() < 0.5:
            out.append(Request(i, float(arrivals[i]), n, int(depths[i]), 10_000 + i, "probs"))
        else:
            k = int(rng.integers(1, 9))
            qs = rng.choice(n, size=min(k, n), replace=False)
            mask = 0
            for q in qs:
                mask |= 1 << int(q)
            out.append(Request(i, float(arrivals[i]), n, int(depths[i]), 10_000 + i,
                               "measure", mask, rng.random(len(qs)).tolist()))
    return out


def with_rate(reqs: Sequence[Request], rate: float, seed: int = 6) -> List[Request]:
    """The same requests re-timed as a Poisson stream of `rate` requests / s."""
    rng = W.rng_for(seed)
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    arr = np.cumsum(gaps) - gaps[0]
    out = []
    for r, a in zip(reqs, arr):
        q = Request(r.rid, float(a), r.n, r.depth, r.seed, r.terminal, r.mask, r.rolls)
        if "_flat" in r.__dict__:  # keep the prepared circuit
            q.__dict__["_flat"] = r.__dict__["_flat"]
        out.append(q)
    return out


def prepare(reqs: Sequence[Request]) -> None:
    """Build every request's circuit arrays ahead of the stream (the
    client's work, outside any timed run)."""
    for r in reqs:
        r.flat()


def _terminal(d, reg, req: Request):
    if req.terminal == "probs":
        return ("probs", d.registry_probs(reg))
    _, res = d.registry_measure(reg, req.mask, req.rolls, -1, False)
    return ("measure", res)


def execute(d, req: Request, precision: int):
    """Run one request on the calling thread's slot: the whole circuit in one
    registry_apply_many call, then its terminal operation."""
    reg = d.registry_apply_many(d.registry_new(req.n, False, precision), *req.flat().arrays())
    return _terminal(d, reg, req)


def execute_per_gate(d, req: Request, precision: int):
    """The plain path for one request: one gate_new + registry_apply call
    per gate from the request's arrays, as a user of the reference module
    writes it (doki.c:722-941)."""
    f = req.flat()
    reg = d.registry_new(req.n, False, precision)
    for i in range(f.count):
        k = int(f.op_k[i])
        m0 = int(f.op_matrix[i])
        g = d.gate_new(k, f.matrices[m0:m0 + (1 << (2 * k))].reshape(1 << k, 1 << k).tolist(),
                       False)
        cm, am = int(f.op_controls[i]), int(f.op_anticontrols[i])
        ctl = {q for q in range(req.n) if (cm >> q) & 1} if (cm or am) else None
        act = {q for q in range(req.n) if (am >> q) & 1} or None
        reg = d.registry_apply(reg, g, [int(t) for t in f.op_targets[i, :k]], ctl, act, -1,
                               False)
    return _terminal(d, reg, req)


def run_plain(d, reqs: Sequence[Request], precision: int = 2,
              deadline_s: float = 3600.0) -> Dict:
    """The plain GPU path: the requests one after another on one slot, each
    through one registry_apply call per gate; returns its throughput and
    the seconds each request took."""
    t0 = time.perf_counter()
    per = []
    for r in reqs:
        a = time.perf_counter()
        execute_per_gate(d, r, precision)
        per.append(time.perf_counter() - a)
        if a - t0 > deadline_s:
            raise TimeoutError(f"plain run exceeded {deadline_s} s")
    total = time.perf_counter() - t0
    return {"requests": len(reqs), "throughput_rps": len(reqs) / total, "seconds": per}


class Server:
    """Continuous batching over `workers` engine slots under an HBM budget.

    Requests are admitted in arrival order as slots and memory free up.
    With `express` > 0, that many of the slots take only requests of at most
    `express_max_qubits` qubits, and such a small request may be admitted
    ahead of an earlier larger one that is waiting for a slot or memory
    (larger requests keep their order among themselves), so small requests
    do not queue behind the large ones that occupy the device."""

    def __init__(self, d, workers: int = 8, budget_bytes: float = 150e9, precision: int = 1,
                 deadline_s: float = 600.0, express: int = 0, express_max_qubits: int = 20):
        if not 0 <= express < workers:
            raise ValueError("express slots must leave at least one general slot")
        self.d = d
        self.workers = workers
        self.budget = budget_bytes
        self.precision = precision
        self.deadline_s = deadline_s
        self.express = express
        self.express_max_qubits = express_max_qubits
        self.slots = [0] + [d.engine_new_slot() for _ in range(workers - 1)]

    def run(self, reqs: Sequence[Request], keep_results: bool = False) -> Dict:
        reqs = sorted(reqs, key=lambda r: r.arrival)
        lock = threading.Condition()
        state = {"mem": 0, "free": list(range(self.workers)), "next": 0, "done": 0}
        queues: List[List[Request]] = [[] for _ in range(self.workers)]
        latency = np.zeros(len(reqs))
        finish = np.zeros(len(reqs))
        results: Dict[int, object] = {}
        errors: List[BaseException] = []
        t0 = time.perf_counter()
        index = {r.rid: i for i, r in enumerate(reqs)}

        def worker(w: int):
            try:
                self.d.engine_set_slot(self.slots[w])
            except BaseException as e:  # noqa: BLE001
                errors.append(e)
            while True:
                with lock:
                    while not queues[w]:
                        lock.wait(timeout=1.0)
                    req = queues[w].pop(0)
                if req is None:
                    return
                res = None
                if not errors:
                    try:
                        res = execute(self.d, req, self.precision)
                    except BaseException as e:  # noqa: BLE001
                        errors.append(e)
                now = time.perf_counter() - t0
                i = index[req.rid]
                finish[i] = now
                latency[i] = now - req.arrival
                if keep_results:
                    results[req.rid] = res
                with lock:
                    state["mem"] -= 2 * req.state_bytes(self.precision)
                    state["free"].append(w)
                    state["done"] += 1
                    lock.notify_all()

        threads = [threading.Thread(target=worker, args=(w,), daemon=True)
                   for w in range(self.workers)]
        for t in threads:
            t.start()
        def check():
            if errors:
                raise RuntimeError(f"serving worker failed: {errors[0]!r}") from errors[0]
            if time.perf_counter() - t0 > self.deadline_s:
                raise TimeoutError(f"serving run exceeded {self.deadline_s} s")

        express = set(range(self.workers - self.express, self.workers))
        # arrived, not yet admitted: the general class and (with express
        # slots) the small class, each in arrival order
        waiting_general: Deque[Request] = collections.deque()
        waiting_small: Deque[Request] = collections.deque()

        def place(req: Request, slots: List[int]) -> bool:
            need = 2 * req.state_bytes(self.precision)
            if not slots or (state["mem"] + need > self.budget and state["mem"] > 0):
                return False
            w = slots[0]
            state["free"].remove(w)
            state["mem"] += need
            queues[w].append(req)
            lock.notify_all()
            return True

        def admit() -> None:
            while waiting_general and place(
                    waiting_general[0], [w for w in state["free"] if w not in express]):
                waiting_general.popleft()
            # small requests: express slots, and general ones nobody waits for
            while waiting_small:
                slots = [w for w in state["free"] if w in express]
                if not waiting_general:
                    slots += [w for w in state["free"] if w not in express]
                if not place(waiting_small[0], slots):
                    break
                waiting_small.popleft()

        try:
            i = 0
            while i < len(reqs) or waiting_general or waiting_small:
                while i < len(reqs) and reqs[i].arrival <= time.perf_counter() - t0:
                    req = reqs[i]
                    small = bool(express) and req.n <= self.express_max_qubits
                    (waiting_small if small else waiting_general).append(req)
                    i += 1
                with lock:
                    admit()
                    if waiting_general or waiting_small:
                        # wait for a completion, or for the next arrival
                        to_next = (reqs[i].arrival - (time.perf_counter() - t0)
                                   if i < len(reqs) else 1.0)
                        lock.wait(timeout=min(1.0, max(1e-4, to_next)))
                        check()
                if not (waiting_general or waiting_small) and i < len(reqs):
                    wait = reqs[i].arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(wait)
            with lock:
                while state["done"] < len(reqs):
                    lock.wait(timeout=1.0)
                    check()
        finally:
            with lock:
                for w in range(self.workers):
                    queues[w].append(None)
                lock.notify_all()
            for t in threads:
                t.join(timeout=60.0)
        check()
        makespan = float(finish.max()) if len(reqs) else 0.0
        return {
            "requests": len(reqs),
            "throughput_rps": len(reqs) / makespan if makespan > 0 else 0.0,
            "p50_ms": float(np.percentile(latency, 50) * 1e3),
            "p99_ms": float(np.percentile(latency, 99) * 1e3),
            "mean_ms": float(latency.mean() * 1e3),
            "makespan_s": makespan,
            "results": results if keep_results else None,
        }
