"""Distributed register (doki_b200.dist) on 2 and 4 gloo ranks on CPU.

Every rank holds a shard of the register's low qubits (EngineShard over a
CPU stand-in of the engine built on the oracle); gates on rank qubits swap
them in by exchanging half a shard with the partner rank.  The results --
all amplitudes, all marginals, measurement outcomes with the collapsed
register, and reduced density matrices -- must equal the single-register
oracle's on the same circuit (reference qops.c:176-261, qops.c:72-95,
doki.c:1023-1192, funmatrix.c:905-1037)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.conftest import ATOL_C128, ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def circuit(n, seed, count=60):
    """Random 1-3-qubit gates with controls and anticontrols on any qubit,
    plus a non-unitary gate (renormalisation across ranks)."""
    import sys
    sys.path.insert(0, ROOT)
    from doki_b200 import workloads as W
    from tests.golden.gen_golden import random_unitary
    rng = W.rng_for(seed)
    ops = []
    for i in range(count):
        k = int(rng.integers(1, 4))
        qs = [int(q) for q in rng.choice(n, size=min(n, k + 2), replace=False)]
        tg, rest = qs[:k], qs[k:]
        ctl = {rest[0]} if rest and rng.random() < 0.4 else set()
        act = {rest[-1]} if len(rest) > 1 and rng.random() < 0.3 else set()
        ops.append(W.Op(random_unitary(rng, k), tg, ctl, act))
    ops.append(W.Op(np.diag([1.0, 0.35]).astype(np.complex128), [n - 1]))
    ops.append(W.Op(np.array([[0.8, 0.1j], [0.2, 1.1]]), [0], {n - 2}))
    return ops


def rank_qubit_ops(n, nl):
    """Qubit n-1 is swapped in for a gate, then swapped back onto a rank
    position by a gate on the qubit that took its place."""
    from doki_b200 import workloads as W
    return [W.Op(W.H.copy(), [n - 1]), W.Op(W.X.copy(), [0], {n - 1}),
            W.Op(W.u3(0.7, 0.1, 0.2), [nl - 1]), W.Op(W.u3(1.1, 0.4, 0.3), [1])]


def _rank_measure(rank, world, port, n, out):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from doki_b200.dist import DistRegister, EngineShard
        from tests.oracle_shard import OracleShardDoki
        d = OracleShardDoki()
        reg = DistRegister(n, lambda nl: EngineShard(d, nl), dist)
        for op in rank_qubit_ops(n, reg.nl):
            reg.apply(op.gate, op.targets, op.controls, op.anticontrols)
        reg.probs()
        on_rank = reg.position(n - 1) >= reg.nl
        res = reg.measure((1 << (n - 1)) | 1, [0.44, 0.58])
        out.put((rank, {"on_rank": on_rank, "measure": res, "after": reg.gather()}))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, {"error": repr(e)}))
        raise
    finally:
        dist.destroy_process_group()


def _rank(rank, world, port, n, seed, out):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from doki_b200.dist import DistRegister, EngineShard
        from tests.oracle_shard import OracleShardDoki
        d = OracleShardDoki()
        reg = DistRegister(n, lambda nl: EngineShard(d, nl), dist)
        ops = circuit(n, seed)
        for op in ops:
            reg.apply(op.gate, op.targets, op.controls, op.anticontrols)
        res = {"probs": reg.probs(), "amps": reg.gather(), "exchanges": reg.exchanges}
        res["rho_low"] = reg.reduced_density([0, 1, 2])
        res["rho_mixed"] = reg.reduced_density([1, n - 1])
        mask = (1 << (n - 1)) | (1 << 2) | 1
        res["measure"] = reg.measure(mask, [0.31, 0.62, 0.47])
        res["after"] = reg.gather()
        res["after_probs"] = reg.probs()
        out.put((rank, res))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, {"error": repr(e)}))
        raise
    finally:
        dist.destroy_process_group()


def run_world(world, n, seed, target=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    fn = target or _rank
    args = (lambda r: (r, world, port, n, seed, q)) if target is None else \
        (lambda r: (r, world, port, n, q))
    procs = [ctx.Process(target=fn, args=args(r)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for r in range(world):
        assert "error" not in res[r], res[r]
    assert all(p.exitcode == 0 for p in procs)
    return res


@pytest.mark.parametrize("world,n,seed", [(2, 7, 1), (4, 8, 2)])
def test_distributed_register_matches_the_oracle(orc, oracle_mod, world, n, seed):
    from doki_b200 import workloads as W
    res = run_world(world, n, seed)
    ops = circuit(n, seed)
    want = W.run_ops(orc, orc.registry_new(n), ops)
    r0 = res[0]
    assert r0["exchanges"] > 0  # gates on rank qubits swapped them in
    assert np.abs(r0["amps"] - orc.registry_get_all(want)).max() < ATOL_C128
    for r in range(world):  # every rank holds the all-reduced results
        assert np.allclose(res[r]["probs"], orc.registry_probs(want), atol=ATOL_C128, rtol=0)
        assert np.allclose(res[r]["rho_low"], oracle_mod.reduced_density(want, 0b111),
                           atol=ATOL_C128, rtol=0)
        mixed = oracle_mod.reduced_density(want, (1 << 1) | (1 << (n - 1)))
        assert np.allclose(res[r]["rho_mixed"], mixed, atol=ATOL_C128, rtol=0)
    mask = (1 << (n - 1)) | (1 << 2) | 1
    after, outcome = orc.registry_measure(want, mask, [0.31, 0.62, 0.47])
    for r in range(world):
        assert res[r]["measure"] == outcome
    assert np.abs(r0["after"] - orc.registry_get_all(after)).max() < ATOL_C128
    assert np.allclose(r0["after_probs"], orc.registry_probs(after), atol=ATOL_C128, rtol=0)


def test_measuring_a_qubit_on_a_rank_position(orc):
    """A measured qubit that sits on a rank position: the ranks on the other
    side of the outcome drop out (weight 0) and the rank bit is frozen; the
    outcomes and the collapsed register equal the oracle's."""
    from doki_b200 import workloads as W
    n, world = 6, 4
    res = run_world(world, n, 0, target=_rank_measure)
    assert res[0]["on_rank"]
    want = W.run_ops(orc, orc.registry_new(n), rank_qubit_ops(n, n - 2))
    after, outcome = orc.registry_measure(want, (1 << (n - 1)) | 1, [0.44, 0.58])
    for r in range(world):
        assert res[r]["measure"] == outcome
    assert np.abs(res[0]["after"] - orc.registry_get_all(after)).max() < ATOL_C128
