"""Distributed register on the engine: two ranks, each an engine shard on
the GPU, exchanging halves through host buffers over gloo (every gate and
read of a shard runs the engine's kernels; one GPU serves both processes,
whose kernels never wait on each other).  The 16-qubit register split over
the two ranks must equal the oracle's single register."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.conftest import ATOL_C128, ROOT
from tests.test_dist_host import _free_port, circuit

pytestmark = pytest.mark.gpu


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
        import doki_b200
        from doki_b200.dist import DistRegister, EngineShard
        d = doki_b200.load()
        reg = DistRegister(n, lambda nl: EngineShard(d, nl), dist)
        for op in circuit(n, seed, count=80):
            reg.apply(op.gate, op.targets, op.controls, op.anticontrols)
        res = {"probs": reg.probs(), "amps": reg.gather(), "exchanges": reg.exchanges,
               "rho": reg.reduced_density([0, 3, n - 1]),
               "measure": reg.measure((1 << (n - 1)) | (1 << 5), [0.37, 0.81])}
        res["after"] = reg.gather()
        out.put((rank, res))
    except BaseException as e:  # noqa: BLE001
        out.put((rank, {"error": repr(e)}))
        raise
    finally:
        dist.destroy_process_group()


def test_engine_shards_match_the_oracle(dk_gpu, orc, oracle_mod):
    from doki_b200 import workloads as W
    n, world, seed = 16, 2, 7
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, seed, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
    for r in range(world):
        assert "error" not in res[r], res[r]
    want = W.run_ops(orc, orc.registry_new(n), circuit(n, seed, count=80))
    assert res[0]["exchanges"] > 0
    assert np.abs(res[0]["amps"] - orc.registry_get_all(want)).max() < ATOL_C128
    keep = 1 | (1 << 3) | (1 << (n - 1))
    for r in range(world):
        assert np.allclose(res[r]["probs"], orc.registry_probs(want), atol=ATOL_C128, rtol=0)
        assert np.allclose(res[r]["rho"], oracle_mod.reduced_density(want, keep),
                           atol=ATOL_C128, rtol=0)
    after, outcome = orc.registry_measure(want, (1 << (n - 1)) | (1 << 5), [0.37, 0.81])
    assert res[0]["measure"] == outcome and res[1]["measure"] == outcome
    assert np.abs(res[0]["after"] - orc.registry_get_all(after)).max() < ATOL_C128
