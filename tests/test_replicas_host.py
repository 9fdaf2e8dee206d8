"""The N-GPU bench path runs independent replicas: per-rank timings are
reduced by their maximum over ranks and the job rate counts every rank's
work.  Checked here with 2 gloo ranks on CPU; the reference arm prints from
rank 0 only."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r was slower on the first timer, faster on the second
        got = bench.max_over_ranks([100.0 + rank, 50.0 - rank, 7.0], world, "cpu")
        out.put((rank, got, bench.job_rate(world, 40, got[0] / 1e3)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_count_all_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, got, rate in res:
        assert got == [101.0, 50.0, 7.0]
        assert rate == pytest.approx(2 * 40 / 0.101)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks([3, 4], 1, "cpu") == [3.0, 4.0]
    assert bench.job_rate(1, 40, 2.0) == 20.0


def test_reference_arm_prints_from_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
