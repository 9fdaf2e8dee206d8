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


def test_reference_arm_line_carries_the_contract_keys():
    """Rank 0 of the reference arm (the reference module on the host cores,
    here on a 12-qubit case) prints one JSON line with the keys the
    benchmark contract names, e2e without host-device copies."""
    from oracle import oracle as O
    if not O.have_reference():
        pytest.skip("reference module not built (oracle/_ref)")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--qubits", "12", "--depth", "2", "--steps", "2", "--warmup", "1"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["qubits"] == 12 and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
