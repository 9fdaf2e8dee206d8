"""Batching form on the GPU: every register of a mixed batch (4-16 qubits:
sub-warp thread groups, whole-CTA groups and registers streamed through tiles)
must match the oracle -- final amplitudes (renormalised) and the reduced
density matrix over the lower half of the qubits."""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import ATOL_C128, ATOL_C64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    # every size from 4 to 16 qubits, shallow circuits so the oracle is quick
    fb = W.batch_arrays(seed=21, count=60, qmin=4, qmax=16, dmin=2, dmax=5)
    return fb


def oracle_case(orc, oracle_mod, fb, c):
    n = int(fb.num_qubits[c])
    reg = W.run_ops(orc, orc.registry_new(n), fb.ops(c))
    keep = (1 << int(fb.keep[c])) - 1
    return orc.registry_get_all(reg), oracle_mod.reduced_density(reg, keep)


@pytest.mark.parametrize("precision,tile_bits", [(2, 12), (2, 10), (1, 12)])
def test_batch_matches_oracle(dk_gpu, orc, oracle_mod, small_batch, precision, tile_bits):
    from doki_b200.batch import BatchEngine

    fb = small_batch
    eng = BatchEngine(fb, precision=precision, tile_bits=tile_bits)
    eng.run(keep_states=True)
    eng.sync()
    atol = ATOL_C128 if precision == 2 else ATOL_C64
    rho_all, offs = eng.rho_all()
    for c in range(fb.count):
        psi, rho = oracle_case(orc, oracle_mod, fb, c)
        got = eng.state(c)
        got = got / np.linalg.norm(got)
        assert np.allclose(got, psi, atol=atol, rtol=0), (c, int(fb.num_qubits[c]))
        dim = 1 << int(fb.keep[c])
        r = rho_all[int(offs[c]):int(offs[c]) + dim * dim].reshape(dim, dim)
        assert np.allclose(r, rho, atol=atol, rtol=0), (c, int(fb.num_qubits[c]))
        assert np.allclose(eng.rho(c), r, atol=0)
    eng.close()


def test_batch_graph_relaunch_is_deterministic(dk_gpu, small_batch):
    from doki_b200.batch import BatchEngine

    eng = BatchEngine(small_batch, precision=2, tile_bits=11)
    eng.run()
    eng.sync()
    first, _ = eng.rho_all()
    for _ in range(3):
        eng.run()
    eng.sync()
    again, _ = eng.rho_all()
    assert np.array_equal(first, again)
    # into a caller's (larger, page-locked) buffer
    import torch
    buf = torch.empty(2 * eng.rho_elems + 8, dtype=torch.float64,
                      pin_memory=True).numpy().view(np.complex128)
    into, _ = eng.rho_all(out=buf)
    assert np.array_equal(into[:eng.rho_elems], first)
    bt = eng.build_times()
    assert set(bt) == {"plan_s", "assemble_s", "upload_s"}
    assert bt["plan_s"] > 0 and min(bt.values()) >= 0
    eng.close()


def test_batch_same_result_alone_and_in_the_mix(dk_gpu, small_batch):
    """Each register's result does not depend on what else is in the batch."""
    from doki_b200.batch import BatchEngine

    eng = BatchEngine(small_batch, precision=1, tile_bits=12)
    eng.run()
    eng.sync()
    mix, offs = eng.rho_all()
    for c in (0, 17, 42):
        alone = BatchEngine(small_batch.subset([c]), precision=1, tile_bits=12)
        alone.run()
        alone.sync()
        dim = 1 << int(small_batch.keep[c])
        a = alone.rho(0)
        b = mix[int(offs[c]):int(offs[c]) + dim * dim].reshape(dim, dim)
        assert np.allclose(a, b, atol=1e-12)
        alone.close()
    eng.close()


def test_autotuner_caches(dk_gpu, small_batch, tmp_path):
    from doki_b200.batch import autotune

    cache = str(tmp_path / "tune.json")
    r1 = autotune(small_batch, 1, tile_bits=(10, 12), ctas=(1,), reps=1, cache_path=cache)
    assert r1["tile_bits"] in (10, 12) and not r1["cached"]
    r2 = autotune(small_batch, 1, tile_bits=(10, 12), ctas=(1,), reps=1, cache_path=cache)
    assert r2["cached"] and r2["tile_bits"] == r1["tile_bits"]
    # the pick minimises host planning plus one device run, over every trial
    assert r1["objective"] == "plan+run"
    best = min(t["objective_s"] for t in r1["trials"])
    assert r1["plan_s"] + r1["seconds"] == best
    for t in r1["trials"]:
        same_fold = [u["plan_s"] for u in r1["trials"] if u["fold"] == t["fold"]]
        assert t["objective_s"] == min(same_fold) + t["seconds"]


def test_batch_config_depths_vs_oracle(dk_gpu, orc, oracle_mod):
    """Circuits of the batching workload itself (depth 10-50), a sample of
    every size class, against the oracle; the fusion setting of the plan
    changes nothing beyond rounding."""
    from doki_b200.batch import BatchEngine

    fb = W.batch_arrays(seed=4, count=4096)
    depth = np.diff(fb.op_start.astype(np.int64)) // (fb.num_qubits + fb.num_qubits // 2)
    idx = []
    for n in range(4, 15):
        cand = [int(c) for c in np.nonzero(fb.num_qubits == n)[0] if depth[c] >= 30]
        idx += cand[:1]
    sub = fb.subset(idx)
    for fold in (0, -1, 400):
        eng = BatchEngine(sub, precision=2, tile_bits=12, fold=fold)
        eng.run(keep_states=True)
        eng.sync()
        rho_all, offs = eng.rho_all()
        for c in range(sub.count):
            psi, rho = oracle_case(orc, oracle_mod, sub, c)
            got = eng.state(c)
            assert np.allclose(got / np.linalg.norm(got), psi, atol=ATOL_C128, rtol=0), (fold, c)
            dim = 1 << int(sub.keep[c])
            r = rho_all[int(offs[c]):int(offs[c]) + dim * dim].reshape(dim, dim)
            assert np.allclose(r, rho, atol=ATOL_C128, rtol=0), (fold, c)
        eng.close()


def test_batch_complex64_fidelity_against_complex128(dk_gpu, small_batch):
    """The device comparison of a complex64 batch with the complex128 batch
    of the same circuits equals the host computation on the exported
    states, and the fidelity stays above 1 - 1e-6."""
    from doki_b200.batch import BatchEngine

    e64 = BatchEngine(small_batch, precision=1, tile_bits=12)
    e128 = BatchEngine(small_batch, precision=2, tile_bits=12)
    e64.run(keep_states=True)
    e128.run(keep_states=True)
    e64.sync()
    e128.sync()
    fid, err = e64.compare(e128)
    assert fid.min() > 1 - 1e-6 and err.max() < 5e-5
    for c in (0, 13, 37, small_batch.count - 1):
        x, y = e64.state(c), e128.state(c)
        x, y = x / np.linalg.norm(x), y / np.linalg.norm(y)
        assert abs(fid[c] - abs(np.vdot(x, y)) ** 2) < 1e-12
        assert abs(err[c] - np.abs(x - y).max()) < 1e-12
    e64.close()
    e128.close()
