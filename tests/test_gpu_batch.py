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
