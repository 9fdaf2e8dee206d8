"""Parity of the CUDA engine with the reference: golden fixtures generated from
the reference module, and the CPU oracle on seeded workloads.

complex128: amplitudes and probabilities within 1e-12 absolute, measurement
outcomes identical.  complex64: within ATOL_C64 of the complex128 oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import (ATOL_C128, ATOL_C64, TIE_C128, TIE_C64, NearTies,
                            assert_same_outcomes)
from tests.golden.gen_golden import random_unitary
from tests.test_plan import random_ops

pytestmark = pytest.mark.gpu


def allamps(d, reg, canonical=False):
    return d.registry_get_all(reg, canonical)


def res_list(res):
    return [-1 if v is None else int(v) for v in res]


# ---------------------------------------------------------------- golden ----

def test_golden_small12(dk_gpu, golden):
    d = dk_gpu
    c = W.small_circuit(seed=1, n=12, depth=20)
    reg = W.run_ops(d, d.registry_new(12, False), c.ops)
    amps = allamps(d, reg)
    assert np.allclose(amps, golden["small12_amps"], atol=ATOL_C128, rtol=0)
    # the element-wise reference accessor agrees with the bulk one
    for i in (0, 1, 777, 4095):
        assert abs(d.registry_get(reg, i, False, False) - golden["small12_amps"][i]) < ATOL_C128
    probs = [d.registry_prob(reg, q, 1, False) for q in range(12)]
    assert np.allclose(probs, golden["small12_probs"], atol=ATOL_C128, rtol=0)
    r0, res = d.registry_measure(reg, (1 << 12) - 1, golden["small12_rolls"].tolist(), 1, False)
    assert r0 is None
    assert res_list(res) == golden["small12_measure_all"].tolist()
    mask = int(golden["small12_half_mask"][0])
    r2, res2 = d.registry_measure(reg, mask, golden["small12_half_rolls"].tolist(), 1, False)
    assert res_list(res2) == golden["small12_half_res"].tolist()
    assert np.allclose(allamps(d, r2, True), golden["small12_half_amps"], atol=ATOL_C128, rtol=0)
    # the measured register is untouched
    assert np.allclose(allamps(d, reg), golden["small12_amps"], atol=ATOL_C128, rtol=0)


@pytest.mark.parametrize("n", range(1, 7))
def test_golden_one_gate(dk_gpu, golden, n):
    d = dk_gpu
    reg = d.registry_new(n, False)
    for q, a in enumerate(golden[f"one_{n}_angles"]):
        reg = d.registry_apply(reg, d.gate_new(1, W.u3(*a).tolist(), False), [q], None, None,
                               1, False)
    assert np.allclose(allamps(d, reg), golden[f"one_{n}_amps"], atol=ATOL_C128, rtol=0)


def test_golden_controls(dk_gpu, golden):
    d = dk_gpu
    order = golden["ctrl_order"].tolist()
    g = d.gate_new(1, W.u3(*golden["ctrl_angles"]).tolist(), False)
    reg = d.registry_apply(d.registry_new(7, False), g, [order[0]], None, None, 1, False)
    ctl, act, is_c = [], [], True
    for prev, q in zip(order, order[1:]):
        (ctl if is_c else act).append(prev)
        reg = d.registry_apply(reg, g, [q], set(ctl), set(act), 1, False)
        is_c = not is_c
    assert np.allclose(allamps(d, reg), golden["ctrl_amps"], atol=ATOL_C128, rtol=0)


def test_golden_pairs(dk_gpu, golden):
    d = dk_gpu
    base = [W.Op(m, [q]) for q, m in enumerate(golden["pair_base"])]
    start = W.run_ops(d, d.registry_new(5, False), base)
    g = d.gate_new(2, golden["pair_u"].tolist(), False)
    i = 0
    for a in range(5):
        for b in range(5):
            if a != b:
                r = d.registry_apply(start, g, [a, b], None, None, 1, False)
                assert np.allclose(allamps(d, r), golden["pair_amps"][i], atol=ATOL_C128,
                                   rtol=0), (a, b)
                i += 1


def test_golden_three_qubit_and_diagonal(dk_gpu, golden):
    d = dk_gpu
    rng = W.rng_for(14)
    random_unitary(rng, 3)
    rng.random(4)
    reg = W.run_ops(d, d.registry_new(6, False),
                    [W.Op(W.u3(*(rng.random(3) * 2 * np.pi)), [q]) for q in range(6)])
    u3q, diag2 = golden["k3_u"], golden["k3_diag2"]
    seq = [(u3q, [4, 0, 2], set(), set()), (diag2, [1, 5], {3}, set()),
           (u3q, [5, 3, 1], set(), {0}), (u3q, [0, 1, 2], {5}, {4})]
    for m, tg, cs, acs in seq:
        reg = d.registry_apply(reg, d.gate_new(len(tg), m.tolist(), False), tg,
                               cs if (cs or acs) else None, acs or None, 1, False)
    assert np.allclose(allamps(d, reg), golden["k3_amps"], atol=ATOL_C128, rtol=0)


def test_golden_join(dk_gpu, golden):
    d = dk_gpu
    regs = [d.registry_apply(d.registry_new(1, False), d.gate_new(1, m.tolist(), False), [0],
                             None, None, 1, False) for m in golden["join_gates"]]
    res = regs[0]
    for r in regs[1:]:
        res = d.registry_join(res, r, 1, False)
    assert np.allclose(allamps(d, res), golden["join_amps"], atol=ATOL_C128, rtol=0)


def test_golden_density_and_partial_trace(dk_gpu, golden):
    d = dk_gpu
    c8 = W.small_circuit(seed=16, n=8, depth=6)
    reg = W.run_ops(d, d.registry_new(8, False), c8.ops)
    rho = d.registry_density(reg, False)
    assert d.funmatrix_shape(rho, False) == (256, 256)
    diag = [d.funmatrix_get(rho, i, i, False) for i in range(256)]
    assert np.allclose(diag, golden["rho8_diag"], atol=ATOL_C128, rtol=0)
    row = [d.funmatrix_get(rho, 5, j, False) for j in range(256)]
    assert np.allclose(row, golden["rho8_row5"], atol=ATOL_C128, rtol=0)
    pt = rho
    for e in golden["rho8_elems"].tolist():
        pt = d.funmatrix_partialtrace(pt, e, False)
    assert d.funmatrix_shape(pt, False) == (32, 32)
    m = np.array([[d.funmatrix_get(pt, i, j, False) for j in range(32)] for i in range(32)])
    assert np.allclose(m, golden["rho8_ptrace"], atol=ATOL_C128, rtol=0)
    assert np.allclose(d.funmatrix_numpy(pt), golden["rho8_ptrace"], atol=ATOL_C128, rtol=0)
    assert abs(d.funmatrix_trace(pt, False) - golden["rho8_ptrace_trace"][0]) < ATOL_C128
    pt2 = rho
    for _ in range(5):
        pt2 = d.funmatrix_partialtrace(pt2, 3, False)
    assert np.allclose(d.funmatrix_numpy(pt2), golden["rho8_low3"], atol=ATOL_C128, rtol=0)


def test_golden_canonical(dk_gpu, golden):
    d = dk_gpu
    rng = W.rng_for(17)
    reg = d.registry_new(4, False)
    for q in range(4):
        ph = np.exp(1j * np.pi * (rng.random() * 2 - 1)) * W.H
        reg = d.registry_apply(reg, d.gate_new(1, ph.tolist(), False), [q], None, None, 1, False)
    assert np.allclose(allamps(d, reg), golden["canon_raw"], atol=ATOL_C128, rtol=0)
    can = [d.registry_get(reg, i, True, False) for i in range(16)]
    assert np.allclose(can, golden["canon_amps"], atol=ATOL_C128, rtol=0)
    r2, res = d.registry_measure(reg, 1, golden["canon_roll"].tolist(), 1, False)
    assert res_list(res) == golden["canon_meas_res"].tolist()
    assert np.allclose(allamps(d, r2, True), golden["canon_meas_amps"], atol=ATOL_C128, rtol=0)


def test_golden_unnormalised_data(dk_gpu, golden):
    d = dk_gpu
    reg = d.registry_new_data(3, golden["data_vals"], False)
    assert np.array_equal(allamps(d, reg), golden["data_raw"])
    assert np.array_equal([d.registry_get(reg, i, False, False) for i in range(8)],
                          golden["data_raw"])
    reg_l = d.registry_new_data(3, golden["data_vals"].tolist(), False)
    assert np.array_equal(allamps(d, reg_l), golden["data_raw"])
    r2 = d.registry_apply(reg, d.gate_new(1, W.H.tolist(), False), [1], None, None, 1, False)
    assert np.allclose(allamps(d, r2), golden["data_after_h"], atol=ATOL_C128, rtol=0)
    probs = [d.registry_prob(reg, q, 1, False) for q in range(3)]
    assert np.allclose(probs, golden["data_prob"], atol=ATOL_C128, rtol=0)


# ---------------------------------------------------------------- oracle ----

@pytest.mark.parametrize("n,count", [(3, 40), (5, 80), (9, 120), (12, 150), (14, 150),
                                     (16, 120), (19, 60)])
def test_random_circuits_vs_oracle(dk_gpu, orc, n, count):
    d = dk_gpu
    rng = W.rng_for(5000 + n)
    ops = random_ops(rng, n, count)
    if n >= 5:
        ops.insert(count // 2, W.Op(random_unitary(rng, 4), [0, n - 1, 1, n // 2]))
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    assert np.allclose(allamps(d, a), orc.registry_get_all(b), atol=ATOL_C128, rtol=0)
    assert np.allclose(d.registry_probs(a), orc.registry_probs(b), atol=ATOL_C128, rtol=0)


@pytest.mark.parametrize("fuse", [False, True])
def test_fused_equals_unfused(dk_gpu, orc, fuse):
    d = dk_gpu
    n = 15
    ops = random_ops(W.rng_for(77), n, 100)
    d.engine_set_fusion(fuse)
    try:
        a = W.run_ops(d, d.registry_new(n, False), ops)
        got = allamps(d, a)
    finally:
        d.engine_set_fusion(True)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    assert np.allclose(got, orc.registry_get_all(b), atol=ATOL_C128, rtol=0)


@pytest.mark.parametrize("n", [22, 23])
def test_conditioned_in_place_sweeps_keep_the_norm(dk_gpu, orc, n):
    """Sweeps whose gates all depend on one qubit outside the tile skip the
    tiles where it is 0 and update the stored norm from the touched tiles
    only; repeated many times, the normalised state must keep unit norm and
    equal the oracle."""
    d = dk_gpu
    rng = W.rng_for(900 + n)
    ops = [W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q]) for q in range(n)]
    reg = W.run_ops(d, d.registry_new(n, False), ops)
    d.registry_flush(reg)
    c = n - 1  # far control: outside every tile
    for rnd in range(24):
        batch = []
        for j in range(6):
            m = W.u3(*rng.uniform(0, 2 * np.pi, 3))
            batch.append(W.Op(m, [(rnd + j) % 6], {c} if rnd % 3 else set(), set() if rnd % 3 else {c}))
        reg = W.run_ops(d, reg, batch)
        d.registry_flush(reg)
        amps = allamps(d, reg)
        assert abs(float(np.sum(np.abs(amps) ** 2)) - 1.0) < 1e-12, rnd
        ops += batch
    want = W.run_ops(orc, orc.registry_new(n), ops)
    assert np.allclose(amps, orc.registry_get_all(want), atol=ATOL_C128, rtol=0)


def test_copy_on_write_semantics(dk_gpu):
    """Every operation returns a new register; inputs are never mutated."""
    d = dk_gpu
    n = 14
    g = d.gate_new(1, W.H.tolist(), False)
    r0 = d.registry_new(n, False)
    r1 = d.registry_apply(r0, g, [0], None, None, 1, False)
    r2 = d.registry_apply(r1, g, [13], None, None, 1, False)
    c2 = d.registry_clone(r2, 1, False)
    r3 = d.registry_apply(r2, g, [0], None, None, 1, False)
    v0, v1, v2, v3 = (allamps(d, r) for r in (r0, r1, r2, r3))
    assert v0[0] == 1 and np.count_nonzero(v0) == 1
    assert np.allclose(abs(v1[[0, 1]]), 2 ** -0.5) and np.count_nonzero(np.abs(v1) > 1e-15) == 2
    assert np.count_nonzero(np.abs(v2) > 1e-15) == 4
    assert np.allclose(abs(v3[[0, 1 << 13]]), 2 ** -0.5)
    assert np.allclose(allamps(d, c2), v2, atol=0)
    d.registry_del(r1, False)
    with pytest.raises(d.error):
        d.registry_get(r1, 0, False, False)
    assert np.allclose(allamps(d, r2), v2, atol=0)


def test_measure_sequence_vs_oracle(dk_gpu, orc):
    d = dk_gpu
    n = 16
    ops = random_ops(W.rng_for(31), n, 120)
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    rng = W.rng_for(32)
    ties = NearTies()
    for trial in range(6):
        mask = int(rng.integers(1, 1 << n))
        rolls = rng.random(bin(mask).count("1")).tolist()
        ra, resa = d.registry_measure(a, mask, rolls, 1, False)
        rb, resb = orc.registry_measure(b, mask, rolls)
        if not ties.check(res_list(resa), res_list(resb), orc.last_margins, TIE_C128,
                          f" (trial {trial})"):
            continue
        if rb is not None:
            assert np.allclose(allamps(d, ra), orc.registry_get_all(rb), atol=ATOL_C128, rtol=0)
    ties.finish()


@pytest.mark.parametrize("n,prec", [(22, 2), (20, 1), (13, 2)])
def test_measure_joint_vs_oracle(dk_gpu, orc, n, prec):
    """Measurement of 1 to 12 qubits in one pass (joint distribution of the
    measured qubits, outcomes decided highest first, one collapse): the
    outcomes equal the reference sequence's and the collapsed register the
    oracle's, for masks with low, high and scattered qubits."""
    d = dk_gpu
    rng = W.rng_for(600 + n)
    ops = random_ops(rng, n, 80)
    ops += [W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q]) for q in range(n)]
    a = W.run_ops(d, d.registry_new(n, False, prec), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    masks = [1, 1 << (n - 1), 0b1011, (1 << (n - 1)) | 1 | (1 << (n // 2)),
             sum(1 << int(q) for q in rng.choice(n, size=min(12, n), replace=False)),
             sum(1 << int(q) for q in rng.choice(n, size=5, replace=False)),
             sum(1 << int(q) for q in rng.choice(n, size=6, replace=False)),
             0b1111111]
    ties = NearTies()
    for mask in masks:
        for _ in range(3):
            rolls = rng.random(bin(mask).count("1")).tolist()
            ra, resa = d.registry_measure(a, mask, rolls, 1, False)
            rb, resb = orc.registry_measure(b, mask, rolls)
            if not ties.check(res_list(resa), res_list(resb), orc.last_margins,
                              TIE_C128 if prec == 2 else TIE_C64, f" (mask {mask:#x})"):
                continue
            if rb is not None:
                tol = ATOL_C128 if prec == 2 else ATOL_C64
                assert np.allclose(allamps(d, ra), orc.registry_get_all(rb), atol=tol, rtol=0)
    ties.finish()


def test_measure_joint_unnormalised_data(dk_gpu, orc):
    """Data registers are not normalised: the first outcome compares the
    probability relative to the stored norm, as the reference does."""
    d = dk_gpu
    rng = W.rng_for(77)
    n = 9
    vals = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) * 0.07
    a = d.registry_new_data(n, vals.tolist(), False)
    b = orc.registry_new_data(n, vals.tolist())
    ties = NearTies()
    for mask in (0b101, 0b110000001, (1 << n) - 1):
        for _ in range(4):
            rolls = rng.random(bin(mask).count("1")).tolist()
            ra, resa = d.registry_measure(a, mask, rolls, 1, False)
            rb, resb = orc.registry_measure(b, mask, rolls)
            if not ties.check(res_list(resa), res_list(resb), orc.last_margins, TIE_C128,
                              f" (mask {mask:#x})"):
                continue
            if rb is not None:
                assert np.allclose(allamps(d, ra), orc.registry_get_all(rb), atol=ATOL_C128,
                                   rtol=0)
    ties.finish()


def test_reduced_density_vs_oracle(dk_gpu, orc, oracle_mod):
    d = dk_gpu
    n = 14
    ops = random_ops(W.rng_for(41), n, 100)
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    rho = d.registry_density(a, False)
    # keep the low 6 qubits (trace out 13..6)
    pt = rho
    for e in range(n - 1, 5, -1):
        pt = d.funmatrix_partialtrace(pt, e, False)
    want = oracle_mod.reduced_density(b, 0b111111)
    assert np.allclose(d.funmatrix_numpy(pt), want, atol=ATOL_C128, rtol=0)
    # a scattered kept set
    elems = [12, 9, 9, 4, 0, 3, 1]
    pt = rho
    for e in elems:
        pt = d.funmatrix_partialtrace(pt, e, False)
    keep = oracle_mod.kept_mask_after_traces(n, elems)
    want = oracle_mod.reduced_density(b, keep)
    got = d.funmatrix_numpy(pt)
    assert np.allclose(got, want, atol=ATOL_C128, rtol=0)
    assert abs(d.funmatrix_trace(pt, False) - np.trace(want)) < 1e-11


def test_density_algebra_vs_oracle(dk_gpu, orc, oracle_mod):
    """Lazy algebra over register-backed density matrices: modifiers on top of
    the device reduced-density path, modified nodes inside a partial-trace
    chain (element-wise path), products and a gate applied to a column."""
    d = dk_gpu
    n = 6
    ops = random_ops(W.rng_for(43), n, 40)
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    psi = orc.registry_get_all(b)
    full = np.outer(psi, psi.conj())
    rho = d.registry_density(a, False)
    tol = dict(atol=ATOL_C128, rtol=0)
    assert np.allclose(d.funmatrix_numpy(d.funmatrix_dagger(rho, False)), full.conj().T, **tol)
    # device path under a scalar and a transpose on the top node
    low5 = oracle_mod.reduced_density(b, 0b011111)
    pt = d.funmatrix_partialtrace(rho, n - 1, False)
    assert np.allclose(d.funmatrix_numpy(d.funmatrix_scalar_mul(pt, 2 - 1j, False)),
                       (2 - 1j) * low5, **tol)
    pt4 = d.funmatrix_partialtrace(pt, n - 2, False)
    low4 = oracle_mod.reduced_density(b, 0b001111)
    assert np.allclose(d.funmatrix_numpy(d.funmatrix_transpose(pt4, False)), low4.T, **tol)
    # a modified node inside the chain: element-wise partial trace
    scaled = d.funmatrix_scalar_div(rho, 4, False)
    ptg = d.funmatrix_partialtrace(d.funmatrix_partialtrace(scaled, 0, False), 2, False)
    keep = oracle_mod.kept_mask_after_traces(n, [0, 2])
    assert np.allclose(d.funmatrix_numpy(ptg), oracle_mod.reduced_density(b, keep) / 4, **tol)
    # products of reduced density matrices and identities
    sq = d.funmatrix_matmul(pt4, pt4, False)
    assert np.allclose(d.funmatrix_numpy(sq), low4 @ low4, **tol)
    assert abs(d.funmatrix_trace(sq, False) - np.trace(low4 @ low4)) < 1e-12
    kr = d.funmatrix_kron(pt4, d.funmatrix_identity(1, False), False)
    assert np.allclose(d.funmatrix_numpy(kr), np.kron(low4, np.eye(2)), **tol)
    ek = d.funmatrix_eyekron(pt4, 1, 0, False)
    assert np.allclose(d.funmatrix_numpy(ek), np.kron(np.eye(2), low4), **tol)
    # a Hadamard on qubit 3 of column 0 of rho (psi * conj(psi_0))
    col = d.funmatrix_matmul(rho, d.funmatrix_statezero(n, False), False)
    h = d.funmatrix_apply(col, d.funmatrix_hadamard(1, False), [3], {1}, None, False)
    x = full[:, 0]
    want = x.copy()
    for i in range(1 << n):
        if i & 2:
            lo, hi = x[i & ~8], x[i | 8]
            want[i] = (lo + hi) / np.sqrt(2) if not i & 8 else (lo - hi) / np.sqrt(2)
    assert np.allclose(d.funmatrix_numpy(h)[:, 0], want, **tol)


@pytest.mark.parametrize("n,keep_bits,prec", [(12, 3, 2), (16, 5, 2), (16, 6, 2), (18, 8, 2),
                                               (20, 10, 2), (18, 7, 1), (20, 10, 1), (17, 9, 2)])
def test_reduced_density_sizes(dk_gpu, orc, oracle_mod, n, keep_bits, prec):
    """The tensor-core product X X^H over kept sets from 8 to 1024 amplitudes:
    one or many output tiles, split and unsplit traced ranges, contiguous and
    scattered kept qubits, complex128 and complex64 registers."""
    d = dk_gpu
    rng = W.rng_for(1300 + n + keep_bits)
    ops = random_ops(rng, n, 60)
    ops += [W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q]) for q in range(n)]
    a = W.run_ops(d, d.registry_new(n, False, prec), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    for scattered in (False, True):
        if scattered:
            kept = sorted(int(x) for x in rng.choice(n, size=keep_bits, replace=False))
        else:
            kept = list(range(keep_bits))
        keep = sum(1 << q for q in kept)
        traced = [q for q in range(n) if q not in kept]
        pt = d.registry_density(a, False)
        for q in sorted(traced, reverse=True):
            pt = d.funmatrix_partialtrace(pt, q, False)
        got = d.funmatrix_numpy(pt)
        want = oracle_mod.reduced_density(b, keep)
        tol = ATOL_C128 if prec == 2 else ATOL_C64
        assert np.allclose(got, want, atol=tol, rtol=0), (scattered, np.abs(got - want).max())
        assert np.allclose(got, got.conj().T, atol=1e-14)


def test_join_vs_oracle(dk_gpu, orc):
    d = dk_gpu
    oa = random_ops(W.rng_for(51), 9, 60)
    ob = random_ops(W.rng_for(52), 8, 60)
    a = W.run_ops(d, d.registry_new(9, False), oa)
    b = W.run_ops(d, d.registry_new(8, False), ob)
    j = d.registry_join(a, b, 1, False)
    ja = W.run_ops(orc, orc.registry_new(9), oa)
    jb = W.run_ops(orc, orc.registry_new(8), ob)
    jo = orc.registry_join(ja, jb)
    assert np.allclose(allamps(d, j), orc.registry_get_all(jo), atol=ATOL_C128, rtol=0)


def test_canonical_phase_vs_oracle(dk_gpu, orc):
    d = dk_gpu
    n = 12
    ops = random_ops(W.rng_for(61), n, 50)
    # zero out a leading block so the first non-zero amplitude is not index 0
    ops.append(W.Op(np.array([[0, 0], [0, 1]], dtype=complex), [0]))
    ops.append(W.Op(np.array([[0, 0], [0, 1]], dtype=complex), [3]))
    a = W.run_ops(d, d.registry_new(n, False), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    assert np.allclose(allamps(d, a, True), orc.registry_get_all(b, canonical=True),
                       atol=ATOL_C128, rtol=0)


def test_inverse_circuit_roundtrip_24q(dk_gpu):
    """Size-independent property at 24 qubits: U then U^dagger returns |0>."""
    d = dk_gpu
    n = 24
    ops = random_ops(W.rng_for(71), n, 150)
    inv = [W.Op(op.gate.conj().T, op.targets, op.controls, op.anticontrols)
           for op in reversed(ops)]
    r = W.run_ops(d, d.registry_new(n, False), ops + inv)
    assert abs(d.registry_get(r, 0, False, False) - 1) < 1e-12
    p = d.registry_probs(r)
    assert max(p) < 1e-12


def test_complex64_vs_complex128_oracle(dk_gpu, orc):
    d = dk_gpu
    n = 16
    ops = random_ops(W.rng_for(81), n, 150)
    a = W.run_ops(d, d.registry_new(n, False, 1), ops)
    assert d.registry_precision(a) == 1
    b = W.run_ops(orc, orc.registry_new(n), ops)
    va, vb = allamps(d, a), orc.registry_get_all(b)
    assert np.max(np.abs(va - vb)) < ATOL_C64
    fid = abs(np.vdot(vb, va)) ** 2 / (np.vdot(va, va).real * np.vdot(vb, vb).real)
    assert fid > 1 - 1e-6
    assert np.allclose(d.registry_probs(a), orc.registry_probs(b), atol=ATOL_C64)
    rolls = [0.3, 0.7, 0.1]
    ra, resa = d.registry_measure(a, 0b1010000000001, rolls, 1, False)
    rb, resb = orc.registry_measure(b, 0b1010000000001, rolls)
    assert_same_outcomes(res_list(resa), res_list(resb), orc.last_margins, TIE_C64)


@pytest.mark.parametrize("n", [8, 9, 10, 11, 13])
def test_complex64_tile_widths_vs_complex128_oracle(dk_gpu, orc, n):
    """complex64 sweeps on every tile width of the split-TF32 kernel (8 to 12
    qubits) against the complex128 oracle, within the complex64 tolerance."""
    d = dk_gpu
    ops = random_ops(W.rng_for(90 + n), n, 120)
    a = W.run_ops(d, d.registry_new(n, False, 1), ops)
    b = W.run_ops(orc, orc.registry_new(n), ops)
    va, vb = allamps(d, a), orc.registry_get_all(b)
    assert np.max(np.abs(va - vb)) < ATOL_C64
    fid = abs(np.vdot(vb, va)) ** 2 / (np.vdot(va, va).real * np.vdot(vb, vb).real)
    assert fid > 1 - 1e-6


def test_complex64_brickwork_vs_complex128_oracle(dk_gpu, orc):
    """The benchmark's brickwork generator (chained pass pairs, conditioned
    variants) on a complex64 register."""
    d = dk_gpu
    n = 14
    c = W.scale_circuit(seed=2, n=n, depth=12, keep=6)
    a = W.run_ops(d, d.registry_new(n, False, 1), c.ops)
    b = W.run_ops(orc, orc.registry_new(n), c.ops)
    va, vb = allamps(d, a), orc.registry_get_all(b)
    assert np.max(np.abs(va - vb)) < ATOL_C64
    assert np.allclose(d.registry_probs(a), orc.registry_probs(b), atol=ATOL_C64)


_C64_RUN = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import doki_b200
from doki_b200 import workloads as W
d = doki_b200.load()
n = int(sys.argv[2])
c = W.scale_circuit(seed=3, n=n, depth=10, keep=6)
a = W.run_ops(d, d.registry_new(n, False, 1), c.ops)
np.save(sys.argv[3], np.asarray(d.registry_get_all(a, False)))
st = d.engine_stats()
print("tm", st["tm_sweeps_presplit"], st["tm_sweeps_entry_b"])
"""


@pytest.mark.parametrize("n", [14, 20])
def test_complex64_tcgen05_b_split_per_entry_and_per_cta(dk_gpu, orc, n, tmp_path):
    """Both ways the tcgen05 sweep gets its B operands -- split once per CTA
    for the whole sweep (default) and split per entry (the path of sweeps
    whose matrices do not fit, forced here by DK_C64_TMEM_PRESPLIT=0) --
    against the complex128 oracle, each in its own process."""
    import os
    import subprocess
    import sys
    from tests.conftest import ROOT
    c = W.scale_circuit(seed=3, n=n, depth=10, keep=6)
    want = orc.registry_get_all(W.run_ops(orc, orc.registry_new(n), c.ops))
    for pre in ("1", "0"):
        out = str(tmp_path / f"amps{pre}.npy")
        r = subprocess.run([sys.executable, "-c", _C64_RUN, ROOT, str(n), out],
                           env=dict(os.environ, DK_C64_TMEM="1", DK_C64_TMEM_PRESPLIT=pre),
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        tm = [ln for ln in r.stdout.splitlines() if ln.startswith("tm ")][0].split()
        presplit, per_entry = int(tm[1]), int(tm[2])
        if pre == "1":
            assert presplit > 0, tm
        else:
            assert presplit == 0 and per_entry > 0, tm
        got = np.load(out)
        assert np.max(np.abs(got - want)) < ATOL_C64


# ------------------------------------------------------- error behaviour ----

def test_device_side_errors(dk_gpu):
    d = dk_gpu
    r = d.registry_new(3, False)
    g = d.gate_new(1, W.X.tolist(), False)
    msgs = {}
    for name, f in [
        ("actrl_none", lambda: d.registry_apply(r, g, [0], None, {1}, 1, False)),
        ("same", lambda: d.registry_apply(r, g, [0], {1}, {1}, 1, False)),
        ("tinc", lambda: d.registry_apply(r, g, [1], {1}, None, 1, False)),
        ("oor", lambda: d.registry_apply(r, g, [5], None, None, 1, False)),
        ("ntg", lambda: d.registry_apply(r, g, [0, 1], None, None, 1, False)),
        ("roll", lambda: d.registry_measure(r, 1, [1.0], 1, False)),
        ("short", lambda: d.registry_measure(r, 3, [0.5], 1, False)),
    ]:
        with pytest.raises(d.error) as ei:
            f()
        msgs[name] = str(ei.value)
    assert msgs["actrl_none"] == "A control cannot also be an anticontrol"
    assert msgs["same"] == "A control cannot also be an anticontrol"
    assert msgs["tinc"] == "A target cannot also be a control or an anticontrol"
    assert msgs["oor"] == "Target qubit out of range"
    assert msgs["ntg"] == "Wrong number of targets specified for that gate"
    assert msgs["roll"] == msgs["short"] == "roll not in interval [0, 1)!"
    r0, res = d.registry_measure(r, 0, [], 1, False)
    assert res == [None, None, None] and r0 is not None


def test_tensor_work_counter(dk_gpu):
    """engine_stats()["mma_entry_amplitudes"] grows by (matrix entries) x
    (register amplitudes) for each tensor sweep, so it is a multiple of 2^n."""
    d = dk_gpu
    n = 14
    before = d.engine_stats()["mma_entry_amplitudes"]
    c = W.scale_circuit(seed=2, n=n, depth=6, keep=6)
    r = W.run_ops(d, d.registry_new(n, False), c.ops)
    d.registry_flush(r)
    grown = d.engine_stats()["mma_entry_amplitudes"] - before
    assert grown > 0 and grown % (1 << n) == 0


def test_registry_mem_reports_device_storage(dk_gpu):
    """registry_mem (reference state_mem_size, qstate.c:123-135: header +
    amplitude storage) reports the register's device amplitude bytes
    (16 or 8 per amplitude) plus a fixed part -- the host header and the
    device scalar block -- that does not depend on the size.  A clone shares
    the storage and reports the same; a deleted registry reports the fixed
    host header only."""
    d = dk_gpu
    fixed = set()
    for n in (1, 5, 12, 20):
        for prec, amp in ((2, 16), (1, 8)):
            r = d.registry_new(n, False, prec)
            fixed.add(d.registry_mem(r, False) - (amp << n))
            c = d.registry_clone(r, 1, False)
            assert d.registry_mem(c, False) == d.registry_mem(r, False)
    assert len(fixed) == 1
    base = fixed.pop()
    assert 48 < base < 4096
    r = d.registry_new(10, False)
    d.registry_del(r, False)
    assert d.registry_mem(r, False) == base - 48  # the 48-byte scalar block is gone
