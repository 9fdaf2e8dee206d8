"""Host logic of the gate-fusion planner (doki_b200/csrc/dk_plan.c), on CPU.

The planner's sweep programs are read back through ctypes and replayed by a
numpy model of the sweep kernel's semantics (tile gather over the sweep's
qubit set, passes in order, gates with local / per-tile controls, packed
matrices).  The replay must equal gate-by-gate application by the oracle.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import ROOT
from tests.golden.gen_golden import random_unitary

MAXK = 10


class FlatOp(ctypes.Structure):
    _fields_ = [("gate", ctypes.c_void_p), ("k", ctypes.c_uint),
                ("tg", ctypes.c_uint * MAXK), ("cm", ctypes.c_uint64),
                ("am", ctypes.c_uint64)]


class Limits(ctypes.Structure):
    _fields_ = [("tile_bits", ctypes.c_int), ("low_bits", ctypes.c_int),
                ("max_gates", ctypes.c_int), ("max_passes", ctypes.c_int),
                ("max_mat", ctypes.c_int), ("fuse", ctypes.c_int),
                ("fold", ctypes.c_int), ("tensor", ctypes.c_int),
                ("bank_mode", ctypes.c_int)]


class Step(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("prog_off", ctypes.c_size_t),
                ("op_index", ctypes.c_int), ("ngates", ctypes.c_int)]


class Plan(ctypes.Structure):
    _fields_ = [("steps", ctypes.POINTER(Step)), ("nsteps", ctypes.c_int),
                ("blob", ctypes.POINTER(ctypes.c_ubyte)), ("blob_bytes", ctypes.c_size_t)]


HDR = np.dtype([("m", "<i4"), ("n", "<i4"), ("npass", "<i4"), ("ngate", "<i4"),
                ("all_touched", "<i4"), ("mode", "<i4"), ("ntiles", "<u8"),
                ("qpos", "u1", 16), ("pass_off", "<u4"), ("gate_off", "<u4"),
                ("mat_off", "<u4"), ("bytes", "<u4"), ("cond_off", "<u4"),
                ("ncond", "<u4"), ("bankv", "<u8")])
PASS = np.dtype([("g0", "<u2"), ("g1", "<u2"), ("flags", "<u4"), ("sp", "<u4", 3),
                 ("pm", "<u4", 3), ("slo", "<u4", 32), ("shi", "<u4", 16),
                 ("rlo", "<u4", 32), ("rhi", "<u4", 16)])
GATE = np.dtype([("code", "<u2"), ("mat", "<u2"), ("gcond", "<u2"), ("info", "<u2"),
                 ("lc", "<u4"), ("la", "<u4")])
COND = np.dtype([("gc", "<u8"), ("ga", "<u8")])
assert HDR.itemsize == 80 and PASS.itemsize == 416 and GATE.itemsize == 16


@pytest.fixture(scope="module")
def lib():
    L = ctypes.CDLL(os.path.join(ROOT, "doki_b200", "libdokigpu.so"))
    L.dk_gate_new.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.dk_plan_default_limits.argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.POINTER(Limits)]
    L.dk_plan_build.argtypes = [ctypes.POINTER(FlatOp), ctypes.c_int, ctypes.c_uint,
                                ctypes.c_int, ctypes.POINTER(Limits), ctypes.POINTER(Plan)]
    L.dk_plan_free.argtypes = [ctypes.POINTER(Plan)]
    L.dk_gate_free.argtypes = [ctypes.c_void_p]
    return L


def build_plan(lib, ops, n, prec=2, fuse=1, tile_bits=None, fold=0, tensor=0, bank_mode=0):
    gates, flat = [], (FlatOp * len(ops))()
    for i, op in enumerate(ops):
        m = np.ascontiguousarray(op.gate, dtype=np.complex128)
        g = ctypes.c_void_p()
        assert lib.dk_gate_new(op.k, m.ctypes.data, ctypes.byref(g)) == 0
        gates.append(g)
        flat[i].gate = g
        flat[i].k = op.k
        for j, t in enumerate(op.targets):
            flat[i].tg[j] = t
        flat[i].cm = sum(1 << c for c in op.controls)
        flat[i].am = sum(1 << c for c in op.anticontrols)
    lim = Limits()
    lim.fold = fold
    lim.tensor = tensor
    lib.dk_plan_default_limits(prec, n, ctypes.byref(lim))
    lim.fuse = fuse
    lim.bank_mode = bank_mode
    if tile_bits is not None:
        lim.tile_bits = tile_bits
    plan = Plan()
    assert lib.dk_plan_build(flat, len(ops), n, prec, ctypes.byref(lim), ctypes.byref(plan)) == 0
    blob = bytes(ctypes.cast(plan.blob, ctypes.POINTER(ctypes.c_ubyte * plan.blob_bytes))
                 .contents) if plan.blob_bytes else b""
    steps = [(plan.steps[i].kind, plan.steps[i].prog_off, plan.steps[i].op_index)
             for i in range(plan.nsteps)]
    lib.dk_plan_free(ctypes.byref(plan))
    for g in gates:
        lib.dk_gate_free(g)
    return steps, blob


def apply_local(vec, mat, tbits, ok):
    """Apply a 2^k x 2^k matrix on local bits `tbits` (targets[0] = LSB) to the
    entries of `vec` whose boolean mask `ok` holds."""
    k = len(tbits)
    out = vec.copy()
    idx = np.arange(vec.size)
    tmask = sum(1 << b for b in tbits)
    bases = idx[(idx & tmask) == 0]
    for b in bases:
        if not ok[b]:
            continue
        members = [b | sum(((g >> j) & 1) << tbits[j] for j in range(k)) for g in range(1 << k)]
        out[members] = mat @ vec[members]
    return out


def assert_code(code, kind, treg, ctl):
    """The kernel's entry code must agree with the gate's kind and bits."""
    one_q = {1: 0, 7: 6, 8: 12, 2: 18, 3: 24, 9: 37}
    if kind in one_q:
        assert code == one_q[kind] + treg[0] + 3 * (ctl != 0)
    elif kind == 4:
        pairs = [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]
        assert code == 30 + pairs.index((treg[0], treg[1]))
    elif kind == 5:
        assert code in (43, 44, 45) and treg == [0, 1, 2]
        assert code == 45 or code == 43 + (ctl != 0)
    else:
        assert kind == 6 and code == 36


def replay_sweep(blob, off, psi):
    h = np.frombuffer(blob, HDR, 1, off)[0]
    m, n = int(h["m"]), int(h["n"])
    qpos = [int(x) for x in h["qpos"][:m]]
    passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
    gates = np.frombuffer(blob, GATE, int(h["ngate"]), off + int(h["gate_off"]))
    conds = np.frombuffer(blob, COND, int(h["ncond"]), off + int(h["cond_off"]))
    nmat = (int(h["bytes"]) - int(h["mat_off"])) // 16
    mats = np.frombuffer(blob, np.complex128, nmat, off + int(h["mat_off"]))
    tensor = int(h["mode"]) == 1
    qmask = sum(1 << q for q in qpos)
    out = psi.copy()
    local = np.arange(1 << m)
    offs = np.zeros(1 << m, dtype=np.int64)
    for j, q in enumerate(qpos):
        offs |= ((local >> j) & 1) << q
    rest = [q for q in range(n) if not (qmask >> q) & 1]
    for t in range(int(h["ntiles"])):
        base = sum(((t >> j) & 1) << q for j, q in enumerate(rest))
        tile = out[base | offs].copy()
        for p in passes:
            for gi in range(int(p["g0"]), int(p["g1"])):
                g = gates[gi]
                if int(g["gcond"]) != 0xffff:
                    c = conds[int(g["gcond"])]
                    gc, ga = int(c["gc"]), int(c["ga"])
                    if (base & gc) != gc or (base & ga):
                        continue
                lc, la = int(g["lc"]), int(g["la"])
                info = int(g["info"])
                k = (info >> 6) & 3
                treg = [info & 3, (info >> 2) & 3, (info >> 4) & 3]
                tb = [int(p["pm"][treg[j]]).bit_length() - 1 for j in range(k)]
                kind, mo = info >> 8, int(g["mat"]) * (64 if tensor else 1)
                assert_code(int(g["code"]), kind, treg, lc | la)
                if int(g["code"]) == 45:
                    # variant entry: the tile's conditions select the matrix
                    assert tensor and 1 <= la <= 3
                    for c in range(la):
                        cc = conds[(lc >> (10 * c)) & 1023]
                        gc, ga = int(cc["gc"]), int(cc["ga"])
                        if (base & gc) == gc and not (base & ga):
                            mo += 64 << c
                    lc = la = 0
                ok = ((local & lc) == lc) & ((local & la) == 0)
                if kind == 1 or kind == 4 or kind == 5:
                    mat = mats[mo:mo + (1 << 2 * k)].reshape(1 << k, 1 << k)
                elif kind == 2:
                    mat = np.diag(mats[mo:mo + 2])
                elif kind == 3:
                    mat = np.array([[0, mats[mo]], [mats[mo + 1], 0]])
                elif kind == 6:
                    mat = np.diag(mats[mo:mo + (1 << k)])
                elif kind == 7:
                    mat = np.array([[0, 1], [1, 0]], dtype=complex)
                elif kind == 8:
                    mat = np.diag([1, mats[mo]])
                elif kind == 9:
                    mat = np.diag([1, -1]).astype(complex)
                else:
                    raise AssertionError(kind)
                tile = apply_local(tile, mat, tb, ok)
        out[base | offs] = tile
    return out


def run_plan(lib, ops, n, psi, **kw):
    steps, blob = build_plan(lib, ops, n, **kw)
    for kind, off, opi in steps:
        if kind == 1:
            psi = replay_sweep(blob, off, psi)
        else:
            op = ops[opi]
            cm = sum(1 << c for c in op.controls)
            am = sum(1 << c for c in op.anticontrols)
            idx = np.arange(psi.size)
            ok = ((idx & cm) == cm) & ((idx & am) == 0)
            psi = apply_local(psi, op.gate, list(op.targets), ok)
    return psi, steps


def oracle_run(orc, ops, n):
    reg = W.run_ops(orc, orc.registry_new(n), ops)
    return orc.registry_get_all(reg) * reg.norm  # raw (unnormalised) product


def random_ops(rng, n, count, kmax=3):
    ops = []
    for _ in range(count):
        k = int(rng.integers(1, min(kmax, n) + 1))
        tg = [int(x) for x in rng.choice(n, size=k, replace=False)]
        free = [q for q in range(n) if q not in tg]
        nc = int(rng.integers(0, min(3, len(free)) + 1)) if rng.random() < 0.4 else 0
        cs = [int(x) for x in rng.choice(free, size=nc, replace=False)] if nc else []
        ctl = {q for q in cs if rng.random() < 0.5}
        r = rng.random()
        if k == 1 and r < 0.2:
            m = W.X.copy()
        elif k == 1 and r < 0.3:
            m = np.diag(np.exp(2j * np.pi * rng.random(2)))
        elif k == 1 and r < 0.35:
            m = np.diag([1, np.exp(2j * np.pi * rng.random())])
        elif k == 1 and r < 0.4:
            m = W.Z.copy()
        elif k == 2 and r < 0.3:
            m = np.diag(np.exp(2j * np.pi * rng.random(4)))
        else:
            m = random_unitary(rng, k)
        ops.append(W.Op(m, tg, ctl, set(cs) - ctl))
    return ops


@pytest.mark.parametrize("fold,tensor", [(0, 0), (0, -1), (-1, -1), (1, -1), (400, -1)])
@pytest.mark.parametrize("n,tile_bits", [(5, None), (8, None), (10, 6), (11, 7), (12, 8),
                                         (12, None), (14, None)])
def test_plan_replay_matches_oracle(lib, orc, n, tile_bits, fold, tensor):
    rng = W.rng_for(1000 + n)
    ops = random_ops(rng, n, 60)
    ops.append(W.Op(random_unitary(rng, 4), [0, n - 1, 2, n - 2]))  # generic step
    ops += random_ops(rng, n, 20)
    psi0 = np.zeros(1 << n, dtype=np.complex128)
    psi0[0] = 1
    got, steps = run_plan(lib, ops, n, psi0, tile_bits=tile_bits, fold=fold, tensor=tensor)
    want = oracle_run(orc, ops, n)
    assert np.allclose(got / np.linalg.norm(got), want / np.linalg.norm(want), atol=1e-12)
    assert any(s[0] == 2 for s in steps)
    assert sum(1 for s in steps if s[0] == 1) < len(ops) / 2  # fusion happened


def test_plan_unfused_one_gate_per_sweep(lib, orc):
    n = 9
    ops = random_ops(W.rng_for(7), n, 30)
    psi0 = np.zeros(1 << n, dtype=np.complex128)
    psi0[0] = 1
    got, steps = run_plan(lib, ops, n, psi0, fuse=0, tile_bits=6)
    assert len(steps) == len(ops)
    want = oracle_run(orc, ops, n)
    assert np.allclose(got / np.linalg.norm(got), want / np.linalg.norm(want), atol=1e-12)


def test_plan_scale_circuit_fusion_ratio(lib):
    """At 30 qubits the depth-40 workload fuses into ~2 sweeps per layer."""
    c = W.scale_circuit(seed=2, n=30, depth=40)
    steps, blob = build_plan(lib, c.ops, 30, fold=-1, tensor=-1)
    nsweeps = sum(1 for s in steps if s[0] == 1)
    assert all(s[0] == 1 for s in steps)
    assert nsweeps <= 3 * c.depth
    tot = sum(int(np.frombuffer(blob, HDR, 1, off)[0]["ngate"]) for _, off, _ in steps)
    assert tot == len(c.ops)
    # pass folding keeps the sweeps and shortens their gate lists
    fsteps, fblob = build_plan(lib, c.ops, 30, tensor=-1)
    assert len(fsteps) == len(steps)
    ftot = sum(int(np.frombuffer(fblob, HDR, 1, off)[0]["ngate"]) for _, off, _ in fsteps)
    assert ftot < 0.75 * tot


def swizzle(i, sw):
    f = 0
    s = sw
    while s < 20:
        f ^= i >> s
        s += sw
    return i ^ (f & ((1 << sw) - 1))


def swizzle_map(i, bankv):
    """The tile layout of a sweep header's bank map (dk_sweep_hdr.bankv)."""
    f = 0
    for b in range(16):
        if (i >> b) & 1:
            f ^= (int(bankv) >> (4 * b)) & 15
    return i ^ f


@pytest.mark.parametrize("prec,n", [(2, 12), (2, 20), (1, 16), (2, 9), (2, 5)])
def test_pass_tables_address_every_slot_once(lib, prec, n):
    """The kernel's shared-memory slots for (thread, register) pairs, taken from
    the per-pass tables, cover the tile exactly once, agree with the swizzle
    of the raw tile index, and give conflict-free quarter-warps where the
    lane mapping allows it."""
    ops = random_ops(W.rng_for(300 + n), n, 40)
    steps, blob = build_plan(lib, ops, n, prec=prec)
    sw = 4 if prec == 1 else 3
    for kind, off, _ in steps:
        if kind != 1:
            continue
        h = np.frombuffer(blob, HDR, 1, off)[0]
        m = int(h["m"])
        nthreads = 1 << (m - 3)
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        for p in passes:
            slots, raws = [], []
            for tid in range(nthreads):
                sg = int(p["slo"][tid & 31]) ^ int(p["shi"][tid >> 5])
                rg = int(p["rlo"][tid & 31]) | int(p["rhi"][tid >> 5])
                for r in range(8):
                    sl, rw = sg, rg
                    for j in range(3):
                        if (r >> j) & 1:
                            sl ^= int(p["sp"][j])
                            rw |= int(p["pm"][j])
                    assert swizzle_map(rw, h["bankv"]) == sl
                    if int(h["mode"]) == 0:  # scalar sweeps: the kernels' fixed swizzle
                        assert swizzle(rw, sw) == sl
                    slots.append(sl)
                    raws.append(rw)
            assert sorted(slots) == list(range(1 << m))
            assert sorted(raws) == list(range(1 << m))


def warp_slots(p, m, w):
    """Raw tile indices the threads of warp `w` address in pass `p`."""
    nthreads = 1 << (m - 3)
    out = set()
    for tid in range(32 * w, min(32 * (w + 1), nthreads)):
        rg = int(p["rlo"][tid & 31]) | int(p["rhi"][tid >> 5])
        for r in range(8):
            rw = rg
            for j in range(3):
                if (r >> j) & 1:
                    rw |= int(p["pm"][j])
            out.add(rw)
    return out


@pytest.mark.parametrize("prec,n,tile_bits", [(2, 14, None), (1, 16, None), (2, 12, 8),
                                              (2, 16, 12), (2, 10, 7)])
def test_warp_phases_stay_inside_warps(lib, prec, n, tile_bits):
    """A pass flagged for a warp barrier only (DK_PASS_WARP) must leave every
    warp on the same tile slots in the next pass; the last pass of a sweep
    always ends with a block barrier, and tiles narrower than a warp never
    use the flag."""
    ops = random_ops(W.rng_for(500 + n), n, 60)
    ops += W.scale_circuit(seed=3, n=n, depth=3).ops
    steps, blob = build_plan(lib, ops, n, prec=prec, tile_bits=tile_bits)
    flagged = 0
    for kind, off, _ in steps:
        if kind != 1:
            continue
        h = np.frombuffer(blob, HDR, 1, off)[0]
        m = int(h["m"])
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        assert not int(passes[-1]["flags"]) & 2
        for i in range(len(passes) - 1):
            if not int(passes[i]["flags"]) & 2:
                continue
            assert m >= 8
            flagged += 1
            for w in range(max(1, (1 << (m - 3)) // 32)):
                assert warp_slots(passes[i], m, w) == warp_slots(passes[i + 1], m, w)
    if (tile_bits or 11) >= 8:
        assert flagged > 0
    else:
        assert flagged == 0


def test_scale_circuit_phases_cut_block_barriers(lib):
    """On the 30-qubit workload most passes end with a warp barrier only."""
    c = W.scale_circuit(seed=2, n=30, depth=8)
    steps, blob = build_plan(lib, c.ops, 30)
    npass = nwarp = 0
    for kind, off, _ in steps:
        h = np.frombuffer(blob, HDR, 1, off)[0]
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        npass += len(passes)
        nwarp += sum(1 for p in passes if int(p["flags"]) & 2)
    assert nwarp >= npass // 3, (nwarp, npass)


def test_tensor_variants_fold_out_of_tile_conditions(lib, orc):
    """Tensor sweeps fold gates whose controls lie outside the tile into the
    pass matrix, one product per combination of the run's tile conditions;
    the replay of those variant entries equals gate-by-gate application."""
    n = 15
    rng = W.rng_for(77)
    ops = []
    for layer in range(4):
        for q in range(n):
            ops.append(W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q]))
        for q in range(layer % 2, n - 1, 2):
            ops.append(W.Op(W.X.copy(), [q], {q + 1}))
        # far controls / anticontrols on low targets
        for q in range(3):
            ops.append(W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q], {n - 1 - q}, {n - 4 - q}))
    psi0 = np.zeros(1 << n, dtype=np.complex128)
    psi0[0] = 1
    got, steps = run_plan(lib, ops, n, psi0)
    want = oracle_run(orc, ops, n)
    assert np.allclose(got / np.linalg.norm(got), want / np.linalg.norm(want), atol=1e-12)
    _, blob = build_plan(lib, ops, n)
    nvar = 0
    for kind, off, _ in steps:
        if kind != 1:
            continue
        h = np.frombuffer(blob, HDR, 1, off)[0]
        assert int(h["mode"]) == 1
        g = np.frombuffer(blob, GATE, int(h["ngate"]), off + int(h["gate_off"]))
        nvar += int((g["code"] == 45).sum())
    assert nvar > 0


def thread_bits(p, m):
    """Tile bit carried by each thread-index bit of a pass (from rlo / rhi)."""
    out = []
    for j in range(m - 3):
        raw = int(p["rlo"][1 << j]) if j < 5 else int(p["rhi"][1 << (j - 5)])
        out.append(raw.bit_length() - 1)
    return out


def pass_bits(p):
    return [int(p["pm"][j]).bit_length() - 1 for j in range(3)]


@pytest.mark.parametrize("prec,n", [(2, 30), (1, 30), (2, 16)])
def test_chained_pairs_keep_the_mma_layout(lib, prec, n):
    """A pass flagged DK_PASS_CHAIN and the next one each hold one entry, the
    first pass's thread bits 0-2 (c0 c1 c2) are the second pass's bits in the
    order (c1 c2 c0), the second pass's thread bits 0-2 are the first pass's
    bits in order, and both keep the remaining thread bits: the MMA output
    layout of the first is the input layout of the second."""
    c = W.scale_circuit(seed=2, n=n, depth=12)
    steps, blob = build_plan(lib, c.ops, n, prec=prec)
    chained = total = 0
    for kind, off, _ in steps:
        h = np.frombuffer(blob, HDR, 1, off)[0]
        m = int(h["m"])
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        total += len(passes)
        for i, p in enumerate(passes):
            if not int(p["flags"]) & 4:
                continue
            chained += 1
            q = passes[i + 1]
            assert int(p["g1"]) - int(p["g0"]) == 1 and int(q["g1"]) - int(q["g0"]) == 1
            assert int(p["flags"]) & 2  # same warp bits
            ta, tb = thread_bits(p, m), thread_bits(q, m)
            assert pass_bits(q) == [ta[1], ta[2], ta[0]]
            assert tb[:3] == pass_bits(p)
            assert ta[3:] == tb[3:]
    assert chained > 0 and chained * 2 <= total


def test_disjoint_neighbour_passes_chain(lib, orc):
    """Two neighbouring single-entry passes whose target bits are disjoint
    chain even when the phase's bits would otherwise fill the second pass with
    a bit of the first: U3 on qubits 4-6 form one pass and U3 on 7-8 the next;
    filling the second from the phase's five bits alone would take bit 6, so
    the planner widens the phase to six bits and fills it with another."""
    n = 12
    rng = W.rng_for(4242)
    ops = [W.Op(W.u3(*rng.uniform(0, 2 * np.pi, 3)), [q]) for q in (4, 5, 6, 7, 8)]
    steps, blob = build_plan(lib, ops, n)
    assert len(steps) == 1 and steps[0][0] == 1
    h = np.frombuffer(blob, HDR, 1, steps[0][1])[0]
    passes = np.frombuffer(blob, PASS, int(h["npass"]), steps[0][1] + int(h["pass_off"]))
    assert len(passes) == 2
    assert int(passes[0]["flags"]) & 4
    assert {4, 5, 6} == set(pass_bits(passes[0]))
    assert {7, 8} <= set(pass_bits(passes[1]))
    assert not set(pass_bits(passes[0])) & set(pass_bits(passes[1]))
    psi0 = np.zeros(1 << n, dtype=np.complex128)
    psi0[0] = 1
    got, _ = run_plan(lib, ops, n, psi0)
    want = oracle_run(orc, ops, n)
    assert np.allclose(got, want, atol=1e-12)


def test_scale_circuit_chains_most_passes(lib):
    """On the 30-qubit depth-40 workload more than half of the tensor passes
    run as chained pairs (the remaining ones hold several entries, overlap
    their neighbour, or are the odd pass of a sweep)."""
    c = W.scale_circuit(seed=2, n=30, depth=40)
    steps, blob = build_plan(lib, c.ops, 30)
    chained = total = 0
    for kind, off, _ in steps:
        h = np.frombuffer(blob, HDR, 1, off)[0]
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        total += len(passes)
        chained += 2 * sum(1 for p in passes if int(p["flags"]) & 4)
    assert chained > total // 2, (chained, total)


def test_phases_keep_chainable_pairs_together(lib, orc):
    """A warp phase grows while its passes fit in m - wbits tile bits; when
    that would end it between two passes that can chain, the planner ends it
    one pass earlier (one more block barrier, one more chained pair).  On this
    12-qubit sweep of CZ and U3 gates both pass pairs chain."""
    n = 12
    rng = W.rng_for(31)

    def u3():
        return W.u3(*rng.uniform(0, 2 * np.pi, 3))

    ops = [W.Op(W.Z.copy(), [0], {5}), W.Op(W.Z.copy(), [2], {3}), W.Op(W.Z.copy(), [3], {4}),
           W.Op(u3(), [9]), W.Op(W.Z.copy(), [1], {3}), W.Op(u3(), [6]),
           W.Op(W.Z.copy(), [0], {2}), W.Op(u3(), [3]), W.Op(u3(), [6]), W.Op(u3(), [9]),
           W.Op(u3(), [11])]
    steps, blob = build_plan(lib, ops, n)
    assert len(steps) == 1 and steps[0][0] == 1
    h = np.frombuffer(blob, HDR, 1, steps[0][1])[0]
    passes = np.frombuffer(blob, PASS, int(h["npass"]), steps[0][1] + int(h["pass_off"]))
    assert sum(2 for p in passes if int(p["flags"]) & 4) == 4
    psi0 = W.rng_for(5).normal(size=1 << n) + 1j * W.rng_for(6).normal(size=1 << n)
    got, _ = run_plan(lib, ops, n, psi0)
    reg = orc.registry_new_data(n, psi0)
    want = orc.registry_get_all(W.run_ops(orc, reg, ops))
    assert np.allclose(got / np.linalg.norm(got), want, atol=1e-12)


def _pair_wavefronts(a, c, res):
    """Fewest shared-memory wavefronts of a chained pair's gather and scatter
    (per quarter-warp group) over the orders of its bit sets: the planner's
    own model (tile bit b lands in 16-byte bank group b % res under the XOR
    swizzle)."""
    import itertools

    def nres(b):
        return len({x % res for x in b})

    best = 99
    for pa in itertools.permutations(a):
        for pc in itertools.permutations(c):
            if res == 3:
                g, t = (pc[0], pa[0], pa[1]), (pc[1], pa[1], pa[2])
                v = (1 << (3 - nres(g))) + (1 << (3 - nres(t)))
            else:
                g, t = (pc[0], pc[1], pa[0], pa[1]), (pc[1], pc[2], pa[1], pa[2])
                v = (1 << (4 - nres(g))) + (1 << (4 - nres(t)))
            best = min(best, v)
    return best


@pytest.mark.parametrize("prec,res,bound", [(2, 3, 1.25), (1, 4, 1.3)])
def test_chained_pairs_fill_for_few_wavefronts(lib, prec, res, bound):
    """Chained pairs take their filler bits for the fewest shared-memory
    wavefronts: on the 30-qubit workload their total stays within `bound`
    of the conflict-free 2 per pair (filling by bit position alone gave 1.21
    for complex128 and 1.34 for complex64)."""
    c = W.scale_circuit(seed=2, n=30, depth=40)
    steps, blob = build_plan(lib, c.ops, 30, prec=prec)
    total = pairs = 0
    for kind, off, _ in steps:
        h = np.frombuffer(blob, HDR, 1, off)[0]
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        for i, p in enumerate(passes):
            if int(p["flags"]) & 4:
                total += _pair_wavefronts(sorted(pass_bits(p)), sorted(pass_bits(passes[i + 1])),
                                          res)
                pairs += 1
    assert pairs > 100
    assert total <= bound * 2 * pairs, (total, pairs)


def test_plan_unfused_keeps_controls_out_of_the_tile(lib):
    """One gate per sweep: the gate's controls and anticontrols stay outside
    the tile (tile conditions), so an in-place sweep moves only the tiles
    where they hold (2 S 2^-c bytes); the pinned low qubits stay in."""
    c = W.scale_circuit(seed=2, n=30, depth=2)
    steps, blob = build_plan(lib, c.ops, 30, fuse=0)
    assert len(steps) == len(c.ops)
    for (kind, off, _), op in zip(steps, c.ops):
        assert kind == 1
        h = np.frombuffer(blob, HDR, 1, off)[0]
        tile = set(int(q) for q in h["qpos"][:h["m"]])
        assert {0, 1} <= tile and set(op.targets) <= tile
        cond = (op.controls | op.anticontrols) - {0, 1}
        assert not (cond & tile), (op.targets, op.controls, op.anticontrols)
        assert bool(h["all_touched"]) == (not cond)


def _wavefronts(slots, groups):
    """Wavefronts of one quarter-warp (16-byte) / half-warp (8-byte) access:
    the most distinct slots that share a bank group."""
    by = {}
    for sl in set(slots):
        by.setdefault(sl % groups, set()).add(sl)
    return max(len(v) for v in by.values())


@pytest.mark.parametrize("prec,mode", [(2, 0), (1, 0), (1, 1)])
def test_bank_map_makes_sweeps_conflict_free(lib, prec, mode):
    """Each tensor sweep carries a bank map chosen for the accesses of the
    kernel that runs it (mode 0: the mma.sync lane layout; mode 1: whole
    columns per thread, the tcgen05 complex64 kernel).  On the 30-qubit
    workload, the slot tables under that map leave no shared-memory bank
    conflict in those accesses (the fixed XOR swizzle left 10.7 %, 13 % and
    96 % extra wavefronts)."""
    c = W.scale_circuit(seed=2, n=30, depth=40)
    steps, blob = build_plan(lib, c.ops, 30, prec=prec, bank_mode=mode)
    sw = 3 if prec == 2 else 4
    groups = 1 << sw
    total = ideal = 0
    for kind, off, _ in steps:
        h = np.frombuffer(blob, HDR, 1, off)[0]
        passes = np.frombuffer(blob, PASS, int(h["npass"]), off + int(h["pass_off"]))
        i = 0
        while i < len(passes):
            p = passes[i]
            chained = mode == 0 and int(p["flags"]) & 4
            q = passes[i + 1] if chained else p
            nent = 1 if chained else max(1, int(p["g1"]) - int(p["g0"]))
            if mode == 1:
                lanes = [int(p["slo"][x]) for x in range(groups)]
                total += 16 * nent * _wavefronts(lanes, groups)
                ideal += 16 * nent
            else:
                nl = groups // 2 if sw == 3 else groups // 4  # lanes per pass-bit combination
                gat, sca = [], []
                for lane in range(groups):
                    gl, gk = lane >> 2, lane & 3
                    gat.append(int(p["slo"][gl]) ^ (int(p["sp"][0]) if gk & 1 else 0) ^
                               (int(p["sp"][1]) if gk & 2 else 0))
                    sr = (int(q["sp"][0]) if gl & 1 else 0) ^ (int(q["sp"][1]) if gl & 2 else 0)
                    sca.append(int(q["slo"][2 * gk]) ^ sr)
                del nl
                total += 2 * nent * (_wavefronts(gat, groups) + _wavefronts(sca, groups))
                ideal += 4 * nent
            i += 2 if chained else 1
    assert total == ideal, (total / ideal)
