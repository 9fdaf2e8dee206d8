"""The debug build (libdokigpu_dbg.so, -DDK_DEBUG_CHECKS) on the GPU.

In that build the table-driven kernels -- both sweep kernels, the
joint-distribution passes and both collapses -- check every global and
shared-memory index they
compute; a failed check is recorded (site and index) and its access skipped,
without a trap.  Seeded circuits run through the debug library's C ABI
(tensor sweeps and, with DK_TENSOR=0, scalar sweeps; complex128 and
complex64; gates with controls inside and outside the tile; joint
measurement of 3, 4 and 6 qubits, and 13 qubits measured one at a time with
the single-qubit collapse kernel).  No check may fire, and the results must equal
the oracle's, as the release library's do.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from doki_b200 import workloads as W
from tests.conftest import ATOL_C128, ATOL_C64, ROOT

pytestmark = pytest.mark.gpu

LIB_DBG = os.path.join(ROOT, "doki_b200", "libdokigpu_dbg.so")

CHILD = textwrap.dedent("""
    import ctypes, json, sys
    import numpy as np
    sys.path.insert(0, sys.argv[3])
    from doki_b200 import workloads as W
    from tests.test_gpu_debug_checks import cases

    P = ctypes.c_void_p
    lib = ctypes.CDLL(sys.argv[1])
    lib.dk_init.argtypes = [ctypes.c_int]
    lib.dk_gate_new.argtypes = [ctypes.c_uint, P, ctypes.POINTER(P)]
    lib.dk_gate_free.argtypes = [P]
    lib.dk_state_new.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.POINTER(P)]
    lib.dk_state_free.argtypes = [P]
    lib.dk_apply_gate.argtypes = [P, P, P, ctypes.c_uint, P, ctypes.c_uint, P, ctypes.c_uint,
                                  ctypes.POINTER(P)]
    lib.dk_get_amplitudes.argtypes = [P, ctypes.c_uint64, ctypes.c_uint64, P]
    lib.dk_marginals.argtypes = [P, P]
    lib.dk_measure_mask.argtypes = [P, ctypes.c_uint64, P, ctypes.c_uint, P, ctypes.POINTER(P)]
    lib.dk_measure.argtypes = [P, ctypes.c_uint, ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(P)]
    lib.dk_debug_checks.argtypes = [ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]

    def ok(rc):
        assert rc == 0, rc

    def u32(xs):
        a = (ctypes.c_uint * max(1, len(xs)))(*xs)
        return ctypes.cast(a, P), a

    def amps(s, n):
        out = np.empty(2 << n)
        ok(lib.dk_get_amplitudes(s, 0, 1 << n, out.ctypes.data))
        return out.view(np.complex128)

    ok(lib.dk_init(0))
    first = ctypes.c_uint64(1)
    ok(lib.dk_debug_checks(ctypes.byref(first), 1))
    res = {}
    for name, (c, prec, mask, rolls, target, roll) in cases().items():
        n = c.num_qubits
        s = P()
        ok(lib.dk_state_new(n, prec, ctypes.byref(s)))
        for op in c.ops:
            m = np.ascontiguousarray(op.gate, dtype=np.complex128)
            g = P()
            ok(lib.dk_gate_new(op.k, m.ctypes.data, ctypes.byref(g)))
            t, keep_t = u32(list(op.targets))
            cc, keep_c = u32(sorted(op.controls))
            aa, keep_a = u32(sorted(op.anticontrols))
            o = P()
            ok(lib.dk_apply_gate(s, g, t, len(op.targets), cc, len(op.controls), aa,
                                 len(op.anticontrols), ctypes.byref(o)))
            lib.dk_state_free(s)
            lib.dk_gate_free(g)
            s = o
        r = {"amps": amps(s, n)}
        marg = np.empty(n)
        ok(lib.dk_marginals(s, marg.ctypes.data))
        r["marg"] = marg
        rl = np.ascontiguousarray(rolls, dtype=np.float64)
        results = np.zeros(n, dtype=np.int8)
        o = P()
        ok(lib.dk_measure_mask(s, mask, rl.ctypes.data, len(rl), results.ctypes.data,
                               ctypes.byref(o)))
        r["mask_results"] = results
        r["mask_amps"] = amps(o, n - bin(mask).count("1"))
        lib.dk_state_free(o)
        bit = ctypes.c_int(-1)
        o = P()
        ok(lib.dk_measure(s, target, roll, ctypes.byref(bit), ctypes.byref(o)))
        r["one_result"] = np.array([bit.value])
        r["one_amps"] = amps(o, n - 1)
        lib.dk_state_free(o)
        lib.dk_state_free(s)
        for k, v in r.items():
            res[name + ":" + k] = v
    ok(lib.dk_sync())
    ok(lib.dk_debug_checks(ctypes.byref(first), 0))
    res["check"] = np.array([first.value], dtype=np.uint64)
    np.savez(sys.argv[2], **res)
""")


def cases():
    """name -> (circuit, precision, measure mask, rolls, single target, roll)."""
    small = W.small_circuit(seed=11, n=12, depth=6)
    wide = W.scale_circuit(seed=5, n=18, depth=5, ctrl_frac=0.3)
    return {
        "small_c128": (small, 2, 0b100000010011, [0.31, 0.77, 0.52, 0.08], 5, 0.4),
        # 13 measured qubits: more than one joint pass takes, so the
        # qubit-by-qubit path with the single-qubit collapse kernel runs
        "wide_c128": (wide, 2, (1 << 13) - 1, [0.66, 0.21, 0.45, 0.93, 0.12, 0.58, 0.37,
                                              0.81, 0.04, 0.49, 0.71, 0.26, 0.55], 13, 0.7),
        "wide_c64": (wide, 1, (1 << 17) | (1 << 9) | 1, [0.66, 0.21, 0.45], 13, 0.7),
        # 6 measured qubits: the joint pass that gathers each outcome's
        # amplitudes through the deposit tables (more than 4 bins)
        "wide6_c128": (wide, 2, 0b10100100010010010, [0.5, 0.15, 0.85, 0.35, 0.62, 0.27], 3,
                       0.2),
    }


def run_child(tmp_path, tensor):
    if not os.path.exists(LIB_DBG):
        raise AssertionError("debug library missing: run the build first")
    out = tmp_path / f"dbg_{tensor}.npz"
    env = dict(os.environ, DK_TENSOR=str(tensor))
    r = subprocess.run([sys.executable, "-c", CHILD, LIB_DBG, str(out), ROOT], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


def oracle_results(orc, c, mask, rolls, target, roll):
    reg = W.run_ops(orc, orc.registry_new(c.num_qubits), c.ops)
    want = {"amps": orc.registry_get_all(reg), "marg": np.array(orc.registry_probs(reg))}
    r1, res = orc.registry_measure(reg, mask, rolls)
    want["mask_results"] = np.array([-1 if v is None else int(v) for v in res], dtype=np.int8)
    want["mask_amps"] = orc.registry_get_all(r1)
    n = c.num_qubits
    r2, res2 = orc.registry_measure(reg, 1 << target, [roll])
    want["one_result"] = np.array([int(res2[n - 1 - target])])
    want["one_amps"] = orc.registry_get_all(r2)
    return want


@pytest.mark.parametrize("tensor", [1, 0])
def test_debug_build_checks_stay_clear(dk_gpu, orc, tmp_path, tensor):
    got = run_child(tmp_path, tensor)
    assert int(got["check"][0]) == 0, json.dumps(
        {"site": int(got["check"][0]) >> 56, "index": int(got["check"][0]) & ((1 << 56) - 1)})
    for name, (c, prec, mask, rolls, target, roll) in cases().items():
        want = oracle_results(orc, c, mask, rolls, target, roll)
        atol = ATOL_C128 if prec == 2 else ATOL_C64
        for key in ("amps", "marg", "mask_amps", "one_amps"):
            assert np.allclose(got[name + ":" + key], want[key], atol=atol, rtol=0), (name, key)
        assert np.array_equal(got[name + ":mask_results"], want["mask_results"]), name
        assert got[name + ":one_result"][0] == want["one_result"][0], name


STARVE = textwrap.dedent("""
    import ctypes, sys
    import numpy as np
    sys.path.insert(0, sys.argv[2])
    from doki_b200 import workloads as W

    P = ctypes.c_void_p
    lib = ctypes.CDLL(sys.argv[1])
    lib.dk_init.argtypes = [ctypes.c_int]
    lib.dk_gate_new.argtypes = [ctypes.c_uint, P, ctypes.POINTER(P)]
    lib.dk_gate_free.argtypes = [P]
    lib.dk_state_new.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.POINTER(P)]
    lib.dk_state_free.argtypes = [P]
    lib.dk_apply_gate.argtypes = [P, P, P, ctypes.c_uint, P, ctypes.c_uint, P, ctypes.c_uint,
                                  ctypes.POINTER(P)]
    lib.dk_marginals.argtypes = [P, P]
    lib.dk_debug_tm_starve.argtypes = [ctypes.c_int]

    def run(n):
        s = P()
        assert lib.dk_state_new(n, 1, ctypes.byref(s)) == 0
        for q in range(n):
            m = np.ascontiguousarray(W.u3(0.3 + q, 0.2, 0.1), dtype=np.complex128)
            g = P()
            assert lib.dk_gate_new(1, m.ctypes.data, ctypes.byref(g)) == 0
            t = (ctypes.c_uint * 1)(q)
            o = P()
            assert lib.dk_apply_gate(s, g, ctypes.cast(t, P), 1, None, 0, None, 0,
                                     ctypes.byref(o)) == 0
            lib.dk_state_free(s)
            lib.dk_gate_free(g)
            s = o
        marg = np.empty(n)
        rc = lib.dk_marginals(s, marg.ctypes.data)
        lib.dk_state_free(s)
        return rc, marg

    assert lib.dk_init(0) == 0
    assert lib.dk_debug_tm_starve(1) == 0
    rc, _ = run(16)
    print("starved", rc)
    assert lib.dk_debug_tm_starve(0) == 0
    rc2, marg = run(16)
    print("after", rc2)
    want = [abs(np.sin((0.3 + q) / 2)) ** 2 for q in range(16)]
    assert rc2 == 0 and np.allclose(marg, want, atol=1e-6), (rc2, marg)
    sys.exit(0 if rc == 23 else 3)
""")


def test_tensor_memory_sweep_wait_expires_cleanly(dk_gpu):
    """Failure detection of the complex64 tcgen05 sweep: with its MMA
    completions starved (a flag that nothing sets, debug build), each bounded
    wait expires, the kernel frees its tensor memory and returns, and the
    read that follows reports DK_ERR_TIMEOUT (23).  The context stays
    usable: the same circuit run right after is correct."""
    r = subprocess.run([sys.executable, "-c", STARVE, LIB_DBG, ROOT],
                       env=dict(os.environ, DK_TENSOR="1", DK_C64_TMEM="1"),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-3000:])
    assert "starved 23" in r.stdout and "after 0" in r.stdout
