"""CPU oracle for the Doki state-vector path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use
this module, and only as the checker / CPU baseline; the product path
(``doki_b200``) never imports it.

Two checkers live here:

* :class:`OracleDoki` -- a doki-shaped API (same function names and argument
  order as the reference module, reference ``src/doki/doki.c:114-192``) backed by
  ``libdkoracle.so``, the C restatement in ``dk_oracle.c``.  Registry-level
  sequencing (measure loop order, roll consumption, lazy norm) is restated
  here from ``src/doki/doki.c:1023-1192`` and ``src/doki/qstate.c:90-105``.
* :func:`reference_module` -- the reference extension itself, compiled from its
  sources into ``oracle/_ref/`` by ``oracle/Makefile``.

The restatement is pinned against the reference module and against the golden
fixtures in ``tests/golden/`` by ``tests/test_oracle.py``.
"""
from __future__ import annotations

import ctypes
import glob
import importlib.machinery
import importlib.util
import os
from typing import Iterable, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint)
_ip = ctypes.POINTER(ctypes.c_int)


def lib() -> ctypes.CDLL:
    """Load ``_build/libdkoracle.so`` (built by ``make -C oracle``)."""
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "libdkoracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.dko_apply_gate.argtypes = [_dp, ctypes.c_double, ctypes.c_uint, _dp,
                                     ctypes.c_uint, _up, ctypes.c_uint64,
                                     ctypes.c_uint64, _dp, _dp]
        L.dko_apply_gate.restype = ctypes.c_int
        L.dko_probability.argtypes = [_dp, ctypes.c_double, ctypes.c_uint,
                                      ctypes.c_uint]
        L.dko_probability.restype = ctypes.c_double
        L.dko_collapse.argtypes = [_dp, ctypes.c_double, ctypes.c_uint,
                                   ctypes.c_uint, ctypes.c_int, ctypes.c_double,
                                   _dp, _dp]
        L.dko_collapse.restype = None
        L.dko_join.argtypes = [_dp, ctypes.c_double, ctypes.c_uint, _dp,
                               ctypes.c_double, ctypes.c_uint, _dp]
        L.dko_join.restype = None
        L.dko_global_phase.argtypes = [_dp, ctypes.c_double, ctypes.c_uint]
        L.dko_global_phase.restype = ctypes.c_double
        L.dko_ptrace_elem.argtypes = [_dp, ctypes.c_double, ctypes.c_uint, _ip,
                                      ctypes.c_uint, ctypes.c_uint64,
                                      ctypes.c_uint64, _dp, _dp]
        L.dko_ptrace_elem.restype = None
        L.dko_reduced_density.argtypes = [_dp, ctypes.c_double, ctypes.c_uint,
                                          ctypes.c_uint64, _dp]
        L.dko_reduced_density.restype = None
        L.dko_marginals.argtypes = [_dp, ctypes.c_double, ctypes.c_uint, _dp]
        L.dko_marginals.restype = None
        _LIB = L
    return _LIB


def reference_module():
    """Import the reference ``doki`` extension compiled into ``oracle/_ref/``.

    It is loaded under its own name (``doki``) without being placed in
    ``sys.modules`` so it never shadows the engine under test.
    """
    global _REF
    if _REF is None:
        cands = glob.glob(os.path.join(_HERE, "_ref", "doki*.so"))
        if not cands:
            raise FileNotFoundError("oracle/_ref/doki*.so missing: run "
                                    "`make -C oracle ref` where the reference "
                                    "sources are mounted")
        loader = importlib.machinery.ExtensionFileLoader("doki", cands[0])
        spec = importlib.util.spec_from_file_location("doki", cands[0],
                                                      loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _REF = mod
    return _REF


def have_reference() -> bool:
    return bool(glob.glob(os.path.join(_HERE, "_ref", "doki*.so")))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class OState:
    """Host register: interleaved complex128 raw amplitudes + norm constant
    (reference ``struct state_vector``, ``src/doki/qstate.h:44-59``)."""

    __slots__ = ("n", "amp", "norm", "phase")

    def __init__(self, n: int, amp: Optional[np.ndarray], norm: float = 1.0):
        self.n = n
        self.amp = amp  # complex128 array of 2^n, or None for 0 qubits
        self.norm = norm
        self.phase = None

    def vector(self) -> np.ndarray:
        """Logical amplitudes amp / norm (reference ``state_get``)."""
        return self.amp / self.norm


class OGate:
    __slots__ = ("k", "matrix")

    def __init__(self, k: int, matrix: np.ndarray):
        self.k = k
        self.matrix = np.ascontiguousarray(matrix, dtype=np.complex128)


class OFMatrix:
    """Density matrix / chained partial trace of a register (lazy)."""

    __slots__ = ("state", "elems")

    def __init__(self, state: OState, elems: tuple):
        self.state = state
        self.elems = elems

    @property
    def dim(self) -> int:
        return 1 << (self.state.n - len(self.elems))


class OracleDoki:
    """doki-shaped API over the C restatement (argument order as the reference
    module; ``num_threads`` / ``verbose`` accepted and ignored)."""

    error = ValueError

    # -- gates -----------------------------------------------------------
    def gate_new(self, k, matrix, verbose=False):
        m = np.array(matrix, dtype=np.complex128)
        if m.shape != (1 << k, 1 << k):
            raise ValueError("Wrong matrix size for specified number of qubits")
        return OGate(k, m)

    def gate_get(self, gate, verbose=False):
        return gate.matrix.tolist()

    # -- registers -------------------------------------------------------
    def registry_new(self, n, verbose=False):
        a = np.zeros(1 << n, dtype=np.complex128)
        a[0] = 1.0
        return OState(n, a, 1.0)

    def registry_new_data(self, n, values, verbose=False):
        a = np.ascontiguousarray(np.asarray(values, dtype=np.complex128).ravel())
        if a.size != (1 << n):
            raise ValueError("Wrong array size for the specified number of qubits")
        return OState(n, a.copy(), 1.0)

    def registry_clone(self, reg, num_threads=-1, verbose=False):
        # qstate.c:90-105 -- the clone stores normalised values, norm = 1
        return OState(reg.n, reg.vector().copy(), 1.0)

    def registry_del(self, reg, verbose=False):
        return None

    def registry_get(self, reg, idx, canonical=False, verbose=False):
        v = complex(reg.amp[idx] / reg.norm)
        if canonical:
            ph = self._phase(reg)
            v = v * complex(np.cos(ph), -np.sin(ph))
        return v

    def registry_get_all(self, reg, canonical=False):
        v = reg.vector()
        if canonical:
            ph = self._phase(reg)
            v = v * complex(np.cos(ph), -np.sin(ph))
        return v

    def _phase(self, reg):
        if reg.phase is None:
            a = np.ascontiguousarray(reg.amp)
            reg.phase = lib().dko_global_phase(_ptr(a.view(np.float64)),
                                               reg.norm, reg.n)
        return reg.phase

    def registry_apply(self, reg, gate, targets, controls, anticontrols,
                       num_threads=-1, verbose=False):
        k = gate.k
        if len(targets) != k:
            raise ValueError("Wrong number of targets specified for that gate")
        cm = 0
        for c in (controls or ()):
            cm |= 1 << c
        am = 0
        for c in (anticontrols or ()):
            am |= 1 << c
        t = (ctypes.c_uint * k)(*targets)
        out = np.empty(1 << reg.n, dtype=np.complex128)
        onorm = ctypes.c_double()
        lib().dko_apply_gate(_ptr(reg.amp.view(np.float64)), reg.norm, reg.n,
                             _ptr(gate.matrix.view(np.float64)), k, t, cm, am,
                             _ptr(out.view(np.float64)), ctypes.byref(onorm))
        return OState(reg.n, out, onorm.value)

    def registry_join(self, most, least, num_threads=-1, verbose=False):
        n = most.n + least.n
        out = np.empty(1 << n, dtype=np.complex128)
        lib().dko_join(_ptr(most.amp.view(np.float64)), most.norm, most.n,
                       _ptr(least.amp.view(np.float64)), least.norm, least.n,
                       _ptr(out.view(np.float64)))
        return OState(n, out, 1.0)

    def registry_prob(self, reg, q, num_threads=-1, verbose=False):
        return lib().dko_probability(_ptr(reg.amp.view(np.float64)), reg.norm,
                                     reg.n, q)

    def registry_probs(self, reg):
        p = np.empty(reg.n, dtype=np.float64)
        lib().dko_marginals(_ptr(reg.amp.view(np.float64)), reg.norm, reg.n,
                            _ptr(p))
        return p

    def registry_measure(self, reg, mask, rolls, num_threads=-1, verbose=False):
        """doki.c:1023-1192: clone, then qubits n-1 .. 0 in mask, one roll each;
        result[i] belongs to qubit n-1-i; returns (register or None, list).
        `last_margins` keeps |P(q=1) - roll| of each decision in measurement
        order, so a checker can tell a rounding-level near-tie from a real
        disagreement."""
        cur = self.registry_clone(reg)
        n0 = reg.n
        result = []
        self.last_margins = []
        rid = 0
        measured = 0
        for i in range(n0):
            q = n0 - i - 1
            val = None
            if mask & (1 << q):
                if cur is None or cur.n == 0:
                    raise ValueError("Could not measure non_existant qubits")
                roll = float(rolls[rid])
                if roll < 0 or roll >= 1:
                    raise ValueError("roll not in interval [0, 1)!")
                rid += 1
                p1 = self.registry_prob(cur, q)
                bit = p1 > roll
                self.last_margins.append(abs(p1 - roll))
                if cur.n == 1:
                    cur = OState(0, None, 0.0)
                else:
                    out = np.empty(1 << (cur.n - 1), dtype=np.complex128)
                    onorm = ctypes.c_double()
                    lib().dko_collapse(_ptr(cur.amp.view(np.float64)), cur.norm,
                                       cur.n, q, int(bit), p1,
                                       _ptr(out.view(np.float64)),
                                       ctypes.byref(onorm))
                    cur = OState(cur.n - 1, out, onorm.value)
                measured += 1
                val = bool(bit)
            result.append(val)
        if n0 - measured > 0:
            return cur, result
        return None, result

    # -- density matrices ------------------------------------------------
    def registry_density(self, reg, verbose=False):
        return OFMatrix(reg, ())

    def funmatrix_partialtrace(self, fm, elem, verbose=False):
        return OFMatrix(fm.state, fm.elems + (int(elem),))

    def funmatrix_shape(self, fm, verbose=False):
        return (fm.dim, fm.dim)

    def funmatrix_get(self, fm, i, j, verbose=False):
        el = (ctypes.c_int * max(1, len(fm.elems)))(*fm.elems)
        re, im = ctypes.c_double(), ctypes.c_double()
        lib().dko_ptrace_elem(_ptr(fm.state.amp.view(np.float64)), fm.state.norm,
                              fm.state.n, el, len(fm.elems), i, j,
                              ctypes.byref(re), ctypes.byref(im))
        return complex(re.value, im.value)

    def funmatrix_trace(self, fm, verbose=False):
        return sum(self.funmatrix_get(fm, i, i) for i in range(fm.dim))


def reduced_density(state: OState, keep_mask: int) -> np.ndarray:
    """Materialised reduced density matrix over the qubits in ``keep_mask``."""
    k = bin(keep_mask).count("1")
    out = np.empty((1 << k, 1 << k), dtype=np.complex128)
    lib().dko_reduced_density(_ptr(state.amp.view(np.float64)), state.norm,
                              state.n, keep_mask, _ptr(out.view(np.float64)))
    return out


def kept_mask_after_traces(n: int, elems: Iterable[int]) -> int:
    """Original-qubit mask that survives successive partial traces ``elems``
    (each id relative to the matrix it is applied to)."""
    alive = list(range(n))
    for e in elems:
        del alive[e]
    m = 0
    for q in alive:
        m |= 1 << q
    return m
