"""Batching form: many independent registers in one CUDA-graph launch.

:class:`BatchEngine` wraps the ``dk_batch_*`` C ABI (``include/dokigpu.h``):
circuits in the flat layout of :class:`doki_b200.workloads.FlatBatch` are
planned on the host (the same fusion planner as the plain path), uploaded
once, and every run queues one graph that executes all registers and leaves
each register's reduced density matrix on the device.

:func:`autotune` is the project's tuner: it times the batch under each
candidate (dense-block fusion of the plan, tile bits of the streamed
registers, CTAs per SM) and caches the best choice in a JSON file keyed by
device, precision and size histogram.
"""
from __future__ import annotations

import ctypes
import json
import os
import time
from typing import Dict, Iterable, List, Optional, Tuple

import numpy as np

from .workloads import FlatBatch

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u32p = ctypes.POINTER(ctypes.c_uint)
_dp = ctypes.POINTER(ctypes.c_double)


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(os.path.join(_HERE, "libdokigpu.so"))
        L.dk_batch_build.argtypes = [ctypes.c_int, ctypes.c_uint, _u32p, _u32p, _u64p, _u32p,
                                     _u32p, _u64p, _u64p, _u64p, _dp, ctypes.c_int,
                                     ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.dk_batch_build.restype = ctypes.c_int
        L.dk_batch_set_ctas.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.dk_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.dk_batch_sync.argtypes = [ctypes.c_void_p]
        L.dk_batch_stream.argtypes = [ctypes.c_void_p]
        L.dk_batch_stream.restype = ctypes.c_void_p
        L.dk_batch_rho.argtypes = [ctypes.c_void_p, ctypes.c_uint, _dp]
        L.dk_batch_rho_all.argtypes = [ctypes.c_void_p, _dp, _u64p]
        L.dk_batch_rho_elems.argtypes = [ctypes.c_void_p]
        L.dk_batch_rho_elems.restype = ctypes.c_uint64
        L.dk_batch_state.argtypes = [ctypes.c_void_p, ctypes.c_uint, _dp]
        L.dk_batch_compare.argtypes = [ctypes.c_void_p, ctypes.c_void_p, _dp, _dp]
        L.dk_batch_build_times.argtypes = [ctypes.c_void_p, _dp, _dp, _dp]
        L.dk_batch_error.argtypes = [ctypes.c_void_p]
        L.dk_batch_error.restype = ctypes.c_char_p
        L.dk_batch_free.argtypes = [ctypes.c_void_p]
        L.dk_strerror.argtypes = [ctypes.c_int]
        L.dk_strerror.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class BatchError(RuntimeError):
    pass


class BatchEngine:
    """A planned, device-resident batch of circuits."""

    def __init__(self, batch: FlatBatch, precision: int = 1, tile_bits: int = 12,
                 ctas_per_sm: int = 1, fold: int = 0):
        L = lib()
        self.batch = batch
        self.precision = precision
        nq = np.ascontiguousarray(batch.num_qubits, dtype=np.uint32)
        keep = np.ascontiguousarray(batch.keep, dtype=np.uint32)
        st = np.ascontiguousarray(batch.op_start, dtype=np.uint64)
        k = np.ascontiguousarray(batch.op_k, dtype=np.uint32)
        tg = np.ascontiguousarray(batch.op_targets, dtype=np.uint32)
        cm = np.ascontiguousarray(batch.op_controls, dtype=np.uint64)
        am = np.ascontiguousarray(batch.op_anticontrols, dtype=np.uint64)
        mi = np.ascontiguousarray(batch.op_matrix, dtype=np.uint64)
        mats = np.ascontiguousarray(batch.matrices, dtype=np.complex128)
        h = ctypes.c_void_p()
        rc = L.dk_batch_build(precision, batch.count, _ptr(nq, _u32p), _ptr(keep, _u32p),
                              _ptr(st, _u64p), _ptr(k, _u32p), _ptr(tg, _u32p),
                              _ptr(cm, _u64p), _ptr(am, _u64p), _ptr(mi, _u64p),
                              _ptr(mats.view(np.float64), _dp), tile_bits, fold,
                              ctypes.byref(h))
        if rc:
            raise BatchError(f"dk_batch_build: {L.dk_strerror(rc).decode()}")
        self._h = h
        self.tile_bits = tile_bits
        self.fold = fold
        if ctas_per_sm != 1:
            self.set_ctas(ctas_per_sm)
        self.ctas_per_sm = ctas_per_sm
        self.rho_elems = int(L.dk_batch_rho_elems(h))

    def _check(self, rc: int, what: str):
        if rc:
            L = lib()
            raise BatchError(f"{what}: {L.dk_strerror(rc).decode()} "
                             f"({L.dk_batch_error(self._h).decode()})")

    def build_times(self) -> Dict[str, float]:
        """Host seconds of the build: planning, blob assembly, device
        allocation and upload."""
        v = [ctypes.c_double(), ctypes.c_double(), ctypes.c_double()]
        self._check(lib().dk_batch_build_times(self._h, *[ctypes.byref(x) for x in v]),
                    "dk_batch_build_times")
        return {"plan_s": v[0].value, "assemble_s": v[1].value, "upload_s": v[2].value}

    def set_ctas(self, ctas_per_sm: int):
        self._check(lib().dk_batch_set_ctas(self._h, ctas_per_sm), "dk_batch_set_ctas")
        self.ctas_per_sm = ctas_per_sm

    def run(self, keep_states: bool = False):
        self._check(lib().dk_batch_run(self._h, int(keep_states)), "dk_batch_run")

    def sync(self):
        self._check(lib().dk_batch_sync(self._h), "dk_batch_sync")

    @property
    def stream(self) -> int:
        return int(lib().dk_batch_stream(self._h) or 0)

    def rho(self, c: int) -> np.ndarray:
        k = int(self.batch.keep[c])
        out = np.empty((1 << k, 1 << k), dtype=np.complex128)
        self._check(lib().dk_batch_rho(self._h, c, _ptr(out.view(np.float64), _dp)),
                    "dk_batch_rho")
        return out

    def rho_all(self, out: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
        """Every register's reduced density matrix, concatenated, and their
        offsets.  `out` (complex128, at least rho_elems long; e.g. a view of
        a reused page-locked buffer) receives them when given."""
        if out is None:
            out = np.empty(self.rho_elems, dtype=np.complex128)
        elif out.dtype != np.complex128 or out.size < self.rho_elems or \
                not out.flags.c_contiguous:
            raise BatchError("rho_all: out must be contiguous complex128 of rho_elems")
        offs = np.empty(self.batch.count, dtype=np.uint64)
        self._check(lib().dk_batch_rho_all(self._h, _ptr(out.view(np.float64), _dp),
                                           _ptr(offs, _u64p)), "dk_batch_rho_all")
        return out, offs

    def state(self, c: int) -> np.ndarray:
        out = np.empty(1 << int(self.batch.num_qubits[c]), dtype=np.complex128)
        self._check(lib().dk_batch_state(self._h, c, _ptr(out.view(np.float64), _dp)),
                    "dk_batch_state")
        return out

    def compare(self, other: "BatchEngine") -> Tuple[np.ndarray, np.ndarray]:
        """Per-circuit fidelity and largest amplitude difference of this
        batch's final registers against `other`'s (same circuits; both run
        with keep_states), computed on the device in FP64."""
        fid = np.empty(self.batch.count)
        err = np.empty(self.batch.count)
        self._check(lib().dk_batch_compare(self._h, other._h, _ptr(fid, _dp), _ptr(err, _dp)),
                    "dk_batch_compare")
        return fid, err

    def close(self):
        if getattr(self, "_h", None):
            lib().dk_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def time_runs(eng: BatchEngine, reps: int = 3) -> float:
    """Mean seconds per run (device-synchronised, after one warm-up)."""
    eng.run()
    eng.sync()
    t0 = time.perf_counter()
    for _ in range(reps):
        eng.run()
    eng.sync()
    return (time.perf_counter() - t0) / reps


def _signature(batch: FlatBatch, precision: int) -> str:
    hist = np.bincount(batch.num_qubits, minlength=17)[4:17]
    ops = int(batch.op_k.size)
    return f"p{precision}-n{batch.count}-ops{ops}-h" + ".".join(str(int(x)) for x in hist)


def default_cache_path() -> str:
    return os.environ.get("DK_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "doki_b200",
                                       "autotune.json"))


def pick_trial(trials: List[Dict]) -> Tuple[Dict, float]:
    """The autotuner's choice among timed trials ({fold, tile_bits,
    ctas_per_sm, plan_s, seconds}): planning work depends on the fold, not
    on the tile width or CTAs per SM, so each trial is charged its fold's
    fastest measured planning (timing noise in planning cannot pick a slower
    kernel configuration) plus its device run; sets each trial's
    `objective_s` and returns the best trial and its fold's planning time."""
    fold_plan: Dict[int, float] = {}
    for t in trials:
        fold_plan[t["fold"]] = min(fold_plan.get(t["fold"], t["plan_s"]), t["plan_s"])
    for t in trials:
        t["objective_s"] = fold_plan[t["fold"]] + t["seconds"]
    best = min(trials, key=lambda t: t["objective_s"])
    return best, fold_plan[best["fold"]]


def autotune(batch: FlatBatch, precision: int, tile_bits: Iterable[int] = (10, 11, 12),
             ctas: Iterable[int] = (1, 2), folds: Iterable[int] = (-1, 0, 400), reps: int = 2,
             cache_path: Optional[str] = None, device_name: str = "") -> Dict:
    """Pick the dense-block fusion of the plan (`fold`: -1 every gate on its
    own, 0 the planner's default, larger values fold runs of gates into 8x8
    products more readily), tile bits (streamed registers) and CTAs per SM
    by timing the batch under every combination.  A batch is planned once
    and run once, so the objective is the host planning and upload time of
    the fold (the fastest of its builds) plus one device run; results, with
    every trial, are cached per (device, precision, batch signature)."""
    path = cache_path or default_cache_path()
    key = f"{device_name}|{_signature(batch, precision)}"
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        cache = {}
    if key in cache and cache[key].get("objective") == "plan+run":
        return dict(cache[key], cached=True)
    trials = []
    for fold in folds:
        for tb in tile_bits:
            t0 = time.perf_counter()
            eng = BatchEngine(batch, precision, tile_bits=tb, fold=fold)
            plan_s = time.perf_counter() - t0
            for c in ctas:
                eng.set_ctas(c)
                run_s = time_runs(eng, reps)
                trials.append({"fold": fold, "tile_bits": tb, "ctas_per_sm": c,
                               "plan_s": plan_s, "seconds": run_s})
            eng.close()
    best, plan = pick_trial(trials)
    result = {"fold": best["fold"], "tile_bits": best["tile_bits"],
              "ctas_per_sm": best["ctas_per_sm"], "seconds": best["seconds"],
              "plan_s": plan, "objective": "plan+run", "trials": trials}
    cache[key] = result
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    except OSError:
        pass
    return dict(result, cached=False)
