#!/usr/bin/env python
"""Benchmark of the plain complex128 state-vector path at 30 qubits.

Workload (one step): a 30-qubit complex128 register (16 GiB) starts in
|0..0>; a seeded depth-40 random circuit is applied (per layer U3 on all 30
qubits with angles ~ U[0, 2pi), then a CZ/CNOT brickwork; 5 % of the gates get
1-3 extra random controls / anticontrols; 1780 gates); then all 30 single-qubit
probabilities, measurement with collapse of 4 random qubits (30 -> 26 qubits)
and the reduced density matrix of qubits 0-9 (1024 x 1024, copied to the host).

metric: gate-layers per second (40 per step), whole job over all GPUs.
  value -- device time (CUDA events on the engine's stream) from the first
           queued sweep to the last result, gates already queued;
  e2e   -- host wall time of the same job through the public `doki` API,
           gate matrices created from host memory and every result read back.
--gpus N runs N independent replicas (the path does not shard at this size).
--impl reference times the reference Doki CPU module (compiled from source
into oracle/_ref) on the host cores, one workload gate per step.
The line also carries `per_gate`: the same register with fusion off (one
sweep per gate, the plain per-gate method) against the HBM roofline.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q gate-layers/s"
UNIT = "gate-layers/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--qubits", type=int, default=30)
    p.add_argument("--depth", type=int, default=40)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fusion", action="store_true",
                   help="one sweep per gate (the per-gate plain method)")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the batching / serving / precision forms")
    p.add_argument("--serve-requests", type=int, default=400,
                   help="requests of the seeded 20,000-request stream the serving form "
                        "runs (a prefix of it)")
    p.add_argument("--serve-plain", type=int, default=600,
                   help="requests the plain path runs (a prefix); its throughput on the "
                        "served sample is scaled from their times by qubit count")
    p.add_argument("--serve-only", action="store_true",
                   help="run only the serving form and print its JSON object")
    p.add_argument("--form-only", choices=("batch", "serve", "precision"),
                   help="run only this form and print its JSON object")
    p.add_argument("--precision", choices=("c128", "c64"), default="c128",
                   help="register precision of the plain workload (c64: split-TF32 "
                        "tensor products, FP64 norms)")
    return p.parse_args()


def workload_config(n, depth, c, prec="c128"):
    amp = 16 if prec == "c128" else 8
    return {
        "workload": (f"{n}-qubit {'complex128' if prec == 'c128' else 'complex64'} register, "
                     f"seeded depth-{depth} random circuit "
                     "(U3 on all qubits + CZ/CNOT brickwork, 5% gates with 1-3 extra "
                     "controls/anticontrols), all marginals, measure+collapse of 4 qubits, "
                     "reduced density matrix of qubits 0-9"),
        "qubits": n, "depth": depth, "gates": len(c.ops),
        "state_bytes": amp << n,
        "l2": (f"inputs larger than L2 (state {(amp << n) / 2**30:g} GiB vs 126 MB L2)"
               if (amp << n) > 126e6 else
               f"state {(amp << n) / 2**20:g} MiB fits in the 126 MB L2 (not flushed)"),
        "parallelism": "replicas",
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the sweep kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "sweep_c128_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


# ------------------------------------------------------------------ engine --

def max_over_ranks(values, world, device):
    """Element-wise maximum of per-rank timings over all ranks (every rank
    receives it); replicas are timed by their slowest member."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.tolist()


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units in `seconds` (the max over ranks)."""
    return world * units_per_rank / seconds


def run_job(d, c, gates, keep, rolls_mask, rolls, prec="c128", reg=None):
    """The workload's gates queued through the public API on a new |0..0>
    register (or on `reg`); returns the register (gates not yet flushed)."""
    n = c.num_qubits
    if reg is None:
        reg = d.registry_new(n, False) if prec == "c128" else d.registry_new(n, False, 1)
    for op, g in zip(c.ops, gates):
        ctl = set(op.controls) if (op.controls or op.anticontrols) else None
        reg = d.registry_apply(reg, g, list(op.targets), ctl, set(op.anticontrols) or None,
                               -1, False)
    return reg


def finish_job(d, reg, n, keep, mask, rolls):
    probs = [d.registry_prob(reg, q, -1, False) for q in range(n)]
    sub, res = d.registry_measure(reg, mask, rolls, -1, False)
    rho = d.registry_density(reg, False)
    for e in range(n - 1, keep - 1, -1):
        rho = d.funmatrix_partialtrace(rho, e, False)
    mat = d.funmatrix_numpy(rho)
    return probs, res, mat


def library_gemm_tflops(torch, c64, n=8192, reps=5):
    """Throughput of the library GEMM of the sweep's arithmetic, timed here
    with CUDA events: cuBLAS DGEMM (complex128 sweeps) or cuBLAS TF32 SGEMM
    (complex64), n x n x n, after one warm-up."""
    dt = torch.float32 if c64 else torch.float64
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = bool(c64)
    try:
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        torch.matmul(a, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return 2.0 * n ** 3 * reps / (ms / 1e3) / 1e12


def tensor_roofline(entry_amps, sweep_s, c64, clk, steps, lib_tflops=None, tcgen05=False):
    """Tensor-pipe work of the timed sweeps.  One matrix entry applied to one
    amplitude is 24 FP64 MMA FMA (complex128: three real m8n8k4 products of
    two k-steps per 64 amplitudes) or 96 TF32 MMA FMA (complex64: three
    TF32 products per 8x16 by 16x16 real block).  The peak is the measured
    library GEMM of the same arithmetic (cuBLAS DGEMM / TF32 SGEMM on this
    GPU) when given; for FP64 the MMA op rate ncu reports
    (sm__ops_path_tensor_src_fp64: 128 per SM per cycle) x SMs x the median SM
    clock of the run is given beside it."""
    import torch
    fma = entry_amps * (96 if c64 else 24)
    achieved = 2.0 * fma / max(sweep_s, 1e-12) / 1e12
    pipe = ("tf32 tcgen05.mma (M=128, N=32/16)" if tcgen05 else "tf32 mma.sync m16n8k8") \
        if c64 else "fp64 mma.sync m8n8k4"
    out = {"pipe": pipe, "achieved": achieved, "unit": "TFLOP/s",
           "flops_per_step": 2.0 * fma / steps}
    if lib_tflops:
        out.update({"peak": lib_tflops, "frac": achieved / lib_tflops,
                    "peak_kind": "measured cuBLAS " + ("TF32 SGEMM" if c64 else "DGEMM")
                                 + " 8192^3 on this GPU"})
    if not c64:
        mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        nominal = 128.0 * sms * mhz * 1e6 / 1e12
        out.update({"peak_op_rate": nominal, "frac_op_rate": achieved / nominal,
                    "peak_op_rate_kind": f"ncu FP64 MMA op rate 128/SM/cycle x {sms} SMs x "
                                         f"{mhz:g} MHz"})
        if not lib_tflops:
            out.update({"peak": nominal, "frac": achieved / nominal,
                        "peak_kind": out["peak_op_rate_kind"]})
    return out


def per_gate_record(d, c, prec, torch, stream, layers=2):
    """The plain per-gate method on the benchmark register: fusion off, so
    every gate of the first `layers` layers is its own in-place sweep over
    the whole register (the reference's one loop per apply_gate,
    qops.c:211-257).  Algorithmic bytes per gate: 2 S 2^-c for c controls
    and anticontrols (amplitudes whose conditions fail need not move);
    achieved = their sum / the sweeps' device time."""
    n = c.num_qubits
    layers = min(layers, c.depth)
    ops = c.ops[:c.layer_starts[layers]] if layers < c.depth else c.ops
    state_bytes = (8 if prec == "c64" else 16) << n
    gates = [d.gate_new(op.k, op.gate.tolist(), False) for op in ops]
    reg = d.registry_new(n, False) if prec == "c128" else d.registry_new(n, False, 1)
    d.registry_flush(reg)
    d.engine_set_fusion(False)
    try:
        reg = run_job(d, W_ops(c, ops), gates, 0, 0, [], prec, reg=reg)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0 = d.engine_stats()["sweeps"]
        e0.record(stream)
        d.registry_flush(reg)
        e1.record(stream)
        e1.synchronize()
        sweeps = d.engine_stats()["sweeps"] - s0
    finally:
        d.engine_set_fusion(True)
    del reg
    ms = e0.elapsed_time(e1)
    algo = sum(2 * state_bytes >> (len(op.controls) + len(op.anticontrols)) for op in ops)
    peak, peak_kind = measured_peak_hbm()
    achieved = algo / (ms / 1e3) / 1e9
    return {"gates": len(ops), "layers": layers, "sweeps": sweeps, "device_ms": ms,
            "avg_sweep_ms": ms / max(1, sweeps),
            "kernel": "one in-place fused-sweep launch per gate (fusion off)",
            "algorithmic_bytes": algo, "achieved": achieved, "unit": "GB/s", "peak": peak,
            "peak_kind": peak_kind + " hbm_gbs (copy)", "frac": achieved / peak,
            "gate_layers_per_s": layers / (ms / 1e3)}


class W_ops:
    """A circuit restricted to a list of its ops (for run_job)."""

    def __init__(self, c, ops):
        self.num_qubits = c.num_qubits
        self.ops = ops


def engine_arm(args, rank, world, local_rank):
    import numpy as np
    import torch

    if world > 1:
        os.environ["DK_DEVICE"] = str(local_rank)
    torch.cuda.set_device(local_rank)
    if world > 1:
        torch.distributed.init_process_group(
            "nccl", timeout=datetime.timedelta(seconds=300),
            device_id=torch.device("cuda", local_rank))

    import doki_b200
    from doki_b200 import workloads as W

    d = doki_b200.load()
    if args.no_fusion:
        d.engine_set_fusion(False)
    n, depth, keep = args.qubits, args.depth, min(10, args.qubits)
    c = W.scale_circuit(seed=2, n=n, depth=depth, keep=keep)
    mask, rolls = c.measure_mask, c.rolls.tolist()
    gates = [d.gate_new(op.k, op.gate.tolist(), False) for op in c.ops]

    # warm-up (also creates the engine stream)
    for _ in range(args.warmup):
        reg = run_job(d, c, gates, keep, mask, rolls, args.precision)
        finish_job(d, reg, n, keep, mask, rolls)
        del reg
    d.engine_sync()
    stream = torch.cuda.ExternalStream(d.engine_stream(), device=torch.device("cuda", local_rank))

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---- device-timed value --------------------------------------------
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    st0 = d.engine_stats()
    dev_ms, sweep_ms, nsweeps = 0.0, 0.0, 0
    for _ in range(args.steps):
        reg = run_job(d, c, gates, keep, mask, rolls, args.precision)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        s_before = d.engine_stats()["sweeps"]
        d.registry_flush(reg)
        e1.record(stream)
        nsweeps += d.engine_stats()["sweeps"] - s_before
        finish_job(d, reg, n, keep, mask, rolls)
        e2.record(stream)
        e2.synchronize()
        dev_ms += e0.elapsed_time(e2)
        sweep_ms += e0.elapsed_time(e1)
        del reg
    d.engine_sync()
    torch.cuda.synchronize()
    st1 = d.engine_stats()
    clk = clocks.stop()
    barrier()

    # ---- end-to-end through the public API -------------------------------
    e2e_s = 0.0
    io0 = d.engine_stats()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        g2 = [d.gate_new(op.k, op.gate.tolist(), False) for op in c.ops]
        reg = run_job(d, c, g2, keep, mask, rolls, args.precision)
        probs, res, mat = finish_job(d, reg, n, keep, mask, rolls)
        e2e_s += time.perf_counter() - t0
        del reg, g2
    io1 = d.engine_stats()
    barrier()

    dev_ms, e2e_s, sweep_ms = max_over_ranks([dev_ms, e2e_s, sweep_ms], world, "cuda")

    layers = depth * args.steps
    value = job_rate(world, layers, dev_ms / 1e3)
    e2e_value = job_rate(world, layers, e2e_s)
    c64 = args.precision == "c64"
    tcgen05 = c64 and os.environ.get("DK_C64_TMEM", "1") != "0"
    lib_tflops = library_gemm_tflops(torch, c64) if rank == 0 and world == 1 else None
    state_bytes = (8 if c64 else 16) << n
    avg_sweep_s = (sweep_ms / 1e3) / max(1, nsweeps)
    achieved = 2 * state_bytes / avg_sweep_s / 1e9
    peak, peak_kind = measured_peak_hbm()
    tr = committed_traffic()
    traffic = None
    if tr and tr.get("qubits") and not c64:
        traffic = float(tr["bytes_per_launch"]) * (state_bytes / (16 << int(tr["qubits"])))

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if c64 else "f64", "data": "synthetic",
        "config": workload_config(n, depth, c, args.precision),
        "roofline": {"bound": "hbm",
                     "kernel": ("k_sweep_tm (fused gate sweep, split-TF32 tcgen05 products "
                                "in tensor memory)" if tcgen05 else
                                "k_sweep_tc<float> (fused gate sweep, split-TF32 tensor-core "
                                "passes)" if c64 else
                                "k_sweep_tc<double> (fused gate sweep, FP64 tensor-core passes)"),
                     "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind + " hbm_gbs (copy)", "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": 2 * state_bytes,
                     "avg_launch_ms": avg_sweep_s * 1e3,
                     "sweeps_per_step": nsweeps / args.steps,
                     "gates_per_step": len(c.ops)},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": (io1["h2d_bytes"] - io0["h2d_bytes"]) // args.steps,
                "d2h_bytes_per_step": (io1["d2h_bytes"] - io0["d2h_bytes"]) // args.steps},
        "tensor_roofline": tensor_roofline(st1["mma_entry_amplitudes"] -
                                           st0["mma_entry_amplitudes"],
                                           sweep_ms / 1e3, c64, clk, args.steps,
                                           lib_tflops, tcgen05),
        "gpu_launches": st1["kernel_launches"] - st0["kernel_launches"],
        "clocks": clk,
        "fusion": not args.no_fusion,
    }
    if rank == 0 and world == 1:
        out["per_gate"] = per_gate_record(d, c, args.precision, torch, stream)
    if rank == 0 and world == 1 and not args.no_forms:
        out["forms"] = run_forms(d, args, torch)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(n, c)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


# ------------------------------------------------------------------- forms --

def plain_circuits_per_s(d, fb, per_size=2):
    """The plain method (one circuit at a time through the doki API,
    complex128) on a stratified sample of the batch, weighted to the mix."""
    import numpy as np
    from doki_b200 import workloads as W
    times = {}
    for n in range(4, 17):
        sel = [int(c) for c in np.nonzero(fb.num_qubits == n)[0][:per_size + 1]]
        if not sel:
            continue
        # one untimed circuit of each size first (first launches of the
        # size's kernels), then the timed ones
        W.run_ops(d, d.registry_new(n, False), fb.ops(sel[0]))
        d.engine_sync()
        for c in sel[1:] or sel:
            t0 = time.perf_counter()
            reg = W.run_ops(d, d.registry_new(n, False), fb.ops(c))
            rho = d.registry_density(reg, False)
            for e in range(n - 1, int(fb.keep[c]) - 1, -1):
                rho = d.funmatrix_partialtrace(rho, e, False)
            d.funmatrix_numpy(rho)
            times.setdefault(n, []).append(time.perf_counter() - t0)
    hist = np.bincount(fb.num_qubits, minlength=17)
    total = sum(hist[n] * statistics.mean(v) for n, v in times.items())
    return fb.count / total


def batch_form(d, torch):
    import numpy as np
    from doki_b200 import batch as B
    from doki_b200 import workloads as W
    fb = W.batch_arrays(seed=4, count=4096)
    dev = torch.cuda.get_device_name()
    res = {"workload": "4096 registers, n ~ U[4,16], depth ~ U[10,50], U3 + CNOT + "
                       "controlled-U3, reduced density matrix of the lower half",
           "gates": int(fb.op_k.size)}
    engines = {}
    host_rho = None  # page-locked, reused by both precisions
    for prec, name in ((1, "c64"), (2, "c128")):
        tune = B.autotune(fb, prec, tile_bits=(11, 12), ctas=(1, 2), folds=(-1, 0, 400),
                          reps=2, device_name=dev)
        t0 = time.perf_counter()
        eng = B.BatchEngine(fb, prec, tile_bits=tune["tile_bits"], fold=tune["fold"],
                            ctas_per_sm=tune["ctas_per_sm"])
        build_s = time.perf_counter() - t0
        eng.run()
        eng.sync()
        st = torch.cuda.ExternalStream(eng.stream)
        ms = []
        for _ in range(5):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            eng.run()
            b.record(st)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        if host_rho is None:
            host_rho = torch.empty(2 * eng.rho_elems, dtype=torch.float64,
                                   pin_memory=True).numpy().view(np.complex128)
        t0 = time.perf_counter()
        eng.run(keep_states=True)
        rho, _ = eng.rho_all(out=host_rho)
        out_s = time.perf_counter() - t0
        engines[name] = eng
        res[name] = {"circuits_per_s": fb.count / (statistics.median(ms) / 1e3),
                     "batch_ms_p50": float(np.percentile(ms, 50)),
                     "batch_ms_p99": float(np.percentile(ms, 99)),
                     "plan_and_upload_s": build_s,
                     "e2e_circuits_per_s": fb.count / (build_s + out_s),
                     "e2e_parts_s": {"plan_and_upload": build_s,
                                     "run_and_copy_rho": out_s, **eng.build_times()},
                     "rho_host_buffer": "page-locked, allocated once and reused",
                     "rho_bytes": int(rho.nbytes), "tile_bits": tune["tile_bits"],
                     "fold": tune["fold"], "ctas_per_sm": tune["ctas_per_sm"],
                     "autotune_cached": tune["cached"],
                     "autotune_objective": "host planning + one device run",
                     "autotune_trials": [{k: t[k] for k in ("fold", "tile_bits", "ctas_per_sm")}
                                         | {"ms": t["seconds"] * 1e3,
                                            "plan_ms": t["plan_s"] * 1e3}
                                         for t in tune["trials"]]}
    fid, err = engines["c64"].compare(engines["c128"])
    # the same figures on the host for a sample of the registers (every
    # 64th), from downloaded states: an independent check of the device
    # comparison
    hf, he = [], []
    for c in range(0, fb.count, 64):
        x, y = engines["c64"].state(c), engines["c128"].state(c)
        hf.append(abs(np.vdot(x, y)) ** 2 / (np.vdot(x, x).real * np.vdot(y, y).real))
        he.append(float(np.max(np.abs(x / np.linalg.norm(x) - y / np.linalg.norm(y)))))
    res["c64"].update({"min_fidelity": float(fid.min()), "max_amp_err": float(err.max()),
                       "fidelity_vs": "the complex128 batch of the same 4096 circuits",
                       "host_check": {"registers": len(hf), "min_fidelity": float(min(hf)),
                                      "max_amp_err": float(max(he)),
                                      "device_min_fidelity_same_registers":
                                          float(fid[::64].min())}})
    for eng in engines.values():
        eng.close()
    plain = plain_circuits_per_s(d, fb)
    res["plain_gpu_circuits_per_s"] = plain
    res["speedup_c64_vs_plain"] = res["c64"]["circuits_per_s"] / plain
    res["e2e_speedup_c64_vs_plain"] = res["c64"]["e2e_circuits_per_s"] / plain
    return res


def plain_rate(per_n_seconds, hist):
    """Throughput of the one-at-a-time plain path on a request mix with qubit
    histogram `hist`, from measured seconds per request grouped by qubit
    count (additive: requests run one after another)."""
    total = 0.0
    for n, cnt in hist.items():
        times = per_n_seconds.get(n)
        if not times:  # no sample of this size: its nearest measured size
            near = min(per_n_seconds, key=lambda m: abs(m - n))
            times = per_n_seconds[near]
        total += cnt * statistics.mean(times)
    return sum(hist.values()) / total


def serve_form(d, count, plain_count=600):
    import numpy as np
    from doki_b200 import serve as S
    stream = S.request_stream(seed=5, count=20000)
    reqs = stream[:count]
    S.prepare(reqs)
    sample = (f"the first {count} requests of the seeded 20,000-request stream "
              "(n log-uniform [8,28], depth U[10,100], probabilities or 1-8 measurements); "
              "circuits prepared as data before the runs")
    srv = S.Server(d, workers=8, budget_bytes=150e9, precision=1, deadline_s=3600)
    cap = srv.run(S.with_rate(reqs, 1e9))
    out = {"sample": sample, "workers": 8, "budget_bytes": 150e9, "precision": "c64",
           "submission": "one registry_apply_many call per request",
           "capacity_rps": cap["throughput_rps"], "loads": {}}
    for load in (0.5, 0.8, 1.0):
        r = srv.run(S.with_rate(reqs, load * cap["throughput_rps"]))
        out["loads"][f"{int(load * 100)}%"] = {k: r[k] for k in
                                              ("throughput_rps", "p50_ms", "p99_ms")}
    ns = np.array([r.n for r in reqs])
    hist = {int(n): int((ns == n).sum()) for n in np.unique(ns)}
    pc = min(plain_count, count)
    plain = {}
    for prec, name in ((2, "c128"), (1, "c64")):
        p = S.run_plain(d, reqs[:pc], precision=prec, deadline_s=3600)
        per_n = {}
        for r, t in zip(reqs[:pc], p["seconds"]):
            per_n.setdefault(r.n, []).append(t)
        plain[name] = {"measured_rps": p["throughput_rps"],
                       "rps": p["throughput_rps"] if pc == count else plain_rate(per_n, hist),
                       "mean_ms_by_qubits": {int(k): round(1e3 * statistics.mean(v), 3)
                                             for k, v in sorted(per_n.items())}}
    out["plain"] = {"path": "one request at a time, one registry_apply call per gate",
                    "measured_on": f"the first {pc} requests"
                                   + ("" if pc == count else
                                      f", scaled to the {count}-request sample by qubit count"),
                    "c128_rps": plain["c128"]["rps"], "c64_rps": plain["c64"]["rps"],
                    "c128_measured_rps": plain["c128"]["measured_rps"],
                    "c64_measured_rps": plain["c64"]["measured_rps"],
                    "c128_mean_ms_by_qubits": plain["c128"]["mean_ms_by_qubits"],
                    "c64_mean_ms_by_qubits": plain["c64"]["mean_ms_by_qubits"]}
    out["speedup_vs_plain_c128"] = cap["throughput_rps"] / plain["c128"]["rps"]
    out["speedup_vs_plain_c64"] = cap["throughput_rps"] / plain["c64"]["rps"]
    out["qubits_histogram"] = hist
    return out


def precision_form(d):
    from doki_b200 import precision as P
    r = P.run(d, n=32, depth=60, seed=1)
    return {"workload": "32-qubit register, complex64 (32 GiB) beside complex128 (64 GiB), "
                        "depth-60 circuit of the 12-qubit generator family",
            "worst": r["worst"],
            "c64_layers_per_s_flushed_each_layer": r["c64_layers_per_s_flushed_each_layer"],
            "c128_layers_per_s_flushed_each_layer": r["c128_layers_per_s_flushed_each_layer"],
            "c64_layers_per_s_fused": r["c64_layers_per_s_fused"],
            "c128_layers_per_s_fused": r["c128_layers_per_s_fused"],
            "fused_final": r["fused_final"],
            "fidelity_per_layer": [round(x["fidelity"], 12) for x in r["layers"]]}


def run_forms(d, args, torch):
    forms = {}
    for name, fn in (("batch", lambda: batch_form(d, torch)),
                     ("serve", lambda: serve_form(d, args.serve_requests, args.serve_plain)),
                     ("precision", lambda: precision_form(d))):
        try:
            forms[name] = fn()
        except Exception as e:  # noqa: BLE001 -- report, keep the headline line
            forms[name] = {"error": f"{type(e).__name__}: {e}"}
        d.engine_set_slot(0)
    return forms


# --------------------------------------------------------------- reference --

def layer_ops(c, layer=0):
    return c.ops[c.layer_starts[layer]:c.layer_starts[layer + 1]]


def gate_kind(op):
    """"cond": a gate the generator gave extra controls / anticontrols;
    "pair": a brickwork CZ / CNOT (one control); "u3": an uncontrolled U3."""
    if op.anticontrols or len(op.controls) > 1:
        return "cond"
    if op.controls:
        return "pair" if abs(op.gate[0, 0]) in (0.0, 1.0) else "cond"
    return "u3"


def stratified_order(ops):
    """Indices of a layer's gates in an order whose every prefix mixes the
    kinds: the conditioned gates first, then pairs and U3s alternating."""
    by = {"cond": [], "pair": [], "u3": []}
    for i, op in enumerate(ops):
        by[gate_kind(op)].append(i)
    order = list(by["cond"])
    pairs, u3s = by["pair"], by["u3"]
    for j in range(max(len(pairs), len(u3s))):
        order += pairs[j:j + 1] + u3s[j:j + 1]
    return order


def ref_apply(ref, reg, op, threads):
    g = ref.gate_new(op.k, op.gate.tolist(), False)
    ctl = set(op.controls) if (op.controls or op.anticontrols) else None
    return ref.registry_apply(reg, g, list(op.targets), ctl, set(op.anticontrols) or None,
                              threads, False)


def reference_layer(n, c, threads):
    """One full layer of the workload through the reference module (all its
    gates in order, conditioned ones included), then registry_prob of one
    qubit and a one-qubit registry_measure (clone + probability + collapse,
    doki.c:1023-1192), each timed around the Python call as the reference's
    tests/timed_test.py:11-44 does."""
    from oracle import oracle as O
    ref = O.reference_module()
    ops = layer_ops(c)
    reg = ref.registry_new(n, False)
    t0 = time.perf_counter()
    for op in ops:
        reg = ref_apply(ref, reg, op, threads)
    t_layer = time.perf_counter() - t0
    q = max(q for q in range(n) if (c.measure_mask >> q) & 1)
    t0 = time.perf_counter()
    ref.registry_prob(reg, q, threads, False)
    t_prob = time.perf_counter() - t0
    t0 = time.perf_counter()
    sub, _ = ref.registry_measure(reg, 1 << q, [float(c.rolls[0])], threads, False)
    t_meas = time.perf_counter() - t0
    del sub, reg
    return {"gates": len(ops), "layer_s": t_layer, "prob_s": t_prob, "measure1_s": t_meas}


def reference_one_gate(n, c, threads):
    """One U3 of the workload on the reference module with `threads` threads."""
    from oracle import oracle as O
    ref = O.reference_module()
    op = next(op for op in layer_ops(c) if gate_kind(op) == "u3")
    reg = ref.registry_new(n, False)
    t0 = time.perf_counter()
    new = ref_apply(ref, reg, op, threads)
    dt = time.perf_counter() - t0
    del new, reg
    return dt


def cpu_baseline(n, c):
    """The reference CPU path on the box's host cores: one measured full
    layer of the 30-qubit workload at all threads (plus one probability and
    one single-qubit measurement), and one U3 at a single thread.  The job's
    layers/s is depth / (depth x layer + n x prob + 4 x one-qubit measure);
    the 30 -> 10-qubit reduced density matrix, which the reference's lazy
    functional matrices cannot evaluate in any useful time
    (funmatrix.c:920-944: 2^20 recursive leaves per element), is left out."""
    threads = os.cpu_count() or 1
    try:
        lay = reference_layer(n, c, threads)
        one = reference_one_gate(n, c, 1)
    except MemoryError:
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": "host memory too small for the reference at this size"}
    nmeas = bin(c.measure_mask).count("1")
    job_s = c.depth * lay["layer_s"] + n * lay["prob_s"] + nmeas * lay["measure1_s"]
    return {"value": c.depth / job_s, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": (f"reference doki module (compiled from its sources, OpenMP, {threads} "
                       f"threads) on the {n}-qubit register: layer 0 of the workload measured "
                       f"whole ({lay['gates']} gates incl. the conditioned ones) in "
                       f"{lay['layer_s']:.1f} s, registry_prob {lay['prob_s']:.2f} s, 1-qubit "
                       f"registry_measure {lay['measure1_s']:.2f} s; job = {c.depth} layers + "
                       f"{n} probabilities + {nmeas} one-qubit measurements"),
            "layer": lay, "one_thread": {"cores": 1, "u3_gate_s": one,
                                         "gate_layers_per_s_est":
                                             1.0 / (one * len(layer_ops(c)))}}


def reference_arm(args, rank, world):
    """The reference's own CPU implementation of the path on the host cores,
    one workload gate per step.  The steps walk the 30-qubit workload's first
    layer in an order that mixes its gate kinds from the start (conditioned
    gates, then CZ / CNOT pairs and U3s alternating); layers/s is estimated
    per kind: 1 / sum over kinds of (gates of that kind per layer x mean
    measured seconds per gate of that kind)."""
    if rank != 0:
        return
    from doki_b200 import workloads as W
    from oracle import oracle as O
    n, depth = args.qubits, args.depth
    c = W.scale_circuit(seed=2, n=n, depth=depth, keep=min(10, n))
    if not O.have_reference():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference module not built (oracle/_ref)"}))
        return
    ref = O.reference_module()
    threads = os.cpu_count() or 1
    ops = layer_ops(c)
    order = stratified_order(ops)
    L = len(order)
    reg = ref.registry_new(n, False)
    for j in range(args.warmup):
        reg = ref_apply(ref, reg, ops[order[(L - args.warmup + j) % L]], threads)
    times = {"cond": [], "pair": [], "u3": []}
    all_t = []
    for k in range(args.steps):
        op = ops[order[k % L]]
        t0 = time.perf_counter()
        new = ref_apply(ref, reg, op, threads)
        dt = time.perf_counter() - t0
        reg = new
        times[gate_kind(op)].append(dt)
        all_t.append(dt)
    del reg
    mean_all = statistics.mean(all_t)
    counts = {kd: sum(1 for op in ops if gate_kind(op) == kd) for kd in times}
    layer_s = sum(counts[kd] * (statistics.mean(v) if v else mean_all)
                  for kd, v in times.items())
    per_layer = len(c.ops) / c.depth
    layer_s *= per_layer / len(ops)  # layers of the workload average per_layer gates
    value = 1.0 / layer_s
    sample = (f"one gate per step on {n} qubits, walking layer 0's {len(ops)} gates "
              f"({counts['cond']} conditioned, {counts['pair']} CZ/CNOT, {counts['u3']} U3) "
              f"in a kind-mixing order; layers/s = 1 / sum over kinds of gates per layer x "
              f"mean measured s/gate ({ {k: len(v) for k, v in times.items()} } samples)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mean_all * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, depth, c),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def form_only(args, name):
    """One form alone (e.g. the serving form over the whole request
    stream)."""
    import torch

    import doki_b200
    d = doki_b200.load()
    fn = {"batch": lambda: batch_form(d, torch),
          "serve": lambda: serve_form(d, args.serve_requests, args.serve_plain),
          "precision": lambda: precision_form(d)}[name]
    t0 = time.perf_counter()
    out = fn()
    out["wall_s"] = time.perf_counter() - t0
    print(json.dumps({"form": name, **out}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.serve_only or args.form_only:
        form_only(args, "serve" if args.serve_only else args.form_only)
        return
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        engine_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
