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
    p.add_argument("--serve-requests", type=int, default=120)
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


def run_job(d, c, gates, keep, rolls_mask, rolls, prec="c128"):
    """One full workload through the public API; returns the host results."""
    n = c.num_qubits
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


def tensor_roofline(entry_amps, sweep_s, c64, clk, steps):
    """Tensor-pipe work of the timed sweeps.  One matrix entry applied to one
    amplitude is 24 FP64 MMA FMA (complex128: three real m8n8k4 products of
    two k-steps per 64 amplitudes) or 96 TF32 MMA FMA (complex64: six m16n8k8
    MMAs per 64 amplitudes).  The FP64 peak is the MMA op rate ncu reports
    (sm__ops_path_tensor_src_fp64: 128 per SM per cycle) x SMs x the median SM
    clock of the run; no TF32 figure is measured, so complex64 has none."""
    import torch
    fma = entry_amps * (96 if c64 else 24)
    achieved = 2.0 * fma / max(sweep_s, 1e-12) / 1e12
    out = {"pipe": "tf32 mma.sync m16n8k8" if c64 else "fp64 mma.sync m8n8k4",
           "achieved": achieved, "unit": "TFLOP/s", "flops_per_step": 2.0 * fma / steps}
    if not c64:
        mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        peak = 128.0 * sms * mhz * 1e6 / 1e12
        out.update({"peak": peak, "frac": achieved / peak,
                    "peak_kind": f"ncu FP64 MMA op rate 128/SM/cycle x {sms} SMs x {mhz:g} MHz"})
    return out


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
                     "kernel": ("k_sweep_tc<float> (fused gate sweep, split-TF32 tensor-core "
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
                                           sweep_ms / 1e3, c64, clk, args.steps),
        "gpu_launches": st1["kernel_launches"] - st0["kernel_launches"],
        "clocks": clk,
        "fusion": not args.no_fusion,
    }
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
    warm = fb.ops(0)
    W.run_ops(d, d.registry_new(int(fb.num_qubits[0]), False), warm)
    for n in range(4, 17):
        idx = [int(c) for c in np.nonzero(fb.num_qubits == n)[0][:per_size]]
        for c in idx:
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
    for prec, name in ((1, "c64"), (2, "c128")):
        tune = B.autotune(fb, prec, tile_bits=(11, 12), ctas=(1,), reps=2, device_name=dev)
        t0 = time.perf_counter()
        eng = B.BatchEngine(fb, prec, tile_bits=tune["tile_bits"])
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
        t0 = time.perf_counter()
        eng.run()
        rho, _ = eng.rho_all()
        out_s = time.perf_counter() - t0
        eng.close()
        res[name] = {"circuits_per_s": fb.count / (statistics.median(ms) / 1e3),
                     "batch_ms_p50": float(np.percentile(ms, 50)),
                     "batch_ms_p99": float(np.percentile(ms, 99)),
                     "plan_and_upload_s": build_s,
                     "e2e_circuits_per_s": fb.count / (build_s + out_s),
                     "rho_bytes": int(rho.nbytes), "tile_bits": tune["tile_bits"],
                     "autotune_cached": tune["cached"]}
    plain = plain_circuits_per_s(d, fb)
    res["plain_gpu_circuits_per_s"] = plain
    res["speedup_c64_vs_plain"] = res["c64"]["circuits_per_s"] / plain
    return res


def serve_form(d, count):
    from doki_b200 import serve as S
    reqs = S.request_stream(seed=5, count=count)
    sample = (f"first {count} requests of the seeded 20,000-request stream "
              "(n log-uniform [8,28], depth U[10,100], probabilities or 1-8 measurements)")
    srv = S.Server(d, workers=8, budget_bytes=150e9, precision=1, deadline_s=240)
    cap = srv.run(S.with_rate(reqs, 1e9))
    out = {"sample": sample, "workers": 8, "budget_bytes": 150e9, "precision": "c64",
           "capacity_rps": cap["throughput_rps"], "loads": {}}
    for load in (0.5, 0.8, 1.0):
        r = srv.run(S.with_rate(reqs, load * cap["throughput_rps"]))
        out["loads"][f"{int(load * 100)}%"] = {k: r[k] for k in
                                              ("throughput_rps", "p50_ms", "p99_ms")}
    plain = S.Server(d, workers=1, budget_bytes=150e9, precision=2, deadline_s=400)
    p = plain.run(S.with_rate(reqs, 1e9))
    out["plain_gpu_rps"] = p["throughput_rps"]
    out["speedup_vs_plain"] = cap["throughput_rps"] / p["throughput_rps"]
    return out


def precision_form(d):
    from doki_b200 import precision as P
    r = P.run(d, n=32, depth=60, seed=1)
    return {"workload": "32-qubit register, complex64 (32 GiB) beside complex128 (64 GiB), "
                        "depth-60 circuit of the 12-qubit generator family",
            "worst": r["worst"], "c64_layers_per_s": r["c64_layers_per_s"],
            "c128_layers_per_s": r["c128_layers_per_s"],
            "fidelity_per_layer": [round(x["fidelity"], 12) for x in r["layers"]]}


def run_forms(d, args, torch):
    forms = {}
    for name, fn in (("batch", lambda: batch_form(d, torch)),
                     ("serve", lambda: serve_form(d, args.serve_requests)),
                     ("precision", lambda: precision_form(d))):
        try:
            forms[name] = fn()
        except Exception as e:  # noqa: BLE001 -- report, keep the headline line
            forms[name] = {"error": f"{type(e).__name__}: {e}"}
        d.engine_set_slot(0)
    return forms


# --------------------------------------------------------------- reference --

def sample_ops(c):
    """Gates of the first layer, spread over low / high qubits and 2-qubit ops."""
    layer = c.ops[c.layer_starts[0]:c.layer_starts[1]]
    idx = [0, len(layer) // 2 - 1, len(layer) - 1, 7, len(layer) // 2 + 3, 15]
    return [layer[i % len(layer)] for i in idx]


def reference_timings(n, c, count, warm=0):
    from oracle import oracle as O
    from doki_b200 import workloads as W
    ref = O.reference_module()
    threads = os.cpu_count() or 1
    ops = sample_ops(c)
    reg = ref.registry_new(n, False)
    times = []
    for i in range(warm + count):
        op = ops[i % len(ops)]
        g = ref.gate_new(op.k, op.gate.tolist(), False)
        ctl = set(op.controls) if (op.controls or op.anticontrols) else None
        t0 = time.perf_counter()
        new = ref.registry_apply(reg, g, list(op.targets), ctl,
                                 set(op.anticontrols) or None, threads, False)
        dt = time.perf_counter() - t0
        del reg
        reg = new
        if i >= warm:
            times.append(dt)
    del reg
    return times, threads


def cpu_baseline(n, c):
    gates_per_layer = len(c.ops) / c.depth
    try:
        times, threads = reference_timings(n, c, 4)
        qn = n
    except MemoryError:
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": "host memory too small for the reference at this size"}
    per_gate = statistics.mean(times)
    return {"value": 1.0 / (per_gate * gates_per_layer), "unit": UNIT, "cores": threads,
            "kind": "reference",
            "sample": (f"reference doki registry_apply (OpenMP, {threads} threads) on {qn} "
                       f"qubits: {len(times)} gates from layer 0 (low/high U3, CNOT/CZ), "
                       f"mean {per_gate:.3f} s/gate x {gates_per_layer:.1f} gates/layer")}


def reference_arm(args, rank, world):
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
    times, threads = reference_timings(n, c, args.steps, warm=args.warmup)
    gates_per_layer = len(c.ops) / c.depth
    per_gate = statistics.mean(times)
    value = 1.0 / (per_gate * gates_per_layer)
    sample = (f"one workload gate per step on {n} qubits (layer-0 U3 low/high, CNOT/CZ), "
              f"layers/s = 1 / (mean s/gate x {gates_per_layer:.1f} gates/layer)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_gate * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, depth, c),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
    else:
        engine_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
