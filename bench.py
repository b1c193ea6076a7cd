#!/usr/bin/env python
"""Benchmark: program.points/s of the fitness engine on B200.

Workload (the vector configuration of the engine's benchmark set): 4,096 random
vector programs of length 4-48 over {AddV3, SubV3, CrossV3, DotV3, NormV3,
ScaleV3, +, -, *, /, constants, E, v, B}, scored (MSE) on 100,000 points with
E, v, B ~ N(0, 1) and y = |E + v x B|.  Seeded synthetic data of the
reference tests' shape (tests/linalg.rs:73-107).

One step = one MSE evaluation of the whole population over every point with
programs and data resident in HBM (a prepared batch replayed through a CUDA
graph).  L2 (126 MB; the dataset is 4 MB) is flushed between steps with a
256 MiB memset outside the timed events.  Device time per step comes from
CUDA events on the launching stream; multi-GPU runs shard programs across
ranks (weak scaling, no collective on the data path) and take the max over
ranks.

`--impl reference` times the reference's CPU evaluator in its restated form
(oracle/simd_baseline.c: the reference Rust crate cannot be built in this
image) on all host cores, on bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "program_points_per_sec"
UNIT = "program*points/s"
N_PROGRAMS = 4096
N_POINTS = 100_000


def rank_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class Clocks:
    """nvidia-smi sampler for the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(pop_packed_fn, ds, target_s: float = 3.0, repeats: int = 3):
    """Times the restated reference evaluator on all host threads on a bounded
    sample of the population; returns (program.points/s, threads, sample)."""
    from oracle import binding as O
    threads = os.cpu_count() or 1
    n = 16
    t0 = time.perf_counter()
    O.simd_mse_batch(pop_packed_fn(n), ds, threads)
    dt = time.perf_counter() - t0
    n = int(max(16, min(N_PROGRAMS, n * target_s / max(dt, 1e-3))))
    pk = pop_packed_fn(n)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.simd_mse_batch(pk, ds, threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return n * ds.num_batches * 8 / t, threads, f"{n} of {N_PROGRAMS} programs x {ds.num_samples} points, median of {repeats}"


def build_workload(rank: int):
    from rsr_b200 import workloads as W
    ds = W.lorentz_dataset(N_POINTS, seed=2)
    pop = W.lorentz_population(N_PROGRAMS, seed=12 + rank)
    return ds, pop


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return 0
    from rsr_b200 import isa as I
    ds, pop = build_workload(0)
    pk_all = I.pack(pop)
    from oracle import binding as O
    threads = os.cpu_count() or 1
    # each step: a bounded sample of the population (about 1.5 s of CPU work)
    n = 16
    t0 = time.perf_counter()
    O.simd_mse_batch(I.pack(pop[:n]), ds, threads)
    dt = time.perf_counter() - t0
    n = int(max(16, min(N_PROGRAMS, n * 1.5 / max(dt, 1e-3))))
    for _ in range(args.warmup):
        O.simd_mse_batch(I.pack(pop[:n]), ds, threads)
    times = []
    for s in range(args.steps):
        lo = (s * n) % (N_PROGRAMS - n + 1)
        pk = I.pack(pop[lo:lo + n])
        t0 = time.perf_counter()
        O.simd_mse_batch(pk, ds, threads)
        times.append(time.perf_counter() - t0)
    pp = n * ds.num_batches * 8
    value = pp * len(times) / sum(times)
    sample = f"{n} of {N_PROGRAMS} programs x {ds.num_samples} points per step"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": "vector: 4096 programs len 4-48 x 100000 points, y=|E+v x B|",
                       "programs": N_PROGRAMS, "points": N_POINTS, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "what": "AVX2 8-lane restatement of the reference's compute_mse "
                                     "(oracle/simd_baseline.c); the Rust reference cannot be built here"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_engine(args):
    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from rsr_b200 import _native as N
    from rsr_b200 import isa as I
    from rsr_b200.evaluator import Engine

    ds, pop = build_workload(rank)
    pk = I.pack(pop)
    eng = Engine(device=local)
    dd = eng.upload(ds)
    fp32_peak = eng.fp32_peak()

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if not dist:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---------------------------------------------------- batched (resident)
    tune = eng.autotune(pk, dd, reps=2)
    b = eng.prepare(pk, dd, kernel=N.KERNEL_AUTO)
    for _ in range(args.warmup):
        eng.flush_l2()
        b.run()
        b.timing()
    mse_ref = b.results()
    step_ms = []
    launches0 = eng.launch_count()
    barrier()
    eng.synchronize()
    with Clocks(local) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            eng.flush_l2()
            b.run()
            step_ms.append(b.timing()[1])
        eng.synchronize()
        t_wall = time.perf_counter() - t_wall
    barrier()
    launches = eng.launch_count() - launches0 - 0  # flushes are memsets, not kernels
    mse = b.results()
    assert np.array_equal(mse, mse_ref), "results changed between replays"
    total_ms = max_over_ranks(sum(step_ms))
    desc = b.describe()
    pp_rank = desc["program_points"]
    value = pp_rank * world * len(step_ms) / (total_ms * 1e-3)
    b.close()

    # per-kernel time of the dominant kernel (same batch, events per kernel, no graph)
    eng2 = Engine(device=local, use_graphs=False)
    dd2 = eng2.upload(ds)
    eng2.autotune(pk, dd2, reps=2)
    b2 = eng2.prepare(pk, dd2, kernel=N.KERNEL_AUTO)
    gms = []
    for i in range(max(3, min(args.steps, 20)) + 3):
        eng2.flush_l2()
        b2.run()
        b2.timing()
        g = b2.describe()["groups"]
        if i >= 3:
            gms.append([x["last_ms"] for x in g])
    groups = b2.describe()["groups"]
    b2.close()
    dom = int(np.argmax([g["flops"] for g in groups]))
    dom_ms = statistics.median([r[dom] for r in gms])
    dom_flops = groups[dom]["flops"]

    # ---------------------------------------------------------- plain kernel
    bp = eng.prepare(pk, dd, kernel=N.KERNEL_PLAIN)
    pms = []
    for i in range(3 + max(3, min(args.steps, 10))):
        eng.flush_l2()
        bp.run()
        t = bp.timing()[1]
        if i >= 3:
            pms.append(t)
    plain_value = pp_rank * world * len(pms) / (max_over_ranks(sum(pms)) * 1e-3)
    bp.close()

    # ------------------------------------------- end to end through the API
    e2e_ms, h2d, d2h = [], 0, 0
    for i in range(2 + max(3, min(args.steps, 20))):
        t0 = time.perf_counter()
        out = eng.compute_mse_batch(pk, dd)
        dt = time.perf_counter() - t0
        h2d, d2h = eng.last_transfer()
        if i >= 2:
            e2e_ms.append(dt * 1e3)
    e2e_value = pp_rank * world * len(e2e_ms) / (max_over_ranks(sum(e2e_ms)) * 1e-3)
    assert np.array_equal(out, mse_ref)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            v, cores, sample = cpu_baseline(lambda n: I.pack(pop[:n]), ds)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
        achieved = dom_flops / (dom_ms * 1e-3) / 1e12
        peak = fp32_peak / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / len(step_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "vector: 4096 programs len 4-48 x 100000 points, y=|E+v x B|",
                       "programs_per_gpu": N_PROGRAMS, "points": N_POINTS,
                       "kernel": "register-stack persistent, CUDA graph replay",
                       "l2": "flushed between steps (256 MiB memset outside the timed events)"},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "max": float(max(step_ms))},
            "plain": {"value": plain_value, "unit": UNIT, "speedup_of_batched": value / plain_value,
                      "ms_per_step": float(np.median(pms))},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": f"reg_eval_kernel profile {groups[dom]['profile']} "
                                   f"P={groups[dom]['points_per_thread']} G={groups[dom]['programs_per_warp']}",
                         "peak_source": "measured unfused FP32 lane-op rate of this GPU (rsr_measure_fp32_peak)",
                         "kernel_ms": dom_ms, "algorithmic_lane_ops": dom_flops},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": float(np.median(e2e_ms)),
                    "what": "rsr_eval_mse_batch with host programs: encode, upload, kernels, MSE download"},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "wall_s_timed": t_wall,
            "autotune": tune["chosen"],
            "programs_on_register_kernel": desc["register_kernel_programs"],
            "programs_on_slot_kernel": desc["slot_kernel_programs"],
        }
        print(json.dumps(line), flush=True)
    eng2.close()
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    return run_reference(args) if args.impl == "reference" else run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
