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

The line also carries the other workloads as legs: `matrix` (256 programs
x 1M points: MSE, MSE + gradient with the adjoint kernel's roofline, a
20-iteration L-BFGS fit) and `uneven` (8192 programs over 16 datasets of
400-262,144 points, graph replay), besides the plain-kernel, adjoint,
end-to-end, serving and search legs.

`--impl reference` times the reference's CPU evaluator in its restated form
(oracle/simd_baseline.c: the reference Rust crate cannot be built in this
image) on all host cores, on bounded samples of the same workload.

`--case` runs one fixed evaluation case for profilers instead (`--workload`,
`--programs`, `--points`, `--kernel register|plain|adjoint|slot-adjoint`,
`--runs`, `--points-per-thread`, `--programs-per-warp`), a small case for an
ncu capture.  Given to the benchmark itself, `--points-per-thread` and
`--programs-per-warp` fix the register kernel's shape in place of the
autotuner (whose timings under ncu are not the bench's).
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

# DRAM bytes (read + write) of the dominant kernel's launches in one step of
# this workload (three spill-depth classes, P=8 G=4), from one ncu capture of
# `bench.py --case --workload vector --programs 4096 --kernel register --runs 3
# --points-per-thread 8 --programs-per-warp 4` (dram__bytes_read/write.sum):
# 4,711,424 + 4,775,680 + 4,116,736 read, 512 written.  ncu replays each launch
# with cold caches, so each re-reads the 4 MB dataset; in a step the second
# and third launches find it in L2.
DOMINANT_KERNEL_DRAM_BYTES = 13_604_352
METRIC = "program_points_per_sec"
UNIT = "program*points/s"
N_PROGRAMS = 4096
N_POINTS = 100_000
# The workload both arms report (the engine and the reference CPU arm print
# the same config).
CONFIG = {"workload": "vector: 4096 programs len 4-48 x 100000 points, y=|E+v x B|",
          "programs": N_PROGRAMS, "points": N_POINTS,
          "l2": "engine arm: flushed between steps (256 MiB memset outside the timed events); "
                "CPU reference arm: no flush"}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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
            "config": dict(CONFIG),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "cpu_model": cpu_model(),
                             "kind": "port", "sample": sample,
                             "what": "AVX2 8-lane restatement of the reference's compute_mse "
                                     "(oracle/simd_baseline.c); the Rust reference cannot be built here"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def serving_bench(eng, jobs: int, rate: float, threads: int = 16, seed: int = 7, slots: int = 4):
    """The serving mix: `threads` island threads submit `jobs` jobs with
    Poisson arrivals at `rate` jobs/s in total; each job holds 64-1024
    programs (uniform) against one of the four workloads' resident datasets
    (scalar 400 points; vector 100k; matrix 1M; uneven: 16 datasets of 400 to
    262,144 points, one per program); 30% of the jobs ask for a 10-step
    constant fit, the rest for MSE fitness.  Latency is submit -> results
    written, measured by the server."""
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    from rsr_b200.serving import Server
    rng = np.random.default_rng(seed)
    pools = {"scalar": (W.scalar_population(1024, seed=31), eng.upload(W.scalar_dataset(400, seed=1))),
             "vector": (W.lorentz_population(1024, seed=32), eng.upload(W.lorentz_dataset(100_000, seed=2))),
             "matrix": (W.transform_population(1024, seed=33), eng.upload(W.transform_dataset(1_000_000, seed=3)))}
    uneven = [eng.upload(W.inverse_dataset(n, seed=40 + i)) for i, n in enumerate(W.uneven_sizes(16))]
    pools["uneven"] = (W.inverse_population(1024, seed=34), None)
    names = list(pools)
    plan = []
    for _ in range(jobs):
        name = names[int(rng.integers(0, 4))]
        n = int(rng.integers(64, 1025))
        lo = int(rng.integers(0, 1024 - n + 1))
        progs, dsd = pools[name]
        pk = I.pack(progs[lo:lo + n])
        handles = None
        if dsd is None:
            handles = np.array([uneven[int(k)].handle for k in rng.integers(0, 16, n)], np.uint64)
        kind = "fit" if rng.random() < 0.3 else "mse"
        plan.append((pk, dsd, handles, kind))
    gaps = rng.exponential(threads / rate, jobs)
    per_thread = [list(range(t, jobs, threads)) for t in range(threads)]
    srv = Server(eng, slots=slots)
    tickets = [None] * jobs
    errors = []

    def island(idx):
        t_next = time.perf_counter()
        for i in idx:
            t_next += gaps[i]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            pk, dsd, handles, kind = plan[i]
            try:
                tickets[i] = srv.submit(pk, dsd, datasets=handles, kind=kind, fit_iterations=10)
            except Exception as e:  # refused: counted by the server
                errors.append(str(e))

    th = [threading.Thread(target=island, args=(idx,)) for idx in per_thread]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    t_submit = time.perf_counter() - t0
    batch_sizes = []
    for t in tickets:
        if t is not None:
            batch_sizes.append(srv.wait(t)["info"]["batch_jobs"])
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    pts = {k: (v[1].num_batches * 8 if v[1] is not None else None) for k, v in pools.items()}
    return {"jobs": jobs, "arrival_rate_jobs_per_s": rate, "submit_s": t_submit, "drain_s": wall,
            "completed": st["completed"], "failed": st["failed"], "refused": st["refused"],
            "latency_ms": {"p50": st["p50_ms"], "p95": st["p95_ms"], "p99": st["p99_ms"], "max": st["max_ms"]},
            "program_points_per_sec": st["program_points_per_sec"],
            "launches": st["launches"], "mean_jobs_per_launch": float(np.mean(batch_sizes)) if batch_sizes else 0.0,
            "peak_inflight_bytes": st["peak_mem_bytes"], "slots": slots, "submitter_threads": threads,
            "what": "rsr_server: 64-1024 programs per job, 30% with a 10-step L-BFGS fit, over the scalar/vector/"
                    "matrix/uneven datasets resident on the device; latency = submit -> results written "
                    "(program_points counts one evaluation per program)"}


def serving_light_bench(eng, jobs: int = 300, rate: float = 150.0, threads: int = 8, seed: int = 9):
    """Evaluation latency below saturation: `threads` island threads submit
    MSE-only jobs of 64-1024 vector-workload programs (100k points) with
    Poisson arrivals at `rate` jobs/s in total, a load the device keeps up
    with, so latency is the jobs' own service time rather than queueing.
    The server is warmed up before the statistics start: 8 jobs of 1024
    programs submitted 0.3 ms apart, so that each slot takes one while the
    others are busy and grows its buffers to the largest job (a slot
    allocates on its first job of a new size), then 16 of the stream's own
    jobs."""
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    from rsr_b200.serving import Server
    rng = np.random.default_rng(seed)
    progs = W.lorentz_population(1024, seed=35)
    d = eng.upload(W.lorentz_dataset(100_000, seed=2))
    plan = []
    for _ in range(jobs):
        n = int(rng.integers(64, 1025))
        lo = int(rng.integers(0, 1024 - n + 1))
        plan.append(I.pack(progs[lo:lo + n]))
    gaps = rng.exponential(threads / rate, jobs)
    srv = Server(eng, slots=4)
    # warm-up outside the statistics: a new server's slots allocate their
    # device and pinned buffers and start their encoding threads on their
    # first jobs, so every slot is given the largest job at least once
    big = I.pack(progs)
    warm = []
    for _ in range(8):
        warm.append(srv.submit(big, d, kind="mse"))
        time.sleep(0.0003)
    for t in warm:
        srv.wait(t)
    for pk in plan[:16]:
        srv.wait(srv.submit(pk, d, kind="mse"))
    srv.stats(reset=True)
    tickets = [None] * jobs

    def island(idx):
        t_next = time.perf_counter()
        for i in idx:
            t_next += gaps[i]
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            tickets[i] = srv.submit(plan[i], d, kind="mse")

    th = [threading.Thread(target=island, args=(list(range(t, jobs, threads)),)) for t in range(threads)]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    for t in tickets:
        srv.wait(t)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    d.release()
    return {"jobs": jobs, "arrival_rate_jobs_per_s": rate, "drain_s": wall, "completed": st["completed"],
            "latency_ms": {"p50": st["p50_ms"], "p95": st["p95_ms"], "p99": st["p99_ms"], "max": st["max_ms"]},
            "what": "rsr_server, MSE jobs of 64-1024 programs x 100k points (vector workload) below saturation; "
                    "latency = submit -> results written"}


def _replay_ms(eng, b, reps: int, warm: int = 3, results: bool = False):
    """Device ms per run of a prepared batch (graph replay when the engine
    uses graphs), L2 flushed before each run."""
    out = []
    for i in range(warm + reps):
        eng.flush_l2()
        b.run()
        if results:
            b.results()
        t = b.timing()[1]
        if i >= warm:
            out.append(t)
    return out


def _group_ms(eng, b, reps: int, warm: int = 3):
    """Per-launch device ms of a prepared batch on an engine without graphs
    (CUDA events around each launch): (per-run lists, group descriptions)."""
    per = []
    for i in range(warm + reps):
        eng.flush_l2()
        b.run()
        b.timing()
        if i >= warm:
            per.append([g["last_ms"] for g in b.describe()["groups"]])
    return per, b.describe()["groups"]


def matrix_bench(eng, eng_nog, fp32_peak: float, reps: int):
    """The matrix workload with constant fitting: M a Mat3 ~ U(-1, 1), v, u
    ~ N(0, 1) Vec3, y = |M v - u| over 1,000,000 points; 256 programs of
    length 8-40 with 1-8 constants.  MSE and MSE + gradient of the whole
    population (graph replay), the adjoint kernel's lane-op rate against the
    FP32 peak, and a 20-iteration L-BFGS fit of the differentiable programs."""
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    ds = W.transform_dataset(1_000_000, seed=3)
    pop = W.transform_population(256, seed=13)
    pk = I.pack(pop)
    d = eng.upload(ds)
    b = eng.prepare(pk, d)
    mse_ms = _replay_ms(eng, b, reps)
    pp = b.describe()["program_points"]
    b.close()
    bg = eng.prepare(pk, d, gradient=True)
    adj_ms = _replay_ms(eng, bg, reps, results=True)
    bg.close()
    d2 = eng_nog.upload(ds)
    bg2 = eng_nog.prepare(pk, d2, gradient=True)
    per, groups = _group_ms(eng_nog, bg2, reps)
    bg2.close()
    d2.release()
    adj = [i for i, g in enumerate(groups) if g["kernel"] in ("adjoint", "register_adjoint")]
    k_ms = statistics.median([sum(r[i] for i in adj) for r in per])
    k_flops = sum(groups[i]["flops"] for i in adj)
    fit = [p for p in pop if p.is_differentiable()]
    eng.fit_lbfgs(fit[:16], d, max_iterations=2)  # warm-up
    eng.synchronize()
    t0 = time.perf_counter()
    _, fit_mse, stats = eng.fit_lbfgs(fit, d, max_iterations=20)
    fit_s = time.perf_counter() - t0
    d.release()
    return {"workload": "matrix: 256 programs len 8-40, 1-8 constants x 1000000 points, y=|M v - u|",
            "mse": {"ms_per_step": float(np.median(mse_ms)), "value": pp / (np.median(mse_ms) * 1e-3),
                    "unit": UNIT},
            "adjoint": {"ms_per_step": float(np.median(adj_ms)), "value": pp / (np.median(adj_ms) * 1e-3),
                        "unit": UNIT, "over_mse": float(np.median(adj_ms) / np.median(mse_ms)),
                        "what": "MSE and d(MSE)/d(constants) of all 256 programs, graph replay"},
            "adjoint_roofline": {"bound": "fp32", "achieved": k_flops / (k_ms * 1e-3) / 1e12,
                                 "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                                 "frac": k_flops / (k_ms * 1e-3) / fp32_peak, "kernel_ms": k_ms,
                                 "algorithmic_lane_ops": k_flops, "launches": len(adj),
                                 "what": "forward + reverse-rule lane-ops of the live trees (encoder.cpp "
                                         "reverse_flops) over the adjoint launches' CUDA-event time"},
            "lbfgs_20": {"programs": len(fit), "seconds": fit_s, "iterations": stats["iterations"],
                         "gradient_launches": stats["gradient_evaluations"],
                         "mse_launches": stats["mse_evaluations"],
                         "mean_final_mse": float(np.mean(fit_mse[fit_mse < np.finfo(np.float32).max]))}}


def uneven_bench(eng, reps: int):
    """The uneven batch: A, B Mat2 (A = 2I + U(-0.5, 0.5), B ~ N(0, 1)),
    y = Tr(A^-1 B) + det(A); 8192 programs of length 4-64 against 16 datasets
    of 400 to 262,144 points (log-uniform), one autotuned launch set replayed
    through a CUDA graph."""
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    sizes = W.uneven_sizes(16)
    dd = [eng.upload(W.inverse_dataset(n, seed=100 + i)) for i, n in enumerate(sizes)]
    pop = W.inverse_population(8192, seed=14)
    which = np.random.default_rng(5).integers(0, 16, len(pop))
    pk = I.pack(pop)
    handles = [dd[k] for k in which]
    tune = eng.autotune(pk, datasets=handles, reps=2)
    b = eng.prepare(pk, datasets=handles)
    ms = _replay_ms(eng, b, reps)
    pp = b.describe()["program_points"]
    b.close()
    for x in dd:
        x.release()
    return {"workload": "uneven: 8192 programs len 4-64 over 16 datasets of 400-262144 points, "
                        "y=Tr(A^-1 B)+det(A)",
            "ms_per_step": float(np.median(ms)), "value": pp / (np.median(ms) * 1e-3), "unit": UNIT,
            "program_points": pp, "autotune": tune["chosen"]}


def search_bench(eng):
    """Config C1 end to end: MSE of 1024 random scalar programs on 400
    points, then the island search (24 islands x 25, the reference's
    defaults, operators {+, -, *, /, sin, cos, exp}) to MSE < 1e-7 with
    every score and constant fit on the engine."""
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    from rsr_b200.search import engine as S
    ds = W.scalar_dataset(400, seed=1)
    d = eng.upload(ds)
    pk = I.pack(W.scalar_population(1024, seed=11))
    eng.compute_mse_batch(pk, d)
    t0 = time.perf_counter()
    eng.compute_mse_batch(pk, d)
    t_pop = time.perf_counter() - t0
    cfg = S.Config(excluded_ops=["SqrF", "SqrtF", "LnF"])
    t0 = time.perf_counter()
    res = S.SymbolicRegressor(cfg).fit(eng, d, [I.FLOAT])
    t_fit = time.perf_counter() - t0
    d.release()
    return {"workload": "scalar: y=2.5x^2-1.2, 400 points; 1024 programs scored, then GP search to MSE<1e-7",
            "population_mse_ms": t_pop * 1e3, "generations": res.generations, "seconds": t_fit,
            "mse": res.mse, "reached_target": bool(res.mse <= 1e-7), "equation": res.equation}


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
    shape = dict(points_per_thread=args.points_per_thread, programs_per_warp=args.programs_per_warp)
    eng = Engine(device=local, **shape)
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
    fixed = {"chosen": [{"fixed": True, "P": args.points_per_thread, "G": args.programs_per_warp}]}
    tune = eng.autotune(pk, dd, reps=2) if not args.points_per_thread else fixed
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
    eng2 = Engine(device=local, use_graphs=False, **shape)
    dd2 = eng2.upload(ds)
    if not args.points_per_thread:
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
    # the dominant kernel: the register kernel of the profile doing most of
    # the work, which runs as one launch per spill-depth class
    prof_flops = {}
    for g in groups:
        if g["kernel"] == "register":
            prof_flops[g["profile"]] = prof_flops.get(g["profile"], 0) + g["flops"]
    dom_prof = max(prof_flops, key=prof_flops.get)
    dom_idx = [i for i, g in enumerate(groups) if g["kernel"] == "register" and g["profile"] == dom_prof]
    dom = dom_idx[0]
    dom_ms = statistics.median([sum(r[i] for i in dom_idx) for r in gms])
    dom_flops = sum(groups[i]["flops"] for i in dom_idx)

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

    # ------------------------------------------ adjoint: MSE and gradient
    bg = eng.prepare(pk, dd, gradient=True)
    ams = []
    for i in range(3 + max(3, min(args.steps, 10))):
        eng.flush_l2()
        bg.run()
        bg.results()
        t = bg.timing()[1]
        if i >= 3:
            ams.append(t)
    adj_value = pp_rank * world * len(ams) / (max_over_ranks(sum(ams)) * 1e-3)
    adj_kinds = sorted({g["kernel"] for g in bg.describe()["groups"]})
    bg.close()
    # the same gradients on the slot-file adjoint alone, for comparison
    eng_s = Engine(device=local, flags=N.OPT_SLOT_ADJOINT)
    bs = eng_s.prepare(pk, eng_s.upload(ds), gradient=True)
    sms = []
    for i in range(3 + max(3, min(args.steps, 10))):
        eng_s.flush_l2()
        bs.run()
        bs.results()
        t = bs.timing()[1]
        if i >= 3:
            sms.append(t)
    bs.close()
    eng_s.close()

    # ------------------- register interpreter without the batching extras
    # one program per work item, 4 points per lane, no autotuning, no graph:
    # the register kernel as a one-program-per-warp interpreter
    eng3 = Engine(points_per_thread=4, programs_per_warp=1, use_graphs=False)
    b3 = eng3.prepare(pk, eng3.upload(ds))
    rms = []
    for i in range(3 + max(3, min(args.steps, 10))):
        eng3.flush_l2()
        b3.run()
        t = b3.timing()[1]
        if i >= 3:
            rms.append(t)
    reg1_value = pp_rank * world * len(rms) / (max_over_ranks(sum(rms)) * 1e-3)
    b3.close()
    eng3.close()

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

    matrix = uneven = None
    if not args.no_configs:
        matrix = matrix_bench(eng, eng2, fp32_peak, max(3, min(args.steps, 10)))
        uneven = uneven_bench(eng, max(3, min(args.steps, 10)))

    serving = None
    if not args.no_serving:
        serving = serving_bench(eng, args.serving_jobs, args.serving_rate, slots=8)
        # the mix's capacity is what the saturated run completed per second;
        # the same mix offered at 50% and 90% of it gives the latency below
        # saturation
        capacity = serving["completed"] / serving["drain_s"]
        serving["capacity_jobs_per_s"] = capacity
        serving["at_fraction_of_capacity"] = {}
        for frac, jobs in ((0.5, 60), (0.9, 100)):
            r = serving_bench(eng, jobs, frac * capacity, slots=8, seed=17)
            serving["at_fraction_of_capacity"][str(frac)] = {
                "arrival_rate_jobs_per_s": r["arrival_rate_jobs_per_s"], "jobs": jobs, "completed": r["completed"],
                "latency_ms": r["latency_ms"], "drain_s": r["drain_s"]}
    serving_light = None
    if not args.no_serving:
        serving_light = serving_light_bench(eng)
    search = None
    if world == 1 and not args.no_search:
        search = search_bench(eng)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            v, cores, sample = cpu_baseline(lambda n: I.pack(pop[:n]), ds)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(), "kind": "port",
                   "sample": sample,
                   "what": "AVX2 8-lane restatement of the reference's compute_mse (oracle/simd_baseline.c) on "
                           "all host threads; the Rust reference cannot be built here"}
        achieved = dom_flops / (dom_ms * 1e-3) / 1e12
        peak = fp32_peak / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / len(step_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": dict(CONFIG),
            "kernel": "register-stack persistent, CUDA graph replay; programs per GPU = config.programs",
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                           "max": float(max(step_ms))},
            "adjoint": {"value": adj_value, "unit": UNIT, "ms_per_step": float(np.median(ams)),
                        "over_mse": float(np.median(ams)) / (total_ms / len(step_ms)), "kernels": adj_kinds,
                        "slot_file_adjoint_ms": float(np.median(sms)),
                        "what": "MSE and d(MSE)/d(constants) of the same batch, reverse-mode adjoint kernels, "
                                "graph replay; slot_file_adjoint_ms: the same with RSR_OPT_SLOT_ADJOINT"},
            "register_one_program_per_item": {
                "value": reg1_value, "unit": UNIT, "speedup_of_batched": value / reg1_value,
                "ms_per_step": float(np.median(rms)),
                "what": "register kernel, G=1, P=4, no autotuning, no CUDA graph"},
            "plain": {"value": plain_value, "unit": UNIT, "speedup_of_batched": value / plain_value,
                      "ms_per_step": float(np.median(pms))},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": DOMINANT_KERNEL_DRAM_BYTES,
                         "traffic_note": "ncu dram__bytes_read+write of the dominant kernel's launches in one step "
                                         "(cold caches per launch); algorithmic bytes ~4.4 MB (dataset once + "
                                         "programs)",
                         "kernel": f"reg_eval_kernel profile {groups[dom]['profile']} "
                                   f"P={groups[dom]['points_per_thread']} G={groups[dom]['programs_per_warp']}, "
                                   f"{len(dom_idx)} launches (one per spill-depth class)",
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
            "matrix": matrix,
            "uneven": uneven,
            "serving": serving,
            "serving_below_saturation": serving_light,
            "search": search,
        }
        print(json.dumps(line), flush=True)
    eng2.close()
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_case(args):
    """One fixed evaluation case for profilers (ncu), one kernel kind at a
    time: a prepared batch of the chosen workload run `--runs` times without
    a CUDA graph (every kernel its own launch); prints the per-launch CUDA
    event times.  Workloads: scalar (400 points), vector (100k points),
    matrix (1M points), uneven (16 datasets of 400-262,144 points)."""
    from rsr_b200 import _native as N
    from rsr_b200 import isa as I
    from rsr_b200 import workloads as W
    from rsr_b200.evaluator import Engine
    eng = Engine(use_graphs=False, points_per_thread=args.points_per_thread,
                 programs_per_warp=args.programs_per_warp,
                 flags=N.OPT_SLOT_ADJOINT if args.kernel == "slot-adjoint" else 0)
    if args.workload == "scalar":
        ds, pop = W.scalar_dataset(args.points or 400, seed=1), W.scalar_population(args.programs, seed=11)
    elif args.workload == "vector":
        ds, pop = W.lorentz_dataset(args.points or N_POINTS, seed=2), W.lorentz_population(args.programs, seed=12)
    elif args.workload == "matrix":
        ds, pop = (W.transform_dataset(args.points or 1_000_000, seed=3),
                   W.transform_population(args.programs, seed=13))
    else:
        ds, pop = None, W.inverse_population(args.programs, seed=14)
    pk = I.pack(pop)
    kernel = N.KERNEL_PLAIN if args.kernel == "plain" else N.KERNEL_AUTO
    grad = args.kernel in ("adjoint", "slot-adjoint")
    if ds is None:
        dss = [eng.upload(W.inverse_dataset(n, seed=100 + i)) for i, n in enumerate(W.uneven_sizes(16))]
        which = np.random.default_rng(5).integers(0, 16, pk.n)
        b = eng.prepare(pk, datasets=[dss[int(k)] for k in which], kernel=kernel, gradient=grad)
    else:
        b = eng.prepare(pk, eng.upload(ds), kernel=kernel, gradient=grad)
    for _ in range(args.runs):
        b.run()
        b.timing()
    d = b.describe()
    print(json.dumps({"workload": args.workload, "programs": pk.n, "kernel": args.kernel,
                      "groups": [{k: g[k] for k in ("kernel", "profile", "points_per_thread", "programs_per_warp",
                                                    "grid", "warps_per_block", "smem_bytes", "last_ms", "flops",
                                                    "program_points")} for g in d["groups"]]}))
    b.close()
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-mix leg")
    ap.add_argument("--no-search", action="store_true", help="skip the GP-search leg (config C1)")
    ap.add_argument("--no-configs", action="store_true", help="skip the matrix and uneven workload legs")
    ap.add_argument("--serving-jobs", type=int, default=400)
    ap.add_argument("--case", action="store_true",
                    help="run one fixed evaluation case for profilers instead of the benchmark (below)")
    ap.add_argument("--workload", default="vector", choices=["scalar", "vector", "matrix", "uneven"])
    ap.add_argument("--programs", type=int, default=1024)
    ap.add_argument("--points", type=int, default=0, help="--case: override the workload's point count")
    ap.add_argument("--kernel", default="register", choices=["register", "plain", "adjoint", "slot-adjoint"],
                    help="--case: adjoint runs the register adjoint where it applies, slot-adjoint the slot-file one")
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--points-per-thread", type=int, default=0,
                    help="register kernel P (0: tuned); given, the benchmark's headline skips the autotuner")
    ap.add_argument("--programs-per-warp", type=int, default=0, help="register kernel G (0: tuned)")
    ap.add_argument("--serving-rate", type=float, default=2000.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.case:
        return run_case(args)
    return run_reference(args) if args.impl == "reference" else run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
