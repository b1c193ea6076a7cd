"""A small, fixed evaluation case for profilers (ncu), one kernel kind at a time.

    python -m rsr_b200.profile_case --workload vector --programs 1024 --kernel register --runs 3

runs one prepared batch `runs` times (no CUDA graph, so every kernel is its
own launch) and prints the per-group kernel times measured with CUDA events.
Workloads: scalar (400 points), vector (100k points, E/v/B), matrix (1M
points, M/v/u), uneven (Mat2 pairs over 16 datasets of 400..262,144 points).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import _native as N
from . import isa as I
from . import workloads as W
from .evaluator import Engine


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="vector", choices=["scalar", "vector", "matrix", "uneven"])
    ap.add_argument("--programs", type=int, default=1024)
    ap.add_argument("--points", type=int, default=0, help="override the workload's point count")
    ap.add_argument("--kernel", default="register", choices=["register", "plain", "adjoint"])
    ap.add_argument("--runs", type=int, default=3)
    ap.add_argument("--points-per-thread", type=int, default=0, help="register kernel P (default: the engine's)")
    ap.add_argument("--programs-per-warp", type=int, default=0, help="register kernel G (default: the engine's)")
    a = ap.parse_args(argv)
    eng = Engine(use_graphs=False, points_per_thread=a.points_per_thread, programs_per_warp=a.programs_per_warp)
    if a.workload == "scalar":
        ds, pop = W.scalar_dataset(a.points or 400, seed=1), W.scalar_population(a.programs, seed=11)
    elif a.workload == "vector":
        ds, pop = W.lorentz_dataset(a.points or 100_000, seed=2), W.lorentz_population(a.programs, seed=12)
    elif a.workload == "matrix":
        ds, pop = W.transform_dataset(a.points or 1_000_000, seed=3), W.transform_population(a.programs, seed=13)
    else:
        ds, pop = None, W.inverse_population(a.programs, seed=14)
    pk = I.pack(pop)
    kernel = N.KERNEL_PLAIN if a.kernel == "plain" else N.KERNEL_AUTO
    if ds is None:
        dss = [eng.upload(W.inverse_dataset(n, seed=100 + i)) for i, n in enumerate(W.uneven_sizes(16))]
        rng = np.random.default_rng(5)
        b = eng.prepare(pk, datasets=[dss[int(k)] for k in rng.integers(0, 16, pk.n)], kernel=kernel,
                        gradient=a.kernel == "adjoint")
    else:
        b = eng.prepare(pk, eng.upload(ds), kernel=kernel, gradient=a.kernel == "adjoint")
    for _ in range(a.runs):
        b.run()
        b.timing()
    d = b.describe()
    print(json.dumps({"workload": a.workload, "programs": pk.n, "kernel": a.kernel,
                      "groups": [{k: g[k] for k in ("kernel", "profile", "points_per_thread", "programs_per_warp",
                                                    "grid", "warps_per_block", "smem_bytes", "last_ms", "flops",
                                                    "program_points")} for g in d["groups"]]}))
    b.close()
    eng.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
