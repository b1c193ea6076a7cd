"""Serving loop (rsr_server in include/rsr_gpu.h) for island threads.

The reference's island threads call ``Individual::calculate_mse``
(src/engine/search/individual.rs:44-54, from island.rs:150-238) and
``optimize_individual_constants`` (src/engine/optimize/mod.rs:10-59) one
individual at a time.  Here each thread submits whole jobs -- a population to
score, score with gradients, or fit -- and waits on a ticket; the server
batches and overlaps them on the device.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Dict, Optional, Sequence

import numpy as np

from . import _native as N
from .evaluator import Engine, PopulationLike, _as_population, _packed

KINDS = {"mse": N.JOB_MSE, "grad": N.JOB_MSE_GRAD, "fit": N.JOB_FIT, "fit_auto": N.JOB_FIT_AUTO}
STATES = {N.JOB_QUEUED: "queued", N.JOB_RUNNING: "running", N.JOB_DONE: "done"}


class Server:
    def __init__(self, engine: Engine, slots: int = 4, max_batch_programs: int = 16384, max_queue: int = 65536,
                 mem_budget_bytes: int = 0):
        self.engine = engine
        o = N.ServerOptions()
        N.lib().rsr_server_options_default(C.byref(o))
        o.slots, o.max_batch_programs, o.max_queue = slots, max_batch_programs, max_queue
        o.mem_budget_bytes = mem_budget_bytes
        h = C.c_void_p()
        N.check(N.lib().rsr_server_create(engine.ctx, C.byref(o), C.byref(h)))
        self.h = h
        # output buffers stay referenced until the ticket is retired, so a
        # submitter that goes away cannot leave the server writing into freed memory
        self._live: Dict[int, dict] = {}
        self._lock = threading.Lock()

    def submit(self, programs: PopulationLike, dataset=None, datasets: Optional[Sequence] = None,
               kind: str = "mse", fit_iterations: int = 10, seed: int = 0) -> int:
        """Queues a job and returns its ticket.  kind: "mse", "grad" (MSE and
        d(MSE)/d(constants)), "fit" (L-BFGS, `fit_iterations` steps) or
        "fit_auto" (the reference's choice per program: L-BFGS, CMA-ES with
        streams from `seed`, or Nelder-Mead)."""
        pk = _packed(programs)
        pop, keep = _as_population(pk)
        n = pk.n
        mse = np.zeros(max(n, 1), np.float32)
        grad = np.zeros(max(n, 1) * 32, np.float32) if kind == "grad" else None
        params = np.array(pk.params, np.float32, copy=True) if kind in ("fit", "fit_auto") else None
        if params is not None and len(params) == 0:
            params = np.zeros(1, np.float32)
        j = N.Job()
        j.kind = KINDS[kind]
        j.fit_iterations = fit_iterations
        j.seed = seed
        j.pop = C.pointer(pop)
        dsp = None
        if datasets is not None:
            if isinstance(datasets, np.ndarray) and datasets.dtype == np.uint64:
                dsp = np.ascontiguousarray(datasets)  # device handles already
            else:
                dsp = np.asarray([self.engine._ds(d).handle for d in datasets], np.uint64)
            j.ds_per_program = dsp.ctypes.data_as(C.POINTER(C.c_uint64))
        else:
            j.ds = self.engine._ds(dataset).handle
        f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        j.mse_out, j.grad_out, j.params_out = f(mse), f(grad), f(params)
        t = C.c_uint64()
        N.check(N.lib().rsr_submit(self.h, C.byref(j), C.byref(t)))
        with self._lock:
            self._live[t.value] = {"n": n, "mse": mse, "grad": grad, "params": params, "n_params": len(pk.params)}
        return t.value

    def poll(self, ticket: int) -> str:
        s = C.c_uint32()
        N.check(N.lib().rsr_poll(self.h, ticket, C.byref(s)))
        return STATES[s.value]

    def wait(self, ticket: int, timeout: Optional[float] = None) -> dict:
        """Results of a job: {"mse", "grad" | "params" (per kind), "info"}.
        Raises RsrError on the job's failure, or ETIMEDOUT (job kept)."""
        info = N.JobInfo()
        us = 0 if timeout is None else max(1, int(timeout * 1e6))
        rc = N.lib().rsr_wait(self.h, ticket, us, C.byref(info))
        if rc == N.RSR_ETIMEDOUT:
            N.check(rc)
        with self._lock:
            bufs = self._live.pop(ticket, None)
        N.check(rc)
        n = bufs["n"]
        out = {"mse": bufs["mse"][:n],
               "info": {"batch_jobs": info.batch_jobs, "queue_ms": info.queue_ms, "latency_ms": info.latency_ms}}
        if bufs["grad"] is not None:
            out["grad"] = bufs["grad"][:n * 32].reshape(n, 32)
        if bufs["params"] is not None:
            out["params"] = bufs["params"][:bufs["n_params"]]
        return out

    def cancel(self, ticket: int) -> None:
        N.check(N.lib().rsr_cancel(self.h, ticket))

    def stats(self, reset: bool = False) -> dict:
        s = N.ServingStats()
        N.check(N.lib().rsr_server_stats(self.h, C.byref(s), int(reset)))
        return {k: getattr(s, k) for k, _ in N.ServingStats._fields_}

    def close(self) -> None:
        if self.h:
            N.check(N.lib().rsr_server_destroy(self.h))
            self.h = None
            with self._lock:
                self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
