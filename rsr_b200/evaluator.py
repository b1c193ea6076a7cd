"""Fitness evaluation on the B200: the reference's evaluator API over the C ABI.

``compute_mse`` and ``compute_mse_with_gradient`` keep the signatures and
semantics of src/engine/eval/evaluator.rs:153 and :177 (one program, one
dataset, f32::MAX for non-finite fitness); the ``*_batch`` forms score a whole
population in one launch, and ``PreparedBatch`` keeps programs and datasets
resident for repeated runs (CUDA-graph replay).
"""
from __future__ import annotations

import ctypes as C
import json
from typing import Dict, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native as N
from .dataset import Dataset
from .isa import PackedPrograms, Program, pack

_f32p = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
_u32p = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))
_u8p = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8))
_u64p = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint64))


def _as_program(p: Program):
    code = np.ascontiguousarray(p.code_array())
    kinds = np.ascontiguousarray(p.kinds())
    params = np.ascontiguousarray(p.flatten_params())
    keep = (code, kinds, params)
    s = N.Program(_u32p(code), len(code), _u8p(kinds), len(kinds), _f32p(params), len(params))
    return s, keep


def _as_population(pk: PackedPrograms):
    arrs = [np.ascontiguousarray(a) for a in (pk.code, pk.code_off, pk.kinds, pk.kind_off, pk.params, pk.param_off)]
    code, code_off, kinds, kind_off, params, param_off = arrs
    s = N.Population(pk.n, _u32p(code), _u64p(code_off), _u8p(kinds), _u64p(kind_off), _f32p(params),
                     _u64p(param_off))
    return s, arrs


class DeviceDataset:
    """A dataset resident on the device (handle of the C ABI)."""

    def __init__(self, engine: "Engine", handle: int, num_features: int, num_batches: int, num_samples: int):
        self.engine, self.handle = engine, handle
        self.num_features, self.num_batches, self.num_samples = num_features, num_batches, num_samples

    def release(self) -> None:
        if self.handle:
            N.check(N.lib().rsr_dataset_release(self.engine.ctx, self.handle))
            self.handle = 0


PopulationLike = Union[Sequence[Program], PackedPrograms]


def _packed(pop: PopulationLike) -> PackedPrograms:
    return pop if isinstance(pop, PackedPrograms) else pack(list(pop))


class Engine:
    """One context on one GPU (rsr_ctx)."""

    def __init__(self, device: int = 0, kernel: int = N.KERNEL_AUTO, points_per_thread: int = 0,
                 programs_per_warp: int = 0, use_graphs: bool = True, mem_budget_bytes: int = 0,
                 flags: int = 0):
        L = N.lib()
        opts = N.Options()
        L.rsr_options_default(C.byref(opts))
        opts.kernel = kernel
        opts.points_per_thread = points_per_thread
        opts.programs_per_warp = programs_per_warp
        opts.use_graphs = 1 if use_graphs else 0
        opts.mem_budget_bytes = mem_budget_bytes
        opts.flags = flags
        ctx = C.c_void_p()
        N.check(L.rsr_ctx_create(device, C.byref(opts), C.byref(ctx)))
        self.ctx = ctx
        self._cache: Dict[int, tuple] = {}

    def close(self) -> None:
        if self.ctx:
            N.lib().rsr_ctx_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ datasets
    def upload(self, ds: Dataset) -> DeviceDataset:
        # cache by object identity; the entry keeps the Dataset alive so its
        # id() cannot be reused by another object
        key = id(ds)
        hit = self._cache.get(key)
        if hit is not None and hit[0] is ds and hit[1].handle:
            return hit[1]
        ff = np.ascontiguousarray(ds.feature_flat, np.float32)
        tb = np.ascontiguousarray(ds.target_batches, np.float32)
        h = C.c_uint64()
        N.check(N.lib().rsr_dataset_upload(self.ctx, ff.ctypes.data, tb.ctypes.data, ds.num_features,
                                           ds.num_batches, ds.num_samples, C.byref(h)))
        d = DeviceDataset(self, h.value, ds.num_features, ds.num_batches, ds.num_samples)
        self._cache[key] = (ds, d)
        return d

    def upload_rows(self, x_rows, y, normalize: bool = False):
        """Dataset::new on the device (src/engine/data/dataset.rs:37-169):
        raw rows in, a resident dataset out, z-scored on the device when
        asked.  Returns (DeviceDataset, {"means", "stds"}) -- the last entry
        of each is the target's."""
        x = np.ascontiguousarray(x_rows, np.float32)
        yy = np.ascontiguousarray(y, np.float32)
        n = len(yy)
        nf = x.shape[1] if x.ndim == 2 else 0
        stats = np.zeros(2 * (nf + 1), np.float32)
        h = C.c_uint64()
        N.check(N.lib().rsr_dataset_upload_rows(self.ctx, x.ctypes.data if nf else None, yy.ctypes.data, nf, n,
                                                int(normalize), stats.ctypes.data, C.byref(h)))
        d = DeviceDataset(self, h.value, nf, (n + 7) // 8, n)
        return d, {"means": stats[:nf + 1], "stds": stats[nf + 1:]}

    def subset(self, dataset, target_samples: int) -> DeviceDataset:
        """Dataset::subset (dataset.rs:360-447) of a resident dataset, resident."""
        src = self._ds(dataset)
        h = C.c_uint64()
        N.check(N.lib().rsr_dataset_subset(self.ctx, src.handle, target_samples, C.byref(h)))
        m = min(target_samples, src.num_samples)
        return DeviceDataset(self, h.value, src.num_features, (m + 7) // 8, m)

    def download(self, dataset):
        """A resident dataset in the AoSoA layout: (feature_flat, target_batches)."""
        d = self._ds(dataset)
        ff = np.zeros(max(1, d.num_batches * d.num_features * 8), np.float32)
        tb = np.zeros(d.num_batches * 8, np.float32)
        N.check(N.lib().rsr_dataset_download(self.ctx, d.handle, ff.ctypes.data, tb.ctypes.data))
        return ff[:d.num_batches * d.num_features * 8], tb

    def _ds(self, ds) -> DeviceDataset:
        return ds if isinstance(ds, DeviceDataset) else self.upload(ds)

    # ----------------------------------------------- reference drop-ins
    def compute_mse(self, program: Program, dataset) -> float:
        d = self._ds(dataset)
        s, keep = _as_program(program)
        out = C.c_float()
        N.check(N.lib().rsr_compute_mse(self.ctx, C.byref(s), d.handle, C.byref(out)))
        return float(out.value)

    def compute_mse_with_gradient(self, program: Program, dataset) -> Tuple[float, np.ndarray]:
        d = self._ds(dataset)
        s, keep = _as_program(program)
        out = C.c_float()
        grad = np.zeros(32, np.float32)
        N.check(N.lib().rsr_compute_mse_with_gradient(self.ctx, C.byref(s), d.handle, C.byref(out),
                                                      grad.ctypes.data))
        return float(out.value), grad

    def eval_points(self, program: Program, dataset) -> np.ndarray:
        d = self._ds(dataset)
        s, keep = _as_program(program)
        out = np.zeros(d.num_batches * 8, np.float32)
        N.check(N.lib().rsr_eval_points(self.ctx, C.byref(s), d.handle, out.ctypes.data))
        return out

    # ------------------------------------------------------------ batched
    def compute_mse_batch(self, programs: PopulationLike, dataset=None, datasets=None,
                          kernel: int = N.KERNEL_AUTO) -> np.ndarray:
        pk = _packed(programs)
        s, keep = _as_population(pk)
        out = np.zeros(pk.n, np.float32)
        h, dsp = self._handles(pk.n, dataset, datasets)
        N.check(N.lib().rsr_eval_mse_batch(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None,
                                           kernel, out.ctypes.data))
        return out

    def compute_mse_grad_batch(self, programs: PopulationLike, dataset=None, datasets=None):
        pk = _packed(programs)
        s, keep = _as_population(pk)
        mse = np.zeros(pk.n, np.float32)
        grad = np.zeros((pk.n, 32), np.float32)
        h, dsp = self._handles(pk.n, dataset, datasets)
        N.check(N.lib().rsr_eval_mse_grad_batch(self.ctx, C.byref(s), h,
                                                dsp.ctypes.data if dsp is not None else None,
                                                mse.ctypes.data, grad.ctypes.data))
        return mse, grad

    def fit_lbfgs(self, programs: PopulationLike, dataset=None, max_iterations: int = 15, datasets=None):
        """run_lbfgs (src/engine/optimize/lbfgs.rs:9-165) for every program at
        once.  Returns (fitted flat params, final mse, stats dict); the
        reference's default is 15 iterations (optimize/mod.rs:50-52)."""
        pk = _packed(programs)
        s, keep = _as_population(pk)
        h, dsp = self._handles(pk.n, dataset, datasets)
        params = np.zeros(max(1, len(pk.params)), np.float32)
        mse = np.zeros(pk.n, np.float32)
        st = N.FitStats()
        N.check(N.lib().rsr_fit_lbfgs(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None,
                                      max_iterations, params.ctypes.data, mse.ctypes.data, C.byref(st)))
        return params[:len(pk.params)], mse, {"iterations": st.iterations,
                                              "gradient_evaluations": st.gradient_evaluations,
                                              "mse_evaluations": st.mse_evaluations}

    def fit_nelder_mead(self, programs: PopulationLike, dataset=None, max_iterations: int = 50, datasets=None):
        """run_nelder_mead (src/engine/optimize/nelder_mead.rs:9-165) for
        every program at once.  Returns (fitted flat params, best mse, stats)."""
        pk = _packed(programs)
        s, keep = _as_population(pk)
        h, dsp = self._handles(pk.n, dataset, datasets)
        params = np.zeros(max(1, len(pk.params)), np.float32)
        mse = np.zeros(pk.n, np.float32)
        st = N.FitStats()
        N.check(N.lib().rsr_fit_nelder_mead(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None,
                                            max_iterations, params.ctypes.data, mse.ctypes.data, C.byref(st)))
        return params[:len(pk.params)], mse, {"iterations": st.iterations,
                                              "gradient_evaluations": st.gradient_evaluations,
                                              "mse_evaluations": st.mse_evaluations}

    def fit_cma_es(self, programs: PopulationLike, dataset=None, max_iterations: int = 6, datasets=None,
                   seed: int = 0, rng: np.random.Generator = None):
        """run_cma_es (src/engine/optimize/cmaes.rs:19-192) for every program
        at once, program i drawing from a stream seeded from (seed, i); with
        `rng` the seed is drawn from it.  Returns (fitted flat params, best
        mse, stats)."""
        pk = _packed(programs)
        s, keep = _as_population(pk)
        h, dsp = self._handles(pk.n, dataset, datasets)
        if rng is not None:
            seed = int(rng.integers(0, 2 ** 63))
        params = np.zeros(max(1, len(pk.params)), np.float32)
        mse = np.zeros(pk.n, np.float32)
        st = N.FitStats()
        N.check(N.lib().rsr_fit_cma_es(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None,
                                       max_iterations, seed, params.ctypes.data, mse.ctypes.data, C.byref(st)))
        return params[:len(pk.params)], mse, {"iterations": st.iterations, "mse_evaluations": st.mse_evaluations}

    def eval_points_batch(self, programs: PopulationLike, dataset, kernel: int = N.KERNEL_AUTO) -> np.ndarray:
        pk = _packed(programs)
        s, keep = _as_population(pk)
        d = self._ds(dataset)
        out = np.zeros((pk.n, d.num_batches * 8), np.float32)
        N.check(N.lib().rsr_eval_points_batch(self.ctx, C.byref(s), d.handle, kernel, out.ctypes.data))
        return out

    def _handles(self, n, dataset, datasets):
        if datasets is not None:
            hs = np.asarray([self._ds(d).handle for d in datasets], np.uint64)
            if len(hs) != n:
                raise ValueError("datasets must have one entry per program")
            return 0, hs
        return self._ds(dataset).handle, None

    def prepare(self, programs: PopulationLike, dataset=None, datasets=None, kernel: int = N.KERNEL_AUTO,
                gradient: bool = False) -> "PreparedBatch":
        pk = _packed(programs)
        s, keep = _as_population(pk)
        h, dsp = self._handles(pk.n, dataset, datasets)
        b = C.c_void_p()
        N.check(N.lib().rsr_batch_prepare(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None,
                                          kernel, 1 if gradient else 0, C.byref(b)))
        return PreparedBatch(self, b, pk.n, gradient)

    def last_transfer(self) -> Tuple[int, int]:
        """(host->device, device->host) bytes of the last evaluation call."""
        a, b = C.c_uint64(), C.c_uint64()
        N.check(N.lib().rsr_ctx_last_transfer(self.ctx, C.byref(a), C.byref(b)))
        return a.value, b.value

    def autotune(self, programs: PopulationLike, dataset=None, datasets=None, reps: int = 3) -> dict:
        """Times the register kernel's launch shapes on this population and
        keeps the fastest for later calls on this engine."""
        pk = _packed(programs)
        s, keep = _as_population(pk)
        h, dsp = self._handles(pk.n, dataset, datasets)
        buf = C.create_string_buffer(1 << 16)
        N.check(N.lib().rsr_autotune(self.ctx, C.byref(s), h, dsp.ctypes.data if dsp is not None else None, reps,
                                     buf, len(buf)))
        return json.loads(buf.value.decode())

    def launch_count(self) -> int:
        return int(N.lib().rsr_ctx_launch_count(self.ctx))

    def flush_l2(self) -> None:
        N.check(N.lib().rsr_flush_l2(self.ctx))

    def fp32_peak(self) -> float:
        """Measured unfused FP32 lane-operations per second of this GPU."""
        v = C.c_double()
        N.check(N.lib().rsr_measure_fp32_peak(self.ctx, C.byref(v)))
        return v.value

    def synchronize(self) -> None:
        N.check(N.lib().rsr_synchronize(self.ctx))


class PreparedBatch:
    def __init__(self, engine: Engine, handle, n: int, gradient: bool):
        self.engine, self.handle, self.n, self.gradient = engine, handle, n, gradient

    def run(self) -> None:
        N.check(N.lib().rsr_batch_run(self.engine.ctx, self.handle))

    def results(self):
        mse = np.zeros(self.n, np.float32)
        grad = np.zeros((self.n, 32), np.float32) if self.gradient else None
        N.check(N.lib().rsr_batch_results(self.engine.ctx, self.handle, mse.ctypes.data,
                                          grad.ctypes.data if grad is not None else None))
        return (mse, grad) if self.gradient else mse

    def timing(self) -> Tuple[float, float]:
        e, t = C.c_float(), C.c_float()
        N.check(N.lib().rsr_batch_last_timing(self.engine.ctx, self.handle, C.byref(e), C.byref(t)))
        return e.value, t.value

    def describe(self) -> dict:
        buf = C.create_string_buffer(8192)
        N.check(N.lib().rsr_batch_describe(self.engine.ctx, self.handle, buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self) -> None:
        if self.handle:
            N.lib().rsr_batch_destroy(self.engine.ctx, self.handle)
            self.handle = None


# ------------------------------------------------ module-level drop-ins
_default: Optional[Engine] = None


def default_engine() -> Engine:
    global _default
    if _default is None:
        _default = Engine()
    return _default


def compute_mse(program: Program, dataset) -> float:
    """evaluator::compute_mse (src/engine/eval/evaluator.rs:153-174)."""
    return default_engine().compute_mse(program, dataset)


def compute_mse_with_gradient(program: Program, dataset) -> Tuple[float, np.ndarray]:
    """evaluator::compute_mse_with_gradient (src/engine/eval/evaluator.rs:177-224)."""
    return default_engine().compute_mse_with_gradient(program, dataset)


def validate(program: Program, num_features: int = 0) -> None:
    s, keep = _as_program(program)
    N.check(N.lib().rsr_validate_program(C.byref(s), num_features))


def analyze(program: Program, num_features: int = 0) -> dict:
    s, keep = _as_program(program)
    info = N.ProgramInfo()
    N.check(N.lib().rsr_program_analyze(C.byref(s), num_features, C.byref(info)))
    return {"depth_ref": list(info.depth_ref), "depth_fast": list(info.depth_fast),
            "n_uops_fast": info.n_uops_fast, "n_uops_plain": info.n_uops_plain,
            "fast_profile": info.fast_profile, "flops_per_point": info.flops_per_point}


def encoding(program: Program, num_features: int = 0, form: int = 1) -> np.ndarray:
    """Device encoding of a program (0 slot form, 1 accumulator form, 2 tape
    form; 3 slot form + slot count + flags, 4 the same from the
    no-allocation entry point's fixed-array encoder; 5 register adjoint:
    profile, tape slots, 5 stack depths, then its code)."""
    s, keep = _as_program(program)
    n = C.c_uint32()
    N.check(N.lib().rsr_program_encoding(C.byref(s), num_features, form, None, 0, C.byref(n)))
    out = np.zeros(max(1, n.value), np.uint32)
    N.check(N.lib().rsr_program_encoding(C.byref(s), num_features, form, out.ctypes.data, n.value, C.byref(n)))
    return out[:n.value]

