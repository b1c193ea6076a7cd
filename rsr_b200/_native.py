"""ctypes binding of librsrgpu.so (include/rsr_gpu.h).

The library is built in-tree by ``rsr_b200/csrc/build.py`` (``__graft_entry__.build()``).
Nothing here falls back to a CPU implementation: if the library is missing or
no sm_100 device is present, the calls raise.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librsrgpu.so"

RSR_OK, RSR_EINVAL, RSR_EPROGRAM, RSR_ENOMEM, RSR_ENODEV, RSR_ECUDA, RSR_ETIMEDOUT, RSR_ENOTFOUND, RSR_EBUSY, \
    RSR_ECANCELED = range(10)
STATUS_NAMES = ["OK", "EINVAL", "EPROGRAM", "ENOMEM", "ENODEV", "ECUDA", "ETIMEDOUT", "ENOTFOUND", "EBUSY",
                "ECANCELED"]
KERNEL_AUTO, KERNEL_PLAIN, KERNEL_BATCHED = 0, 1, 2
OPT_NO_LOAD_FUSION = 1
OPT_SLOT_ADJOINT = 2


class RsrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        self.code = code
        name = STATUS_NAMES[code] if 0 <= code < len(STATUS_NAMES) else str(code)
        super().__init__(f"rsr {name}: {msg}")


class Program(C.Structure):
    _fields_ = [("code", C.POINTER(C.c_uint32)), ("len", C.c_uint32), ("const_kinds", C.POINTER(C.c_uint8)),
                ("n_consts", C.c_uint32), ("params", C.POINTER(C.c_float)), ("n_params", C.c_uint32)]


class Population(C.Structure):
    _fields_ = [("n_programs", C.c_uint32), ("code", C.POINTER(C.c_uint32)), ("code_off", C.POINTER(C.c_uint64)),
                ("const_kinds", C.POINTER(C.c_uint8)), ("kind_off", C.POINTER(C.c_uint64)),
                ("params", C.POINTER(C.c_float)), ("param_off", C.POINTER(C.c_uint64))]


class Options(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("kernel", C.c_int32), ("points_per_thread", C.c_int32),
                ("programs_per_warp", C.c_int32), ("use_graphs", C.c_int32), ("mem_budget_bytes", C.c_uint64),
                ("tune_cache_path", C.c_char_p), ("flags", C.c_uint32)]


class FitStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("gradient_evaluations", C.c_uint32), ("mse_evaluations", C.c_uint32)]


JOB_MSE, JOB_MSE_GRAD, JOB_FIT, JOB_FIT_AUTO = 0, 1, 2, 3
JOB_QUEUED, JOB_RUNNING, JOB_DONE = 0, 1, 2


class ServerOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("slots", C.c_uint32), ("max_batch_programs", C.c_uint32),
                ("max_queue", C.c_uint32), ("mem_budget_bytes", C.c_uint64)]


class Job(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("fit_iterations", C.c_uint32), ("pop", C.POINTER(Population)),
                ("ds", C.c_uint64), ("ds_per_program", C.POINTER(C.c_uint64)), ("mse_out", C.POINTER(C.c_float)),
                ("grad_out", C.POINTER(C.c_float)), ("params_out", C.POINTER(C.c_float)), ("seed", C.c_uint64)]


class JobInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_jobs", C.c_uint32), ("queue_ms", C.c_double),
                ("latency_ms", C.c_double)]


class ServingStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("cancelled", C.c_uint64), ("refused", C.c_uint64), ("launches", C.c_uint64),
                ("peak_mem_bytes", C.c_uint64), ("p50_ms", C.c_double), ("p95_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("program_points_per_sec", C.c_double), ("wall_s", C.c_double)]


class ProgramInfo(C.Structure):
    _fields_ = [("depth_ref", C.c_uint32 * 5), ("depth_fast", C.c_uint32 * 5), ("n_uops_fast", C.c_uint32),
                ("n_uops_plain", C.c_uint32), ("fast_profile", C.c_int32), ("flops_per_point", C.c_uint32)]


_lib = None

_SIGS = {
    "rsr_options_default": (None, [C.POINTER(Options)]),
    "rsr_ctx_create": (C.c_int, [C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "rsr_ctx_destroy": (C.c_int, [C.c_void_p]),
    "rsr_last_error": (C.c_char_p, []),
    "rsr_version": (C.c_char_p, []),
    "rsr_dataset_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64,
                                     C.POINTER(C.c_uint64)]),
    "rsr_dataset_upload_columns": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                             C.POINTER(C.c_uint64)]),
    "rsr_dataset_release": (C.c_int, [C.c_void_p, C.c_uint64]),
    "rsr_dataset_info": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64)]),
    "rsr_compute_mse": (C.c_int, [C.c_void_p, C.POINTER(Program), C.c_uint64, C.POINTER(C.c_float)]),
    "rsr_compute_mse_with_gradient": (C.c_int, [C.c_void_p, C.POINTER(Program), C.c_uint64, C.POINTER(C.c_float),
                                                C.c_void_p]),
    "rsr_eval_points": (C.c_int, [C.c_void_p, C.POINTER(Program), C.c_uint64, C.c_void_p]),
    "rsr_eval_mse_batch": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_int,
                                     C.c_void_p]),
    "rsr_eval_mse_grad_batch": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    "rsr_eval_points_batch": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_int, C.c_void_p]),
    "rsr_server_options_default": (None, [C.POINTER(ServerOptions)]),
    "rsr_server_create": (C.c_int, [C.c_void_p, C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "rsr_server_destroy": (C.c_int, [C.c_void_p]),
    "rsr_submit": (C.c_int, [C.c_void_p, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "rsr_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint32)]),
    "rsr_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(JobInfo)]),
    "rsr_cancel": (C.c_int, [C.c_void_p, C.c_uint64]),
    "rsr_server_stats": (C.c_int, [C.c_void_p, C.POINTER(ServingStats), C.c_int]),
    "rsr_eval_sums_batch": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_int,
                                      C.c_void_p]),
    "rsr_finalize_sums": (C.c_int, [C.c_uint32, C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "rsr_compute_mse_noalloc": (C.c_int, [C.c_void_p, C.POINTER(Program), C.c_uint64, C.POINTER(C.c_float)]),
    "rsr_dataset_upload_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_int,
                                          C.c_void_p, C.POINTER(C.c_uint64)]),
    "rsr_dataset_subset": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
    "rsr_dataset_download": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "rsr_fit_nelder_mead": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_uint32,
                                      C.c_void_p, C.c_void_p, C.POINTER(FitStats)]),
    "rsr_fit_lbfgs": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p,
                                C.c_void_p, C.POINTER(FitStats)]),
    "rsr_fit_cma_es": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint64,
                                 C.c_void_p, C.c_void_p, C.POINTER(FitStats)]),
    "rsr_batch_prepare": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_int, C.c_int,
                                    C.POINTER(C.c_void_p)]),
    "rsr_batch_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rsr_batch_results": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "rsr_batch_last_timing": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "rsr_batch_describe": (C.c_int, [C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t]),
    "rsr_batch_destroy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rsr_ctx_launch_count": (C.c_uint64, [C.c_void_p]),
    "rsr_ctx_last_transfer": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "rsr_flush_l2": (C.c_int, [C.c_void_p]),
    "rsr_autotune": (C.c_int, [C.c_void_p, C.POINTER(Population), C.c_uint64, C.c_void_p, C.c_int, C.c_char_p,
                               C.c_size_t]),
    "rsr_synchronize": (C.c_int, [C.c_void_p]),
    "rsr_measure_fp32_peak": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "rsr_validate_program": (C.c_int, [C.POINTER(Program), C.c_uint32]),
    "rsr_program_analyze": (C.c_int, [C.POINTER(Program), C.c_uint32, C.POINTER(ProgramInfo)]),
    "rsr_program_encoding": (C.c_int, [C.POINTER(Program), C.c_uint32, C.c_int, C.c_void_p, C.c_uint32,
                                       C.POINTER(C.c_uint32)]),
}


def lib() -> C.CDLL:
    """Loads librsrgpu.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (nvcc, sm_100a) first")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != RSR_OK:
        raise RsrError(rc, lib().rsr_last_error().decode(errors="replace"))


def exported_symbols():
    return list(_SIGS)
