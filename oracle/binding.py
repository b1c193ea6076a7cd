"""ctypes binding of the C oracle (oracle/rsr_oracle.c, oracle/simd_baseline.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
baseline.  Built by ``make -C oracle`` into oracle/_build/liboracle.so.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None

u32p, u8p, f32p, f64p, u64p = (C.POINTER(t) for t in (C.c_uint32, C.c_uint8, C.c_float, C.c_double, C.c_uint64))
PROG = [u32p, C.c_uint32, u8p, C.c_uint32, f32p, C.c_uint32]
DS = [f32p, f32p, C.c_uint32, C.c_uint64, C.c_uint64]


def build() -> Path:
    srcs = [HERE / "rsr_oracle.c", HERE / "simd_baseline.c", HERE / "Makefile"]
    if not LIB.exists() or LIB.stat().st_mtime < max(s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        for fn in ("orc_sinf", "orc_cosf", "orc_expf", "orc_logf"):
            getattr(L, fn).restype = C.c_float
            getattr(L, fn).argtypes = [C.c_float]
        L.orc_n_opcodes.restype = C.c_int
        L.orc_validate.restype = C.c_int
        L.orc_validate.argtypes = [u32p, C.c_uint32, u8p, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_eval_points.restype = None
        L.orc_eval_points.argtypes = PROG + [f32p, C.c_uint32, C.c_uint64, f32p]
        L.orc_mse_ref32.restype = C.c_float
        L.orc_mse_ref32.argtypes = PROG + DS
        L.orc_mse_f64.restype = C.c_double
        L.orc_mse_f64.argtypes = PROG + DS
        L.orc_mse_grad_dual.restype = C.c_float
        L.orc_mse_grad_dual.argtypes = PROG + DS + [f32p]
        L.orc_grad_dual_f64.restype = C.c_double
        L.orc_grad_dual_f64.argtypes = PROG + DS + [f64p, f64p]
        L.orc_grad_fd.restype = None
        L.orc_grad_fd.argtypes = PROG + DS + [C.c_double, f64p]
        L.orc_mse_batch.restype = None
        L.orc_mse_batch.argtypes = [u32p, u64p, u8p, u64p, f32p, u64p, C.c_uint32, f32p, f32p, C.c_uint32,
                                    C.c_uint64, C.c_uint64, C.c_int, f64p, f32p]
        L.simd_mse_batch.restype = None
        L.simd_mse_batch.argtypes = [u32p, u64p, u8p, u64p, f32p, u64p, C.c_uint32, f32p, f32p, C.c_uint32,
                                     C.c_uint64, C.c_uint64, C.c_int, f32p]
        L.simd_transcendental.restype = None
        L.simd_transcendental.argtypes = [C.c_int, f32p, f32p, C.c_uint64]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _prog(p):
    code = np.ascontiguousarray(p.code_array(), np.uint32)
    kinds = np.ascontiguousarray(p.kinds(), np.uint8)
    params = np.ascontiguousarray(p.flatten_params(), np.float32)
    if len(params) == 0:
        params = np.zeros(1, np.float32)
        n = 0
    else:
        n = len(params)
    if len(kinds) == 0:
        kinds_arr = np.zeros(1, np.uint8)
    else:
        kinds_arr = kinds
    keep = (code, kinds_arr, params)
    return [_p(code, u32p), len(code), _p(kinds_arr, u8p), len(kinds), _p(params, f32p), n], keep


def _ds(ds):
    ff = np.ascontiguousarray(ds.feature_flat, np.float32)
    tb = np.ascontiguousarray(ds.target_batches, np.float32)
    return [_p(ff, f32p), _p(tb, f32p), ds.num_features, ds.num_batches], (ff, tb)


def eval_points(p, ds) -> np.ndarray:
    a, k = _prog(p)
    ff = np.ascontiguousarray(ds.feature_flat, np.float32)
    out = np.zeros(ds.num_batches * 8, np.float32)
    lib().orc_eval_points(*a, _p(ff, f32p), ds.num_features, ds.num_batches, _p(out, f32p))
    return out


def mse_ref32(p, ds) -> float:
    a, k = _prog(p)
    d, k2 = _ds(ds)
    return float(lib().orc_mse_ref32(*a, *d, ds.num_samples))


def mse_f64(p, ds) -> float:
    a, k = _prog(p)
    d, k2 = _ds(ds)
    return float(lib().orc_mse_f64(*a, *d, ds.num_samples))


def sse_f64(p, ds) -> float:
    """Unscaled FP64 sum of squared errors over every padded point."""
    a, k = _prog(p)
    d, k2 = _ds(ds)
    return float(lib().orc_mse_f64(*a, *d, 1))


def mse_grad_dual(p, ds):
    a, k = _prog(p)
    d, k2 = _ds(ds)
    g = np.zeros(32, np.float32)
    m = lib().orc_mse_grad_dual(*a, *d, ds.num_samples, _p(g, f32p))
    return float(m), g


def grad_dual_f64(p, ds):
    """(f64 MSE, gradient, per-component L1 scale): the reference's dual
    rules per point, sums over points in f64 (orc_grad_dual_f64)."""
    a, k = _prog(p)
    d, k2 = _ds(ds)
    g = np.zeros(32, np.float64)
    l1 = np.zeros(32, np.float64)
    m = lib().orc_grad_dual_f64(*a, *d, ds.num_samples, _p(g, f64p), _p(l1, f64p))
    return float(m), g, l1


def grad_fd(p, ds, h: float = 1e-3) -> np.ndarray:
    a, k = _prog(p)
    d, k2 = _ds(ds)
    g = np.zeros(max(1, p.param_count()), np.float64)
    lib().orc_grad_fd(*a, *d, ds.num_samples, h, _p(g, f64p))
    return g[:p.param_count()]


def _packed(pk):
    arrs = [np.ascontiguousarray(pk.code, np.uint32), np.ascontiguousarray(pk.code_off, np.uint64),
            np.ascontiguousarray(pk.kinds if len(pk.kinds) else np.zeros(1, np.uint8), np.uint8),
            np.ascontiguousarray(pk.kind_off, np.uint64),
            np.ascontiguousarray(pk.params if len(pk.params) else np.zeros(1, np.float32), np.float32),
            np.ascontiguousarray(pk.param_off, np.uint64)]
    ptrs = [_p(arrs[0], u32p), _p(arrs[1], u64p), _p(arrs[2], u8p), _p(arrs[3], u64p), _p(arrs[4], f32p),
            _p(arrs[5], u64p)]
    return ptrs, arrs


def mse_batch(pk, ds, threads: int = 0):
    """(FP64-oracle MSE, reference-order f32 MSE) for every program."""
    ptrs, keep = _packed(pk)
    d, k2 = _ds(ds)
    m64 = np.zeros(pk.n, np.float64)
    m32 = np.zeros(pk.n, np.float32)
    lib().orc_mse_batch(*ptrs, pk.n, d[0], d[1], ds.num_features, ds.num_batches, ds.num_samples,
                        threads or os.cpu_count() or 1, _p(m64, f64p), _p(m32, f32p))
    return m64, m32


def simd_mse_batch(pk, ds, threads: int = 0) -> np.ndarray:
    """The timed CPU baseline: 8-lane AVX2 restatement of compute_mse."""
    ptrs, keep = _packed(pk)
    ff = np.empty(ds.feature_flat.size + 8, np.float32)  # 32-byte aligned copy
    off = (-ff.ctypes.data % 32) // 4
    ffa = ff[off:off + ds.feature_flat.size]
    ffa[:] = ds.feature_flat
    tb = np.ascontiguousarray(ds.target_batches, np.float32)
    out = np.zeros(pk.n, np.float32)
    lib().simd_mse_batch(*ptrs, pk.n, _p(ffa, f32p), _p(tb, f32p), ds.num_features, ds.num_batches, ds.num_samples,
                         threads or os.cpu_count() or 1, _p(out, f32p))
    return out


def transcendental(which: str, x: np.ndarray, simd: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    if simd:
        n8 = len(x) // 8 * 8
        y = np.zeros(n8, np.float32)
        lib().simd_transcendental({"sin": 0, "cos": 1, "exp": 2, "log": 3}[which], _p(x, f32p), _p(y, f32p), n8)
        return y
    f = getattr(lib(), {"sin": "orc_sinf", "cos": "orc_cosf", "exp": "orc_expf", "log": "orc_logf"}[which])
    return np.array([f(float(v)) for v in x], np.float32)


def validate(p, num_features: int) -> int:
    a, k = _prog(p)
    return int(lib().orc_validate(a[0], a[1], a[2], a[3], p.param_count(), num_features))
