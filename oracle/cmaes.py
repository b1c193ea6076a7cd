"""CPU restatement of the reference's CMA-ES constant fitting.

TEST INFRASTRUCTURE ONLY: the checker for ``rsr_fit_cma_es``.  It follows
run_cma_es (src/engine/optimize/cmaes.rs:19-192) step for step in f32
arithmetic, one program at a time, with a pluggable MSE evaluation (default:
the oracle's f32 restatement of compute_mse).  Two inputs replace what the
reference leaves open:

* random numbers: the reference draws from rand::rng() (unseeded); here
  program ``index`` of a batch draws from the splitmix64 stream seeded with
  ``seed ^ (0xD1B54A32D192ED03 * (index + 1))``, 24-bit uniforms, and the
  reference's Box-Muller normal (cmaes.rs:13-17) with the C library's logf
  and cosf (the functions the engine's host code calls);
* ties: the candidates are ordered with a stable sort (the reference's
  sort_unstable_by leaves the order of ties open).

The search vector is the flat parameters followed by a copy of them, as the
reference builds it (cmaes.rs:27-75).
"""
from __future__ import annotations

import ctypes
import ctypes.util
from typing import Callable

import numpy as np

from . import binding as B

f32 = np.float32
MAX_PARAMS, LAMBDA = 32, 16     # cmaes.rs:8-9
MU = LAMBDA // 2
L1 = f32(0.01)                  # cmaes.rs:11
SIGMA_DECAY = f32(float.fromhex("0x1.fae7dp-1"))  # exp(-0.01) rounded to f32, cmaes.rs:176
MASK = (1 << 64) - 1

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
for _fn in ("logf", "cosf", "sqrtf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]


def logf(x) -> np.float32:
    return f32(_libm.logf(float(x)))


def cosf(x) -> np.float32:
    return f32(_libm.cosf(float(x)))


def sqrtf(x) -> np.float32:
    return f32(_libm.sqrtf(float(x)))


class SplitMix:
    def __init__(self, state: int):
        self.s = state & MASK

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> np.float32:
        return f32(f32(self.next() >> 40) * f32(1.0 / 16777216.0))

    def normal(self) -> np.float32:
        u1 = max(self.uniform(), f32(1e-8))
        u2 = self.uniform()
        return f32(sqrtf(f32(f32(-2.0) * logf(u1))) * cosf(f32(f32(f32(2.0) * f32(3.14159265358979)) * u2)))


def stream_seed(seed: int, index: int) -> int:
    return (seed ^ ((0xD1B54A32D192ED03 * (index + 1)) & MASK)) & MASK


def run_cma_es(program, dataset, max_iterations: int, seed: int = 0, index: int = 0,
               mse_fn: Callable = None):
    """Returns (flat params after fitting, best mse, counters); the program is
    left at the fitted parameters."""
    mse_fn = mse_fn or (lambda p: f32(B.mse_ref32(p, dataset)))
    stats = {"iterations": 0, "mse_evaluations": 0}
    flat = program.flatten_params().astype(f32)
    pc = min(len(flat), MAX_PARAMS)

    def evaluate(x):
        buf = flat.copy()
        buf[:pc] = x[:pc]
        program.unflatten_params(buf)
        stats["mse_evaluations"] += 1
        return f32(mse_fn(program))

    mean = np.zeros(MAX_PARAMS, f32)
    mean[:pc] = flat[:pc]
    n = pc
    for j in range(pc):
        if n < MAX_PARAMS:
            mean[n] = flat[j]
            n += 1
    if pc == 0:
        return flat, float(evaluate(mean)), stats
    rng = SplitMix(stream_seed(seed, index))
    sigma = f32(0.5)
    c_diag = np.ones(MAX_PARAMS, f32)
    p_c = np.zeros(MAX_PARAMS, f32)
    w = np.zeros(MU, f32)
    sw = f32(0)
    for i in range(MU):  # the two logarithms rounded to f32
        w[i] = max(f32(f32(np.log(float(f32(f32(MU) + f32(0.5))))) - f32(np.log(float(i + 1)))), f32(0))
        sw = f32(sw + w[i])
    mu_eff = f32(0)
    for i in range(MU):
        w[i] = f32(w[i] / sw)
        mu_eff = f32(mu_eff + f32(w[i] * w[i]))
    mu_eff = f32(f32(1) / mu_eff)
    fn = f32(n)
    c_c = f32(f32(f32(4) + f32(mu_eff / fn)) / f32(f32(fn + f32(4)) + f32(f32(f32(2) * mu_eff) / fn)))
    a, b = f32(fn + f32(1.414)), f32(fn + f32(2))
    c_cov = f32(f32(f32(f32(1) / mu_eff) * f32(f32(2) / f32(a * a))) +
                f32(f32(f32(1) - f32(f32(1) / mu_eff)) * f32(f32(f32(f32(2) * mu_eff) - f32(1)) / f32(f32(b * b) + mu_eff))))

    best_mse = evaluate(mean)
    l1 = f32(0)
    for j in range(n):
        l1 = f32(l1 + abs(mean[j]))
    best_fit = f32(best_mse + f32(L1 * l1))
    best_point = mean.copy()
    pop = np.zeros((LAMBDA, MAX_PARAMS), f32)
    step = np.zeros((LAMBDA, MAX_PARAMS), f32)
    for _ in range(max_iterations):
        stats["iterations"] += 1
        fits = []
        for r in range(LAMBDA):
            l1 = f32(0)
            for j in range(n):
                z = f32(rng.normal() * sqrtf(c_diag[j]))
                step[r, j] = z
                pop[r, j] = f32(mean[j] + f32(sigma * z))
                l1 = f32(l1 + abs(pop[r, j]))
            m = evaluate(pop[r])
            fits.append((f32(m + f32(L1 * l1)), m, r))
        order = sorted(fits, key=lambda t: (1, 0.0) if np.isnan(t[0]) else (0, float(t[0])))
        if order[0][0] < best_fit:
            best_fit, best_mse = order[0][0], order[0][1]
            best_point = pop[order[0][2]].copy()
        if best_mse < f32(1e-8):
            break
        step_mean = np.zeros(MAX_PARAMS, f32)
        old = mean.copy()
        for k in range(MU):
            r = order[k][2]
            for j in range(n):
                step_mean[j] = f32(step_mean[j] + f32(w[k] * step[r, j]))
                mean[j] = f32(mean[j] + f32(w[k] * f32(pop[r, j] - old[j])))
        path = sqrtf(f32(f32(c_c * f32(f32(2) - c_c)) * mu_eff))
        for j in range(n):
            p_c[j] = f32(f32(f32(f32(1) - c_c) * p_c[j]) + f32(path * step_mean[j]))
            cov = f32(0)
            for k in range(MU):
                r = order[k][2]
                cov = f32(cov + f32(w[k] * f32(step[r, j] * step[r, j])))
            c = f32(f32(f32(f32(1) - c_cov) * c_diag[j]) + f32(f32(c_cov / mu_eff) * f32(p_c[j] * p_c[j])))
            c = f32(c + f32(f32(c_cov * f32(f32(1) - f32(f32(1) / mu_eff))) * cov))
            c_diag[j] = min(max(c, f32(1e-6)), f32(1e6))
        sigma = f32(sigma * SIGMA_DECAY)
    out = flat.copy()
    out[:pc] = best_point[:pc]
    program.unflatten_params(out)
    return out, float(best_mse), stats
