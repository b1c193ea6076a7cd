"""CPU restatement of the reference's Nelder-Mead constant fitting.

TEST INFRASTRUCTURE ONLY: the checker for ``rsr_fit_nelder_mead``.  It
follows run_nelder_mead (src/engine/optimize/nelder_mead.rs:9-165) step for
step in f32 arithmetic, one program at a time, with a pluggable MSE
evaluation (default: the oracle's f32 restatement of compute_mse).  The
simplex is ordered with a stable sort (ties keep their order); the
reference's sort_unstable_by leaves the order of ties unspecified.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

from rsr_b200.isa import KIND_WIDTH

from . import binding as B

f32 = np.float32
L1 = f32(0.01)                      # nelder_mead.rs:7
ALPHA, GAMMA, RHO, SIGMA = f32(1.0), f32(2.0), f32(0.5), f32(0.5)
FLOAT_KIND = 0


def _key(v):
    fit = v[0]
    return (1, 0.0) if np.isnan(fit) else (0, float(fit))


def run_nelder_mead(program, dataset, max_iterations: int, mse_fn: Callable = None):
    """Returns (flat params after fitting, best mse, counters); the program is
    left at the fitted constants.  Programs without Float constants are left
    alone and report their starting MSE."""
    mse_fn = mse_fn or (lambda p: f32(B.mse_ref32(p, dataset)))
    stats = {"iterations": 0, "mse_evaluations": 0}
    flat = program.flatten_params().astype(f32)
    opt, off = [], 0
    for c in program.constants:
        if c.kind == FLOAT_KIND and len(opt) < 32:
            opt.append(off)
        off += KIND_WIDTH[c.kind]
    n = len(opt)

    def evaluate(vals):
        buf = flat.copy()
        for j in range(n):
            buf[opt[j]] = vals[j]
        program.unflatten_params(buf)
        m = f32(mse_fn(program))
        stats["mse_evaluations"] += 1
        l1 = f32(0)
        for j in range(n):
            l1 = f32(l1 + f32(abs(vals[j])))
        return f32(m + f32(L1 * l1)), m

    start = np.zeros(32, f32)
    for j in range(n):
        start[j] = flat[opt[j]]
    fit0, mse0 = evaluate(start)
    if n == 0:
        return flat, float(mse0), stats
    simplex = [(fit0, mse0, start.copy())]
    for i in range(n):
        p = start.copy()
        val = p[i]
        p[i] = f32(p[i] + (f32(0.01) if abs(val) < f32(1e-4) else f32(val * f32(0.10))))
        f, m = evaluate(p)
        simplex.append((f, m, p))
    for _ in range(max_iterations):
        simplex.sort(key=_key)
        best_fit, best_mse, worst_fit = simplex[0][0], simplex[0][1], simplex[n][0]
        if abs(f32(worst_fit - best_fit)) < f32(1e-7) or best_mse < f32(1e-8):
            break
        stats["iterations"] += 1
        centroid = np.zeros(32, f32)
        for v in simplex[:n]:
            for j in range(n):
                centroid[j] = f32(centroid[j] + v[2][j])
        for j in range(n):
            centroid[j] = f32(centroid[j] / f32(n))
        worst = simplex[n][2]
        second_worst = simplex[n - 1][0]
        refl = np.zeros(32, f32)
        for j in range(n):
            refl[j] = f32(centroid[j] + f32(ALPHA * f32(centroid[j] - worst[j])))
        rfit, rmse = evaluate(refl)
        if rfit >= best_fit and rfit < second_worst:
            simplex[n] = (rfit, rmse, refl)
            continue
        if rfit < best_fit:
            exp = np.zeros(32, f32)
            for j in range(n):
                exp[j] = f32(centroid[j] + f32(GAMMA * f32(refl[j] - centroid[j])))
            efit, emse = evaluate(exp)
            simplex[n] = (efit, emse, exp) if efit < rfit else (rfit, rmse, refl)
            continue
        con = np.zeros(32, f32)
        if rfit < worst_fit:
            for j in range(n):
                con[j] = f32(centroid[j] + f32(RHO * f32(refl[j] - centroid[j])))
            limit = rfit
        else:
            for j in range(n):
                con[j] = f32(centroid[j] + f32(RHO * f32(worst[j] - centroid[j])))
            limit = worst_fit
        cfit, cmse = evaluate(con)
        if cfit < limit:
            simplex[n] = (cfit, cmse, con)
            continue
        best = simplex[0][2].copy()
        for k in range(1, n + 1):
            x = simplex[k][2].copy()
            for j in range(n):
                x[j] = f32(best[j] + f32(SIGMA * f32(x[j] - best[j])))
            f, m = evaluate(x)
            simplex[k] = (f, m, x)
    simplex.sort(key=_key)
    out = flat.copy()
    for j in range(n):
        out[opt[j]] = simplex[0][2][j]
    program.unflatten_params(out)
    return out, float(simplex[0][1]), stats
