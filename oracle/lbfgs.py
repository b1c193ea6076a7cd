"""CPU restatement of the reference's L-BFGS constant fitting.

TEST INFRASTRUCTURE ONLY: the checker for ``rsr_fit_lbfgs``.  It follows
run_lbfgs (src/engine/optimize/lbfgs.rs:9-165) step for step in f32
arithmetic (every intermediate is an ``np.float32``, accumulated in the
reference's loop order), one program at a time.  The two evaluations are
pluggable so that the same control flow can be driven by the oracle's own
f32 evaluator (``orc_mse_ref32`` / ``orc_mse_grad_dual``, the restatement of
evaluator.rs) or by any other (mse, gradient) source.
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np

from . import binding as B

f32 = np.float32
MAX_PARAMS = 32   # lbfgs.rs:6
M = 6             # lbfgs.rs:7


def run_lbfgs(program, dataset, max_iterations: int,
              mse_fn: Callable = None, grad_fn: Callable = None) -> Tuple[np.ndarray, float, dict]:
    """Returns (flat params after fitting, final mse, counters).  ``program``
    is an rsr_b200.isa.Program; it is left at the fitted parameters, as the
    reference leaves the individual's program (lbfgs.rs:154).  With no
    parameters nothing runs and the mse is None (lbfgs.rs:18-21)."""
    mse_fn = mse_fn or (lambda p: f32(B.mse_ref32(p, dataset)))
    grad_fn = grad_fn or (lambda p: _dual(p, dataset))
    stats = {"iterations": 0, "gradient_evaluations": 0, "mse_evaluations": 0}
    flat = program.flatten_params().astype(f32)
    n = min(len(flat), MAX_PARAMS)
    if n == 0:
        return flat, None, stats
    x = np.zeros(MAX_PARAMS, f32)
    x[:n] = flat[:n]
    s = np.zeros((M, MAX_PARAMS), f32)
    y = np.zeros((M, MAX_PARAMS), f32)
    rho = np.zeros(M, f32)
    alpha = np.zeros(M, f32)

    def set_params(v):
        buf = flat.copy()
        buf[:n] = v[:n]
        program.unflatten_params(buf)

    cur_mse, cur_grad = grad_fn(program)
    stats["gradient_evaluations"] += 1
    history = 0
    head = 0
    for _ in range(max_iterations):
        gn = f32(0)
        for k in range(n):
            gn = f32(gn + f32(cur_grad[k] * cur_grad[k]))
        if np.sqrt(gn, dtype=f32) < f32(1e-5):
            break
        stats["iterations"] += 1
        q = np.zeros(MAX_PARAMS, f32)
        q[:n] = cur_grad[:n]
        cur = head
        for _h in range(history):
            cur = M - 1 if cur == 0 else cur - 1
            d = f32(0)
            for j in range(n):
                d = f32(d + f32(s[cur, j] * q[j]))
            alpha[cur] = f32(rho[cur] * d)
            for j in range(n):
                q[j] = f32(q[j] - f32(alpha[cur] * y[cur, j]))
        gamma = f32(1)
        if history > 0:
            last = M - 1 if head == 0 else head - 1
            sy = f32(0)
            yy = f32(0)
            for j in range(n):
                sy = f32(sy + f32(s[last, j] * y[last, j]))
                yy = f32(yy + f32(y[last, j] * y[last, j]))
            if yy > f32(1e-10):
                gamma = f32(sy / yy)
        for k in range(n):
            q[k] = f32(q[k] * gamma)
        cur = 0 if history < M else head
        for _h in range(history):
            d = f32(0)
            for j in range(n):
                d = f32(d + f32(y[cur, j] * q[j]))
            beta = f32(rho[cur] * d)
            for j in range(n):
                q[j] = f32(q[j] + f32(s[cur, j] * f32(alpha[cur] - beta)))
            cur = (cur + 1) % M
        p = np.zeros(MAX_PARAMS, f32)
        dd = f32(0)
        for j in range(n):
            p[j] = -q[j]
            dd = f32(dd + f32(p[j] * cur_grad[j]))
        if dd > f32(-1e-8):
            for j in range(n):
                p[j] = -cur_grad[j]
            dd = -gn
            history = 0
        step = f32(1)
        c1 = f32(1e-4)
        nx = np.zeros(MAX_PARAMS, f32)
        ls = 0
        while True:
            for j in range(n):
                nx[j] = f32(x[j] + f32(step * p[j]))
            set_params(nx)
            m = f32(mse_fn(program))
            stats["mse_evaluations"] += 1
            if m <= f32(cur_mse + f32(f32(c1 * step) * dd)) or ls > 10:
                next_mse = m
                break
            step = f32(step * f32(0.5))
            ls += 1
        _, next_grad = grad_fn(program)
        stats["gradient_evaluations"] += 1
        sn = np.zeros(MAX_PARAMS, f32)
        yn = np.zeros(MAX_PARAMS, f32)
        sy = f32(0)
        for j in range(n):
            sn[j] = f32(nx[j] - x[j])
            yn[j] = f32(next_grad[j] - cur_grad[j])
            sy = f32(sy + f32(sn[j] * yn[j]))
        if sy > f32(1e-10):
            s[head, :n] = sn[:n]
            y[head, :n] = yn[:n]
            rho[head] = f32(f32(1) / sy)
            head = (head + 1) % M
            if history < M:
                history += 1
        x[:n] = nx[:n]
        cur_mse = next_mse
        cur_grad = np.asarray(next_grad, f32)
    set_params(x)
    out = flat.copy()
    out[:n] = x[:n]
    return out, float(cur_mse), stats


def _dual(p, ds):
    m, g = B.mse_grad_dual(p, ds)
    return f32(m), np.asarray(g, f32)
