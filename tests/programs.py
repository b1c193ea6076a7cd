"""Programs and data used by the tests.

Known-answer targets: the closed-form targets of the reference's own tests
(tests/basic.rs:34-173, tests/linalg.rs:44-188), each encoded as a program
whose operation order matches the test's f32 expression, with the tests'
input ranges drawn from a seeded generator.  When every op in the expression
is an IEEE operation (+ - * / sqrt) the reference evaluator reproduces the
target bit for bit, so the program's MSE is exactly 0; for the others
(sin/cos/exp from `wide`, the inverse's reciprocal-multiply) it is tiny.
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

from rsr_b200 import isa as I
from rsr_b200.dataset import Dataset
from rsr_b200.isa import FLOAT, MAT2, MAT3, VEC2, VEC3, Program, Scalar

f32 = np.float32
op = I.op


def cf(v):  # a Float constant load placeholder: resolved by _prog
    return ("C", FLOAT, (v,))


def cv(t, vals):
    return ("C", t, tuple(vals))


def var(t, off):
    return ("V", t, off)


def _prog(items) -> Program:
    code, consts = [], []
    for it in items:
        if isinstance(it, tuple) and it[0] == "C":
            consts.append(Scalar(it[1], it[2]))
            code.append(I.load_const(it[1], len(consts) - 1))
        elif isinstance(it, tuple) and it[0] == "V":
            code.append(I.load_var(it[1], it[2]))
        else:
            code.append(op(it))
    return Program(code, consts)


X0, X1, X2, X3 = (var(FLOAT, i) for i in range(4))


def kat_cases(n: int = 256, seed: int = 100) -> Dict[str, Tuple[Program, Dataset, bool]]:
    """name -> (program, dataset, exact) for the reference tests' targets."""
    rng = np.random.default_rng(seed)
    U = lambda lo, hi, *s: rng.uniform(lo, hi, s).astype(f32)
    out = {}
    # tests/basic.rs:34-45  y = 2.5 x^2 - 1.2
    x = U(-5, 5, n)
    out["basic1"] = (_prog([cf(2.5), X0, "MulF", X0, "MulF", cf(1.2), "SubF"]),
                     Dataset.new(x[:, None], f32(2.5) * x * x - f32(1.2), [FLOAT]), True)
    # tests/basic.rs:47-57  y = 3 cos(2x) + 1
    x = U(-4, 4, n)
    y = (f32(3.0) * np.cos(f32(2.0) * x).astype(f32) + f32(1.0)).astype(f32)
    out["basic2"] = (_prog([cf(3.0), cf(2.0), X0, "MulF", "CosF", "MulF", cf(1.0), "AddF"]),
                     Dataset.new(x[:, None], y, [FLOAT]), False)
    # tests/basic.rs:59-70  y = 1.5 exp(0.5 x)
    x = U(-2, 4, n)
    y = (f32(1.5) * np.exp(f32(0.5) * x).astype(f32)).astype(f32)
    out["basic3"] = (_prog([cf(1.5), cf(0.5), X0, "MulF", "ExpF", "MulF"]), Dataset.new(x[:, None], y, [FLOAT]), False)
    # tests/basic.rs:72-83  y = exp(-0.5 x) cos(3 x)
    x = U(0, 10, n)
    y = (np.exp(f32(-0.5) * x).astype(f32) * np.cos(f32(3.0) * x).astype(f32)).astype(f32)
    out["basic4"] = (_prog([cf(-0.5), X0, "MulF", "ExpF", cf(3.0), X0, "MulF", "CosF", "MulF"]),
                     Dataset.new(x[:, None], y, [FLOAT]), False)
    # tests/basic.rs:85-98  y = 2 x0 - 3.5 x1 + 1.2 x2
    X = U(-5, 5, n, 3)
    y = (f32(2.0) * X[:, 0] - f32(3.5) * X[:, 1]) + f32(1.2) * X[:, 2]
    out["basic5"] = (_prog([cf(2.0), X0, "MulF", cf(3.5), X1, "MulF", "SubF", cf(1.2), X2, "MulF", "AddF"]),
                     Dataset.new(X, y, [FLOAT] * 3), True)
    # tests/basic.rs:100-113  y = x0^2 + sin(x1) - x2
    X = np.stack([U(-3, 3, n), U(-4, 4, n), U(-5, 5, n)], 1)
    y = ((X[:, 0] * X[:, 0] + np.sin(X[:, 1]).astype(f32)) - X[:, 2]).astype(f32)
    out["basic6"] = (_prog([X0, X0, "MulF", X1, "SinF", "AddF", X2, "SubF"]), Dataset.new(X, y, [FLOAT] * 3), False)
    # tests/basic.rs:129-144  y = x0 * x3 over 5 features
    X = U(-5, 5, n, 5)
    out["basic8"] = (_prog([X0, X3, "MulF"]), Dataset.new(X, X[:, 0] * X[:, 3], [FLOAT] * 5), True)
    # tests/basic.rs:146-157  y = (x + 1.5) / (x^2 + 2)
    x = U(-5, 5, n)
    y = ((x + f32(1.5)) / (x * x + f32(2.0))).astype(f32)
    out["basic9"] = (_prog([X0, cf(1.5), "AddF", X0, X0, "MulF", cf(2.0), "AddF", "DivF"]),
                     Dataset.new(x[:, None], y, [FLOAT]), True)
    # tests/basic.rs:159-173  y = exp(-x0) + cos(x1) - x2^2 / (x3 + 1.1)
    X = np.stack([U(-3, 3, n), U(-5, 5, n), U(-5, 5, n), U(0, 5, n)], 1)
    y = ((np.exp(-X[:, 0]).astype(f32) + np.cos(X[:, 1]).astype(f32)) -
         (X[:, 2] * X[:, 2]) / (X[:, 3] + f32(1.1))).astype(f32)
    out["basic10"] = (_prog([cf(0.0), X0, "SubF", "ExpF", X1, "CosF", "AddF", X2, X2, "MulF", X3, cf(1.1), "AddF",
                             "DivF", "SubF"]), Dataset.new(X, y, [FLOAT] * 4), False)
    # tests/linalg.rs:44-71  y = w . (I w), I a constant Mat3 (column-major)
    imat = [2.0, 0.1, 0.0, 0.1, 1.5, -0.2, 0.0, -0.2, 1.0]
    W = U(-5, 5, n, 3)
    iw = [(f32(imat[r]) * W[:, 0] + f32(imat[3 + r]) * W[:, 1]) + f32(imat[6 + r]) * W[:, 2] for r in range(3)]
    y = ((W[:, 0] * iw[0] + W[:, 1] * iw[1]) + W[:, 2] * iw[2]).astype(f32)
    out["linalg1"] = (_prog([var(VEC3, 0), cv(MAT3, imat), var(VEC3, 0), "MulM3V3", "DotV3"]),
                      Dataset.new(W, y, [VEC3]), True)
    # tests/linalg.rs:73-107  y = |E + v x B|
    E_, V_, B_ = U(-5, 5, n, 3), U(-5, 5, n, 3), U(-5, 5, n, 3)
    c = [V_[:, 1] * B_[:, 2] - V_[:, 2] * B_[:, 1], V_[:, 2] * B_[:, 0] - V_[:, 0] * B_[:, 2],
         V_[:, 0] * B_[:, 1] - V_[:, 1] * B_[:, 0]]
    fx = [E_[:, i] + c[i] for i in range(3)]
    y = np.sqrt((fx[0] * fx[0] + fx[1] * fx[1]) + fx[2] * fx[2]).astype(f32)
    out["linalg2"] = (_prog([var(VEC3, 0), var(VEC3, 3), var(VEC3, 6), "CrossV3", "AddV3", "NormV3"]),
                      Dataset.new(np.concatenate([E_, V_, B_], 1), y, [VEC3] * 3), True)
    # tests/linalg.rs:109-142  y = Tr(A^-1 B) + det(A)
    A = np.stack([U(1, 8, n), U(-4, 4, n), U(-1, 1, n), U(1, 8, n)], 1)
    B = np.stack([U(-6, 2, n), U(-2, 6, n), U(-2, 2, n), U(-10, 0, n)], 1)
    det = A[:, 0] * A[:, 3] - A[:, 1] * A[:, 2]
    inv = [A[:, 3] / det, -A[:, 1] / det, -A[:, 2] / det, A[:, 0] / det]
    y = (((inv[0] * B[:, 0] + inv[2] * B[:, 1]) + (inv[1] * B[:, 2] + inv[3] * B[:, 3])) + det).astype(f32)
    out["linalg3"] = (_prog([var(MAT2, 0), "InverseM2", var(MAT2, 4), "MulM2", "TraceM2", var(MAT2, 0), "DetM2",
                             "AddF"]), Dataset.new(np.concatenate([A, B], 1), y, [MAT2, MAT2]), False)
    # tests/linalg.rs:144-188  y = |M v - u|
    M, V_, Uu = U(-5, 5, n, 9), U(-5, 5, n, 3), U(-5, 5, n, 3)
    mv = [(M[:, r] * V_[:, 0] + M[:, 3 + r] * V_[:, 1]) + M[:, 6 + r] * V_[:, 2] for r in range(3)]
    d = [mv[r] - Uu[:, r] for r in range(3)]
    y = np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]).astype(f32)
    out["linalg4"] = (_prog([var(MAT3, 0), var(VEC3, 9), "MulM3V3", var(VEC3, 12), "SubV3", "NormV3"]),
                      Dataset.new(np.concatenate([M, V_, Uu], 1), y, [MAT3, VEC3, VEC3]), True)
    return out


# ---------------------------------------------------------- one op each
_LEAF_OFF = {FLOAT: 0, VEC2: 1, VEC3: 3, MAT2: 6, MAT3: 10}   # feature layout of op_dataset
OP_NUM_FEATURES = 19


def op_dataset(n: int = 200, seed: int = 7, scale: float = 2.0) -> Dataset:
    """Features: F at 0, V2 at 1, V3 at 3, M2 at 6, M3 at 10 (19 floats)."""
    rng = np.random.default_rng(seed)
    X = rng.normal(0, scale, (n, OP_NUM_FEATURES)).astype(f32)
    X[:5] = 0.0            # zero vectors / singular matrices
    X[5, 6:10] = [1, 2, 2, 4]  # singular Mat2
    y = rng.normal(0, 1, n).astype(f32)
    return Dataset.new(X, y, [FLOAT, VEC2, VEC3, MAT2, MAT3])


def single_op_programs() -> Dict[str, Program]:
    """For every operator: its operands as features (or a constant for the
    second operand of the same type), then the op, then a reduction of the
    result to a Float so that stack_f[0] carries it."""
    progs = {}
    to_float = {FLOAT: [], VEC2: ["NormV2"], VEC3: ["NormV3"], MAT2: ["DetM2"], MAT3: ["DetM3"]}
    consts = {FLOAT: (0.75,), VEC2: (0.5, -1.25), VEC3: (0.5, -1.25, 2.0), MAT2: (1.5, -0.5, 0.25, 2.0),
              MAT3: (1.5, -0.5, 0.25, 2.0, 0.75, -1.0, 0.3, 0.1, 1.2)}
    for name in I.BASIC_NAMES + I.LINALG_NAMES:
        args, ret = I.SIGNATURE[name]
        seen = set()
        items = []
        for t in args:
            if t in seen:
                items.append(cv(t, consts[t]))
            else:
                items.append(var(t, _LEAF_OFF[t]))
                seen.add(t)
        items.append(name)
        items += to_float[ret]
        progs[name] = _prog(items)
        # component access of vector/matrix results is covered via Get*/Trace
    return progs
