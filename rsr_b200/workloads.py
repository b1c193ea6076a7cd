"""Seeded synthetic workloads: the datasets and populations of the engine's
benchmark configurations.

The reference draws its test data unseeded (tests/basic.rs, tests/linalg.rs);
here every array comes from a seeded numpy generator with the distributions
and target formulas of those tests, the targets computed in f32 in the same
operation order as the tests compute them.

  scalar   y = 2.5 x^2 - 1.2, x ~ U(-3, 3)                (tests/basic.rs:34-45)
  lorentz  y = |E + v x B|, E, v, B ~ N(0, 1)               (tests/linalg.rs:74-107)
  transform y = |M v - u|, M ~ U(-1, 1), v, u ~ N(0, 1)     (tests/linalg.rs:145-188)
  inverse  y = Tr(A^-1 B) + det(A), A = 2I + U(-.5, .5)     (tests/linalg.rs:110-142)
"""
from __future__ import annotations

from typing import List

import numpy as np

from .dataset import Dataset
from .generator import NEG, Generator, OpSet
from .isa import FLOAT, MAT2, MAT3, VEC3, Program

f32 = np.float32


def scalar_dataset(n: int = 400, seed: int = 1) -> Dataset:
    rng = np.random.default_rng(seed)
    x = rng.uniform(-3.0, 3.0, n).astype(f32)
    y = (f32(2.5) * x * x - f32(1.2)).astype(f32)
    return Dataset.new(x[:, None], y, [FLOAT])


def lorentz_dataset(n: int = 100_000, seed: int = 2) -> Dataset:
    rng = np.random.default_rng(seed)
    e, v, b = (rng.standard_normal((n, 3)).astype(f32) for _ in range(3))
    cx = v[:, 1] * b[:, 2] - v[:, 2] * b[:, 1]
    cy = v[:, 2] * b[:, 0] - v[:, 0] * b[:, 2]
    cz = v[:, 0] * b[:, 1] - v[:, 1] * b[:, 0]
    fx, fy, fz = e[:, 0] + cx, e[:, 1] + cy, e[:, 2] + cz
    y = np.sqrt((fx * fx + fy * fy) + fz * fz).astype(f32)
    return Dataset.new(np.concatenate([e, v, b], 1), y, [VEC3, VEC3, VEC3])


def transform_dataset(n: int = 1_000_000, seed: int = 3) -> Dataset:
    rng = np.random.default_rng(seed)
    m = rng.uniform(-1.0, 1.0, (n, 9)).astype(f32)      # column-major Mat3
    v = rng.standard_normal((n, 3)).astype(f32)
    u = rng.standard_normal((n, 3)).astype(f32)
    mv = [(m[:, r] * v[:, 0] + m[:, 3 + r] * v[:, 1]) + m[:, 6 + r] * v[:, 2] for r in range(3)]
    d = [mv[r] - u[:, r] for r in range(3)]
    y = np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]).astype(f32)
    return Dataset.new(np.concatenate([m, v, u], 1), y, [MAT3, VEC3, VEC3])


def inverse_dataset(n: int, seed: int) -> Dataset:
    rng = np.random.default_rng(seed)
    a = (np.array([2, 0, 0, 2], f32) + rng.uniform(-0.5, 0.5, (n, 4))).astype(f32)  # column-major Mat2
    b = rng.standard_normal((n, 4)).astype(f32)
    det = a[:, 0] * a[:, 3] - a[:, 1] * a[:, 2]
    inv = [a[:, 3] / det, -a[:, 1] / det, -a[:, 2] / det, a[:, 0] / det]
    ab0 = inv[0] * b[:, 0] + inv[2] * b[:, 1]
    ab3 = inv[1] * b[:, 2] + inv[3] * b[:, 3]
    y = ((ab0 + ab3) + det).astype(f32)
    return Dataset.new(np.concatenate([a, b], 1), y, [MAT2, MAT2])


def uneven_sizes(k: int = 16, lo: int = 400, hi: int = 262_144, seed: int = 4) -> List[int]:
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), k)).astype(int)
    s[0], s[-1] = lo, hi  # span the whole range
    return [int(v) for v in s]


# --------------------------------------------------------------- populations
def scalar_population(n: int = 1024, seed: int = 11, lo: int = 3, hi: int = 32) -> List[Program]:
    ops = OpSet(["AddF", "SubF", "MulF", "DivF", "SinF", "CosF", "ExpF", NEG], [(FLOAT, 0)], [FLOAT], 2.0)
    return Generator(ops, seed).population(n, lo, hi)


def lorentz_population(n: int = 4096, seed: int = 12, lo: int = 4, hi: int = 48) -> List[Program]:
    ops = OpSet(["AddV3", "SubV3", "CrossV3", "DotV3", "NormV3", "ScaleV3", "AddF", "SubF", "MulF", "DivF"],
                [(VEC3, 0), (VEC3, 3), (VEC3, 6)], [FLOAT, VEC3], 1.0)
    return Generator(ops, seed).population(n, lo, hi)


def transform_population(n: int = 256, seed: int = 13, lo: int = 8, hi: int = 40) -> List[Program]:
    ops = OpSet(["MulM3V3", "AddV3", "SubV3", "NormV3", "DotV3", "ScaleV3", "CrossV3", "AddF", "SubF", "MulF",
                 "DivF", "SqrtF"],
                [(MAT3, 0), (VEC3, 9), (VEC3, 12)], [FLOAT], 1.0, p_const=0.35)
    return Generator(ops, seed).population(n, lo, hi, min_consts=1, max_consts=8)


def inverse_population(n: int = 8192, seed: int = 14, lo: int = 4, hi: int = 64) -> List[Program]:
    ops = OpSet(["InverseM2", "MulM2", "TraceM2", "DetM2", "AddM2", "SubM2", "TransposeM2", "ScaleM2",
                 "AddF", "SubF", "MulF", "DivF"],
                [(MAT2, 0), (MAT2, 4)], [FLOAT], 1.0)
    return Generator(ops, seed).population(n, lo, hi)
