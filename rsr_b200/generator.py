"""Seeded random typed programs.

Grows random expression trees over a typed operator set, the way rsr's
generator builds individuals (src/engine/search/operators/generator.rs:9-105:
typed recursive growth, variables or constants at the leaves), and emits them
in postfix as compiled ``Program``s (src/engine/expr/program.rs:34-55:
constants renumbered in order of appearance).  Lengths are drawn uniformly in
a range and reached by rejection, so populations have the uneven length mix
the workloads ask for.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

from . import isa as I
from .isa import FLOAT, MAT2, MAT3, VEC2, VEC3, Program, Scalar

# Pseudo-op: unary negation, emitted as 0 - x (the reference ISA has no Neg).
NEG = "Neg"


@dataclass
class OpSet:
    ops: List[str]                                 # operator names (isa.OP_NAMES) plus NEG
    variables: List[Tuple[int, int]]               # (type, feature offset)
    const_types: List[int] = field(default_factory=lambda: [FLOAT])
    const_std: float = 1.0
    p_const: float = 0.3                           # leaf is a constant (when both are possible)

    def returning(self, t: int) -> List[str]:
        out = []
        for o in self.ops:
            if o == NEG:
                if t == FLOAT:
                    out.append(o)
            elif I.SIGNATURE[o][1] == t:
                out.append(o)
        return out


def _arity_types(op: str) -> List[int]:
    return [FLOAT] if op == NEG else I.SIGNATURE[op][0]


def _own_size(op: str) -> int:
    """Nodes an operator adds besides its operands (Neg adds its zero constant)."""
    return 2 if op == NEG else 1


class Generator:
    def __init__(self, opset: OpSet, seed: int):
        self.os = opset
        self.rng = np.random.default_rng(seed)
        # smallest subtree size producible for each type (leaf = 1)
        self.min_size: Dict[int, int] = {}
        types = {FLOAT, VEC2, VEC3, MAT2, MAT3}
        for t in types:
            has_leaf = any(v[0] == t for v in opset.variables) or t in opset.const_types
            self.min_size[t] = 1 if has_leaf else 10**6
        for _ in range(8):
            for t in types:
                for o in opset.returning(t):
                    s = _own_size(o) + sum(self.min_size[a] for a in _arity_types(o))
                    self.min_size[t] = min(self.min_size[t], s)

    def _leaf(self, t: int, nodes: list, consts: list) -> None:
        vs = [v for v in self.os.variables if v[0] == t]
        use_const = t in self.os.const_types and (not vs or self.rng.random() < self.os.p_const)
        if use_const:
            w = I.KIND_WIDTH[t]
            vals = self.rng.normal(0.0, self.os.const_std, size=w).astype(np.float32)
            consts.append(Scalar(t, tuple(vals)))
            nodes.append(I.load_const(t, len(consts) - 1))
        else:
            v = vs[self.rng.integers(len(vs))]
            nodes.append(I.load_var(t, v[1]))

    def _grow(self, t: int, budget: int, nodes: list, consts: list) -> None:
        ops = [o for o in self.os.returning(t)
               if _own_size(o) + sum(self.min_size[a] for a in _arity_types(o)) <= budget]
        if (budget <= 1 or not ops) and self.min_size[t] == 1:
            self._leaf(t, nodes, consts)
            return
        o = ops[self.rng.integers(len(ops))]
        args = _arity_types(o)
        rest = budget - _own_size(o) - sum(self.min_size[a] for a in args)
        # split the remaining budget among the operands
        cuts = np.sort(self.rng.integers(0, rest + 1, size=len(args) - 1)) if len(args) > 1 else np.array([], int)
        shares = np.diff(np.concatenate([[0], cuts, [rest]])).astype(int)
        if o == NEG:
            consts.append(Scalar(FLOAT, (0.0,)))
            nodes.append(I.load_const(FLOAT, len(consts) - 1))
            self._grow(FLOAT, self.min_size[FLOAT] + shares[0], nodes, consts)
            nodes.append(I.op("SubF"))
            return
        for a, s in zip(args, shares):
            self._grow(a, self.min_size[a] + int(s), nodes, consts)
        nodes.append(I.op(o))

    def program(self, lo: int, hi: int, min_consts: int = 0, max_consts: int = 10**9,
                root: int = FLOAT, tries: int = 1000) -> Program:
        for _ in range(tries):
            target = int(self.rng.integers(lo, hi + 1))
            nodes: list = []
            consts: list = []
            self._grow(root, target, nodes, consts)
            if lo <= len(nodes) <= hi and min_consts <= len(consts) <= max_consts:
                return Program(nodes, consts)
        raise RuntimeError(f"could not generate a program with length in [{lo}, {hi}]")

    def population(self, n: int, lo: int, hi: int, **kw) -> List[Program]:
        return [self.program(lo, hi, **kw) for _ in range(n)]
