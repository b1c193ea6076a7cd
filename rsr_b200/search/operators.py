"""Variation operators of the search: random trees, mutation, crossover.

Restates src/engine/search/operators/generator.rs:9-222 (typed random
growth), mutation.rs:10-160 (point mutation, constant perturbation, subtree
mutation) and crossover.rs:7-101 (typed subtree crossover).  The random
draws come from a numpy Generator; the reference draws from rand 0.10's
xoshiro256++ streams, which are not restated, so the operators follow the
reference's decisions and distributions but not its exact sequences.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from .. import isa as I
from . import expr as E
from .expr import CONST, OPER, VAR

f32 = np.float32
Registry = Sequence[Tuple[int, int]]  # (value type, feature offset), dataset.rs:200-222


def _uniform(rng: np.random.Generator, lo: float, hi: float) -> float:
    return float(f32(rng.uniform(lo, hi)))


def random_constant(vtype: int, rng: np.random.Generator) -> Optional[I.Scalar]:
    """generator.rs:185-222: components uniform in [-5, 5)."""
    if vtype in (I.FLOAT, I.VEC2, I.VEC3, I.MAT2, I.MAT3):
        return I.Scalar(vtype, tuple(_uniform(rng, -5.0, 5.0) for _ in range(I.KIND_WIDTH[vtype])))
    if vtype == I.BOOL:
        return I.Scalar(I.BOOL, ())
    return I.Scalar(I.INT, ())


def random_operator(vtype: int, allowed: Sequence[int], parent: Optional[int],
                    rng: np.random.Generator) -> Optional[int]:
    """generator.rs:162-183: uniform over the allowed operators returning
    `vtype` that the parent does not forbid."""
    valid = [op for op in allowed if E.return_type(op) == vtype
             and not (parent is not None and E.is_forbidden_child(parent, op))]
    if not valid:
        return None
    return valid[int(rng.integers(0, len(valid)))]


def _terminal(nodes: List, consts: List, vtype: int, registry: Registry, rng: np.random.Generator) -> bool:
    """A variable or a constant of `vtype` (a coin decides when both exist);
    False when neither exists."""
    vars_ = [r for r in registry if r[0] == vtype]
    c = random_constant(vtype, rng)
    if vars_ and rng.random() < 0.5:
        t, off = vars_[int(rng.integers(0, len(vars_)))]
        nodes.append((VAR, off, vtype))
        return True
    if c is not None:
        nodes.append((CONST, len(consts), vtype))
        consts.append(c)
        return True
    return False


def _grow(nodes, consts, vtype, depth, max_depth, rng, registry, allowed, parent) -> None:
    terminal = depth >= max_depth or (depth > 0 and rng.random() < 0.2)
    if terminal and _terminal(nodes, consts, vtype, registry, rng):
        return
    op = random_operator(vtype, allowed, parent, rng)
    if op is not None:
        for child in E.expected_types(op):
            _grow(nodes, consts, child, depth + 1, max_depth, rng, registry, allowed, op)
        nodes.append((OPER, op, vtype))
        return
    if not _terminal(nodes, consts, vtype, registry, rng):
        raise ValueError(f"no operator, variable or constant of type {I.KIND_NAMES[vtype]}")


def generate_random_tree(vtype: int, max_depth: int, rng: np.random.Generator, registry: Registry,
                         allowed: Sequence[int]) -> Tuple[List[E.Node], List[I.Scalar]]:
    """generate_random_ast (generator.rs:9-30): grows a tree of type `vtype`;
    below the root a node is a terminal with probability 0.2, and always at
    `max_depth`."""
    nodes: List[E.Node] = []
    consts: List[I.Scalar] = []
    _grow(nodes, consts, vtype, 0, max_depth, rng, registry, allowed, None)
    return nodes, consts


# ---------------------------------------------------------------- mutation
def point_mutation(nodes: List[E.Node], consts: List[I.Scalar], rng: np.random.Generator, registry: Registry,
                   allowed: Sequence[int]) -> None:
    """mutation.rs:10-59: a leaf becomes another leaf of its type; an
    operator becomes another operator with the same operand types."""
    if not nodes:
        return
    idx = int(rng.integers(0, len(nodes)))
    node = nodes[idx]
    vtype = node[2]
    if E.arity(node) == 0:
        tmp_nodes: List[E.Node] = []
        n0 = len(consts)
        if _terminal(tmp_nodes, consts, vtype, registry, rng):
            leaf = tmp_nodes[0]
            nodes[idx] = (CONST, n0, vtype) if leaf[0] == CONST else leaf
    else:
        op = random_operator(vtype, allowed, None, rng)
        if op is not None and E.expected_types(op) == E.expected_types(node[1]):
            nodes[idx] = (OPER, op, vtype)


def perturb_constant(c: I.Scalar, rng: np.random.Generator) -> I.Scalar:
    """mutation.rs:83-118: a Float is scaled by U(0.9, 1.1) (80%), shifted by
    U(-0.1, 0.1) (10%) or redrawn from U(-5, 5) (10%); vector and matrix
    components are shifted by U(-0.5, 0.5)."""
    r = rng.random()
    if c.kind == I.FLOAT:
        v = f32(c.values[0])
        if r < 0.8:
            v = f32(v * f32(rng.uniform(0.9, 1.1)))
        elif r < 0.9:
            v = f32(v + f32(rng.uniform(-0.1, 0.1)))
        else:
            v = f32(rng.uniform(-5.0, 5.0))
        return I.Scalar(I.FLOAT, (float(v),))
    if c.kind in (I.VEC2, I.VEC3, I.MAT2, I.MAT3):
        return I.Scalar(c.kind, tuple(float(f32(f32(x) + f32(rng.uniform(-0.5, 0.5)))) for x in c.values))
    return c


def constant_perturbation(nodes: List[E.Node], consts: List[I.Scalar], rng: np.random.Generator) -> None:
    """mutation.rs:61-81: one constant node chosen by reservoir sampling is
    perturbed."""
    target = None
    count = 0
    for i, n in enumerate(nodes):
        if n[0] == CONST:
            count += 1
            if int(rng.integers(0, count)) == 0:
                target = i
    if target is not None:
        ci = nodes[target][1]
        consts[ci] = perturb_constant(consts[ci], rng)


def subtree_mutation(nodes: List[E.Node], consts: List[I.Scalar], rng: np.random.Generator, registry: Registry,
                     max_size: int, max_depth: int, allowed: Sequence[int]) -> List[E.Node]:
    """mutation.rs:120-160: a random subtree is replaced by a new random tree
    of its type, unless the result would exceed `max_size` nodes."""
    if not nodes:
        return nodes
    point = int(rng.integers(0, len(nodes)))
    start, end = E.subtree_bounds(nodes, point)
    vtype = nodes[end][2]
    allowed_len = max(0, max_size - (len(nodes) - (end - start + 1)))
    if allowed_len == 0:
        return nodes
    sub, sub_c = generate_random_tree(vtype, max_depth, rng, registry, allowed)
    off = len(consts)
    sub = [(CONST, n[1] + off, n[2]) if n[0] == CONST else n for n in sub]
    consts.extend(sub_c)
    return nodes[:start] + sub + nodes[end + 1:]


# --------------------------------------------------------------- crossover
def _select_node(nodes: Sequence[E.Node], rng: np.random.Generator, vtype: Optional[int]) -> Optional[int]:
    """crossover.rs:63-101: an operator node with probability 0.9 (when one
    of the wanted type exists), else any node of the type; the first 64
    candidates of each kind are eligible."""
    internal, every = [], []
    for i, n in enumerate(nodes):
        if vtype is None or n[2] == vtype:
            if len(every) < 64:
                every.append(i)
            if E.arity(n) > 0 and len(internal) < 64:
                internal.append(i)
    if not every:
        return None
    if internal and rng.random() < 0.9:
        return internal[int(rng.integers(0, len(internal)))]
    return every[int(rng.integers(0, len(every)))]


def crossover(a_nodes, a_consts, b_nodes, b_consts, rng: np.random.Generator, max_size: int):
    """crossover.rs:7-61: a subtree of parent A is replaced by a subtree of
    the same type from parent B; constants are renumbered in order of use.
    Returns (nodes, constants), or None when the child would be parent A."""
    if not a_nodes or not b_nodes:
        return None
    ra = _select_node(a_nodes, rng, None)
    if ra is None:
        return None
    rb = _select_node(b_nodes, rng, a_nodes[ra][2])
    if rb is None:
        return None
    sa, ea = E.subtree_bounds(a_nodes, ra)
    sb, eb = E.subtree_bounds(b_nodes, rb)
    if sa + (eb - sb + 1) + (len(a_nodes) - ea - 1) > max_size:
        return None
    nodes: List[E.Node] = []
    consts: List[I.Scalar] = []

    def append(src, src_c):
        for n in src:
            if n[0] == CONST:
                nodes.append((CONST, len(consts), n[2]))
                consts.append(src_c[n[1]])
            else:
                nodes.append(n)

    append(a_nodes[:sa], a_consts)
    append(b_nodes[sb:eb + 1], b_consts)
    append(a_nodes[ea + 1:], a_consts)
    return nodes, consts
