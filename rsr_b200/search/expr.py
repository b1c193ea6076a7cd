"""Expression trees of the search: nodes, simplification, compilation.

An expression is a postfix list of nodes, as in the reference
(src/engine/expr/node.rs:4-9): ``(OPER, opcode, return type)``,
``(VAR, feature offset, type)`` or ``(CONST, constant index, type)``.

* ``simplify`` restates ``simplify_ast`` (src/engine/expr/simplify.rs:13-135)
  with the domains' ``try_simplify`` rules (src/domains/basic/mod.rs:45-130,
  src/domains/linalg/mod.rs:227-315) and constant folding
  (linalg/mod.rs:728-892), in f32 arithmetic.  The transcendental folds
  (sin/cos/exp/ln of a constant) use numpy's float32 functions where the
  reference calls Rust's; those two may differ in the last place.
* ``compile`` restates ``Program::from_nodes`` (src/engine/expr/program.rs:34-80).
* ``complexity``, ``has_forbidden_patterns`` and ``subtree_bounds`` restate
  src/engine/search/individual.rs:112-205 with the weight tables of
  node.rs:20-33, basic/mod.rs:156-163 and linalg/mod.rs:434-477.
* ``format_expr`` restates format_ast (src/engine/expr/format.rs:4-36).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from .. import isa as I

OPER, VAR, CONST = 0, 1, 2
Node = Tuple[int, int, int]

f32 = np.float32

# ------------------------------------------------------------------ tables
_OP_WEIGHT = {
    # basic/mod.rs:156-163
    "AddF": 1, "SubF": 1, "MulF": 1, "DivF": 2, "SqrF": 2, "SqrtF": 2, "SinF": 3, "CosF": 3, "ExpF": 4, "LnF": 4,
    # linalg/mod.rs:434-477
    "AddV2": 1, "SubV2": 1, "AddV3": 1, "SubV3": 1, "AddM2": 1, "SubM2": 1, "AddM3": 1, "SubM3": 1,
    "MakeVec2": 2, "GetXV2": 2, "GetYV2": 2, "ScaleV2": 2, "DotV2": 2, "MakeVec3": 2, "GetXV3": 2, "GetYV3": 2,
    "GetZV3": 2, "ScaleV3": 2, "DotV3": 2, "ScaleM2": 2, "ScaleM3": 2,
    "NormV2": 3, "NormV3": 3, "MakeMat2": 3, "MulM2": 3, "MulM2V2": 3, "TraceM2": 3, "TransposeM2": 3,
    "MulM3V3": 3, "TraceM3": 3, "TransposeM3": 3,
    "CrossV3": 4, "DetM2": 4, "InverseM2": 4, "MulM3": 4, "MakeMat3": 5, "DetM3": 5, "InverseM3": 6,
}
OP_WEIGHT = {I.OP[n]: w for n, w in _OP_WEIGHT.items()}
CONST_WEIGHT = [1, 1, 1, 2, 3, 4, 9]  # node.rs:24-31, by ValueType

# Children an operator may not have in generated trees (basic/mod.rs:165-195,
# linalg/mod.rs:479-491).
_FORBIDDEN = {
    "SinF": {"SinF", "CosF", "ExpF", "LnF"}, "CosF": {"SinF", "CosF", "ExpF", "LnF"},
    "ExpF": {"ExpF", "SinF", "CosF", "SqrF", "LnF"},
    "SqrtF": {"SqrtF", "SqrF", "SinF", "CosF", "LnF", "ExpF"},
    "SqrF": {"SqrF", "SqrtF"}, "LnF": {"LnF", "ExpF", "SinF", "CosF"},
    "TransposeM2": {"TransposeM2"}, "TransposeM3": {"TransposeM3"},
    "InverseM2": {"InverseM2"}, "InverseM3": {"InverseM3"},
    "GetXV2": {"MakeVec2"}, "GetYV2": {"MakeVec2"},
    "GetXV3": {"MakeVec3"}, "GetYV3": {"MakeVec3"}, "GetZV3": {"MakeVec3"},
}
FORBIDDEN_CHILD = {I.OP[p]: {I.OP[c] for c in cs} for p, cs in _FORBIDDEN.items()}

_SIG = {I.OP[n]: (tuple(a), r) for n, (a, r) in I.SIGNATURE.items()}


def expected_types(opcode: int) -> Tuple[int, ...]:
    return _SIG[opcode][0]


def return_type(opcode: int) -> int:
    return _SIG[opcode][1]


def arity(node: Node) -> int:
    return len(_SIG[node[1]][0]) if node[0] == OPER else 0


def weight(node: Node) -> int:
    if node[0] == OPER:
        return OP_WEIGHT[node[1]]
    if node[0] == VAR:
        return 1
    return CONST_WEIGHT[node[2]]


def is_forbidden_child(parent: int, child: int) -> bool:
    return child in FORBIDDEN_CHILD.get(parent, ())


def is_differentiable(opcode: int) -> bool:
    return opcode not in I.NON_DIFFERENTIABLE


def complexity(nodes: Sequence[Node]) -> int:
    return sum(weight(n) for n in nodes)


def subtree_bounds(nodes: Sequence[Node], root: int) -> Tuple[int, int]:
    """(first, last) node of the subtree whose root is ``root``
    (individual.rs:89-106)."""
    needed = 1
    i = root
    while True:
        needed += arity(nodes[i]) - 1
        if needed == 0:
            return i, root
        if i == 0:
            break
        i -= 1
    return 0, root


_TRIG, _EXP, _LN, _POW, _TRANSPOSE, _INVERSE, _DET = (1 << k for k in range(7))
_PATTERN = {}
for _n, (_bad, _flag) in {
    "SinF": (_TRIG | _EXP | _LN, _TRIG), "CosF": (_TRIG | _EXP | _LN, _TRIG),
    "ExpF": (_TRIG | _EXP | _LN | _POW, _EXP), "LnF": (_TRIG | _EXP | _LN, _LN),
    "SqrtF": (_POW | _TRIG | _LN | _EXP, _POW), "SqrF": (_POW | _TRIG | _LN | _EXP, _POW),
    "TransposeM2": (_TRANSPOSE, _TRANSPOSE), "TransposeM3": (_TRANSPOSE, _TRANSPOSE),
    "InverseM2": (_INVERSE, _INVERSE), "InverseM3": (_INVERSE, _INVERSE),
    "DetM2": (_DET, _DET), "DetM3": (_DET, _DET),
}.items():
    _PATTERN[I.OP[_n]] = (_bad, _flag)


def has_forbidden_patterns(nodes: Sequence[Node]) -> bool:
    """Nested transcendental/power/transpose/inverse/det patterns, or a
    malformed stack (individual.rs:112-196)."""
    stack: List[int] = []
    for n in nodes:
        if n[0] != OPER:
            stack.append(0)
            continue
        a = arity(n)
        if len(stack) < a:
            return True
        flags = 0
        for _ in range(a):
            flags |= stack.pop()
        rule = _PATTERN.get(n[1])
        if rule is None:
            stack.append(flags)
            continue
        bad, flag = rule
        if flags & bad:
            return True
        stack.append(flags | flag)
    return False


# --------------------------------------------------------------- scalars
def _vals(c: I.Scalar) -> List[np.float32]:
    return [f32(v) for v in c.values]


def is_zero(c: I.Scalar) -> bool:
    """scalar.rs:15-25 (Int and Bool constants are never zero here)."""
    if c.kind in (I.INT, I.BOOL):
        return False
    return all(abs(v) < f32(1e-6) for v in _vals(c))


def is_one(c: I.Scalar) -> bool:
    return c.kind == I.FLOAT and abs(_vals(c)[0] - f32(1.0)) < f32(1e-6)


def is_identity(c: I.Scalar) -> bool:
    if c.kind == I.MAT2:
        m = _vals(c)
        ident = (1, 0, 0, 1)
    elif c.kind == I.MAT3:
        m = _vals(c)
        ident = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    else:
        return False
    return all(abs(v - f32(e)) < f32(1e-6) for v, e in zip(m, ident))


def apply_threshold(c: I.Scalar, threshold: float) -> I.Scalar:
    """Components below the threshold in magnitude become 0 (scalar.rs:60-94)."""
    if c.kind in (I.INT, I.BOOL):
        return c
    t = f32(threshold)
    return I.Scalar(c.kind, tuple(0.0 if abs(v) < t else float(v) for v in _vals(c)))


def _S(kind: int, vals) -> I.Scalar:
    return I.Scalar(kind, tuple(float(f32(v)) for v in vals))


def _fold_basic(op: str, a: np.float32, b: Optional[np.float32]) -> Optional[I.Scalar]:
    with np.errstate(all="ignore"):
        if b is None:
            r = {"SinF": lambda: np.sin(a), "CosF": lambda: np.cos(a), "ExpF": lambda: np.exp(a),
                 "SqrF": lambda: a * a, "SqrtF": lambda: np.sqrt(a), "LnF": lambda: np.log(a)}.get(op)
        else:
            r = {"AddF": lambda: a + b, "SubF": lambda: a - b, "MulF": lambda: a * b,
                 "DivF": lambda: a / b}.get(op)
        if r is None:
            return None
        v = f32(r())
    return _S(I.FLOAT, [v]) if np.isfinite(v) else None


def _det3(m):
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7]) + m[6] * (m[1] * m[5] - m[2] * m[4])


def _fold_linalg(op: str, args: List[I.Scalar]) -> Optional[I.Scalar]:
    """fold_linalg_constants (linalg/mod.rs:743-892): the op on constant
    operands of the expected kinds, in f32."""
    kinds = [a.kind for a in args]
    v = [_vals(a) for a in args]
    F, V2, V3, M2, M3 = I.FLOAT, I.VEC2, I.VEC3, I.MAT2, I.MAT3
    with np.errstate(all="ignore"):
        if op == "MakeVec2" and kinds == [F, F]:
            return _S(V2, [v[0][0], v[1][0]])
        if op == "MakeVec3" and kinds == [F, F, F]:
            return _S(V3, [v[0][0], v[1][0], v[2][0]])
        if op in ("GetXV2", "GetYV2") and kinds == [V2]:
            return _S(F, [v[0][0 if op == "GetXV2" else 1]])
        if op in ("GetXV3", "GetYV3", "GetZV3") and kinds == [V3]:
            return _S(F, [v[0]["XYZ".index(op[3])]])
        for vk, w, add, sub, scale in ((V2, 2, "AddV2", "SubV2", "ScaleV2"), (V3, 3, "AddV3", "SubV3", "ScaleV3"),
                                       (M2, 4, "AddM2", "SubM2", "ScaleM2"), (M3, 9, "AddM3", "SubM3", "ScaleM3")):
            if op == add and kinds == [vk, vk]:
                return _S(vk, [v[0][i] + v[1][i] for i in range(w)])
            if op == sub and kinds == [vk, vk]:
                return _S(vk, [v[0][i] - v[1][i] for i in range(w)])
            if op == scale and kinds == [F, vk]:
                return _S(vk, [v[0][0] * v[1][i] for i in range(w)])
        if op == "DotV2" and kinds == [V2, V2]:
            return _S(F, [v[0][0] * v[1][0] + v[0][1] * v[1][1]])
        if op == "NormV2" and kinds == [V2]:
            return _S(F, [np.sqrt(v[0][0] * v[0][0] + v[0][1] * v[0][1])])
        if op == "DotV3" and kinds == [V3, V3]:
            a, b = v
            return _S(F, [a[0] * b[0] + a[1] * b[1] + a[2] * b[2]])
        if op == "NormV3" and kinds == [V3]:
            a = v[0]
            return _S(F, [np.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])])
        if op == "CrossV3" and kinds == [V3, V3]:
            a, b = v
            return _S(V3, [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])
        if op == "MakeMat2" and kinds == [V2, V2]:
            return _S(M2, v[0] + v[1])
        if op == "MulM2" and kinds == [M2, M2]:
            a, b = v
            return _S(M2, [a[0] * b[0] + a[2] * b[1], a[1] * b[0] + a[3] * b[1],
                           a[0] * b[2] + a[2] * b[3], a[1] * b[2] + a[3] * b[3]])
        if op == "MulM2V2" and kinds == [M2, V2]:
            m, x = v
            return _S(V2, [m[0] * x[0] + m[2] * x[1], m[1] * x[0] + m[3] * x[1]])
        if op == "DetM2" and kinds == [M2]:
            m = v[0]
            return _S(F, [m[0] * m[3] - m[1] * m[2]])
        if op == "TraceM2" and kinds == [M2]:
            m = v[0]
            return _S(F, [m[0] + m[3]])
        if op == "TransposeM2" and kinds == [M2]:
            m = v[0]
            return _S(M2, [m[0], m[2], m[1], m[3]])
        if op == "InverseM2" and kinds == [M2]:
            m = v[0]
            det = m[0] * m[3] - m[1] * m[2]
            if abs(det) > f32(1e-9):
                return _S(M2, [m[3] / det, -m[1] / det, -m[2] / det, m[0] / det])
            return None
        if op == "MakeMat3" and kinds == [V3, V3, V3]:
            return _S(M3, v[0] + v[1] + v[2])
        if op == "MulM3" and kinds == [M3, M3]:
            a, b = v
            return _S(M3, [a[r] * b[3 * c] + a[3 + r] * b[3 * c + 1] + a[6 + r] * b[3 * c + 2]
                           for c in range(3) for r in range(3)])
        if op == "MulM3V3" and kinds == [M3, V3]:
            m, x = v
            return _S(V3, [m[r] * x[0] + m[3 + r] * x[1] + m[6 + r] * x[2] for r in range(3)])
        if op == "TraceM3" and kinds == [M3]:
            m = v[0]
            return _S(F, [m[0] + m[4] + m[8]])
        if op == "TransposeM3" and kinds == [M3]:
            m = v[0]
            return _S(M3, [m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]])
        if op == "DetM3" and kinds == [M3]:
            return _S(F, [_det3(v[0])])
        if op == "InverseM3" and kinds == [M3]:
            m = v[0]
            det = _det3(m)
            if abs(det) > f32(1e-9):
                inv = f32(1.0) / det
                return _S(M3, [(m[4] * m[8] - m[5] * m[7]) * inv, -(m[1] * m[8] - m[2] * m[7]) * inv,
                               (m[1] * m[5] - m[2] * m[4]) * inv, -(m[3] * m[8] - m[5] * m[6]) * inv,
                               (m[0] * m[8] - m[2] * m[6]) * inv, -(m[0] * m[5] - m[2] * m[3]) * inv,
                               (m[3] * m[7] - m[4] * m[6]) * inv, -(m[0] * m[7] - m[1] * m[6]) * inv,
                               (m[0] * m[4] - m[1] * m[3]) * inv])
            return None
    return None


_ZERO_FOR = {"SubV2": I.VEC2, "ScaleV2": I.VEC2, "MulM2V2": I.VEC2, "SubV3": I.VEC3, "ScaleV3": I.VEC3,
             "CrossV3": I.VEC3, "MulM3V3": I.VEC3, "SubM2": I.MAT2, "ScaleM2": I.MAT2, "MulM2": I.MAT2,
             "SubM3": I.MAT3, "ScaleM3": I.MAT3, "MulM3": I.MAT3}


def _zero(kind: int) -> I.Scalar:
    return I.Scalar(kind, (0.0,) * I.KIND_WIDTH[kind])


def try_simplify(opcode: int, consts: List[Optional[I.Scalar]], args_equal: bool):
    """('const', Scalar) | ('keep', arg index) | None (domain.rs:5-9)."""
    name = I.OP_NAMES[opcode]
    n = len(consts)
    basic = name in I.BASIC_NAMES
    if n and all(c is not None for c in consts):
        if basic:
            if consts[0].kind == I.FLOAT:
                if n == 1:
                    r = _fold_basic(name, f32(consts[0].values[0]), None)
                    if r is not None:
                        return ("const", r)
                elif n == 2 and consts[1].kind == I.FLOAT:
                    r = _fold_basic(name, f32(consts[0].values[0]), f32(consts[1].values[0]))
                    if r is not None:
                        return ("const", r)
        else:
            r = _fold_linalg(name, consts)
            if r is not None:
                return ("const", r)
    if n != 2:
        return None
    az = consts[0] is not None and is_zero(consts[0])
    bz = consts[1] is not None and is_zero(consts[1])
    a1 = consts[0] is not None and is_one(consts[0])
    b1 = consts[1] is not None and is_one(consts[1])
    if basic:
        if name == "AddF":
            if bz:
                return ("keep", 0)
            if az:
                return ("keep", 1)
        elif name == "MulF":
            if b1:
                return ("keep", 0)
            if a1:
                return ("keep", 1)
            if az or bz:
                return ("const", _zero(I.FLOAT))
        elif name == "SubF":
            if bz:
                return ("keep", 0)
            if args_equal:
                return ("const", _zero(I.FLOAT))
        elif name == "DivF":
            if b1:
                return ("keep", 0)
            if az and not bz:
                return ("const", _zero(I.FLOAT))
            if args_equal:
                return ("const", I.Scalar.float(1.0))
        return None
    if name in ("AddV2", "AddV3", "AddM2", "AddM3"):
        if bz:
            return ("keep", 0)
        if az:
            return ("keep", 1)
    elif name in ("SubV2", "SubV3", "SubM2", "SubM3"):
        if bz:
            return ("keep", 0)
        if args_equal:
            return ("const", _zero(_ZERO_FOR[name]))
    elif name in ("ScaleV2", "ScaleV3", "ScaleM2", "ScaleM3"):
        if az:
            return ("const", _zero(_ZERO_FOR[name]))
        if a1:
            return ("keep", 1)
    elif name in ("DotV2", "DotV3"):
        if az or bz:
            return ("const", _zero(I.FLOAT))
    elif name == "CrossV3":
        if az or bz or args_equal:
            return ("const", _zero(I.VEC3))
    elif name in ("MulM2", "MulM3"):
        ai = consts[0] is not None and is_identity(consts[0])
        bi = consts[1] is not None and is_identity(consts[1])
        if ai:
            return ("keep", 1)
        if bi:
            return ("keep", 0)
        if az or bz:
            return ("const", _zero(_ZERO_FOR[name]))
    elif name in ("MulM2V2", "MulM3V3"):
        if consts[0] is not None and is_identity(consts[0]):
            return ("keep", 1)
        if az or bz:
            return ("const", _zero(_ZERO_FOR[name]))
    return None


_INVERSE_PAIRS = {(I.OP["LnF"], I.OP["ExpF"]), (I.OP["ExpF"], I.OP["LnF"]),
                  (I.OP["SqrtF"], I.OP["SqrF"]), (I.OP["SqrF"], I.OP["SqrtF"])}


def simplify(nodes: Sequence[Node], constants: Sequence[I.Scalar]) -> Tuple[List[Node], List[I.Scalar]]:
    """simplify_ast (simplify.rs:13-135): one postfix pass that folds constant
    operands, applies the identity rules, drops ln(exp(x))-style pairs and
    renumbers the constants in their order of use."""
    if not nodes:
        return [], []
    out: List[Node] = []
    out_c: List[I.Scalar] = []
    stack: List[Tuple[int, Optional[I.Scalar]]] = []  # (start index in out, constant value)
    for node in nodes:
        if node[0] == CONST:
            val = constants[node[1]]
            start = len(out)
            out.append((CONST, len(out_c), node[2]))
            out_c.append(val)
            stack.append((start, val))
            continue
        if node[0] == VAR:
            stack.append((len(out), None))
            out.append(node)
            continue
        a = arity(node)
        if len(stack) < a:
            stack.append((len(out), None))
            out.append(node)
            continue
        args = stack[len(stack) - a:]
        del stack[len(stack) - a:]
        equal = False
        if a == 2:
            sa, sb = args[0][0], args[1][0]
            if sa < sb <= len(out):
                equal = out[sa:sb] == out[sb:]
        action = try_simplify(node[1], [c for _, c in args], equal)
        if action is not None and action[0] == "const":
            val = action[1]
            del out[args[0][0]:]
            start = len(out)
            out.append((CONST, len(out_c), return_type(node[1])))
            out_c.append(val)
            stack.append((start, val))
        elif action is not None:
            k = action[1]
            s0 = args[0][0]
            ts = args[k][0]
            te = len(out) if k == a - 1 else args[k + 1][0]
            if ts > s0:
                out[s0:s0 + (te - ts)] = out[ts:te]
            del out[s0 + (te - ts):]
            stack.append((s0, args[k][1]))
        else:
            if a == 1 and len(out) > args[0][0] and out[-1][0] == OPER and (node[1], out[-1][1]) in _INVERSE_PAIRS:
                out.pop()
                stack.append((args[0][0], None))
                continue
            out.append(node)
            stack.append((args[0][0], None))
    return out, out_c


# ------------------------------------------------------------ compilation
_LOAD_VAR = {I.FLOAT: I.OP["LoadVarF"], I.BOOL: I.OP["LoadVarB"], I.INT: I.OP["LoadVarI"],
             I.VEC2: I.OP["LoadVarV2"], I.VEC3: I.OP["LoadVarV3"], I.MAT2: I.OP["LoadVarM2"],
             I.MAT3: I.OP["LoadVarM3"]}
_LOAD_CONST = {t: op + 1 for t, op in _LOAD_VAR.items()}


def compile_program(nodes: Sequence[Node], constants: Sequence[I.Scalar]) -> I.Program:
    """Program::from_nodes (program.rs:34-56): postfix code, and the constants
    in their order of use (one copy per use)."""
    code: List[int] = []
    consts: List[I.Scalar] = []
    for n in nodes:
        if n[0] == VAR:
            code.append(I.word(_LOAD_VAR[n[2]], n[1]))
        elif n[0] == CONST:
            code.append(I.word(_LOAD_CONST[n[2]], len(consts)))
            c = constants[n[1]]
            consts.append(I.Scalar(c.kind, c.values))
        else:
            code.append(I.word(n[1]))
    return I.Program(code, consts)


# -------------------------------------------------------------- formatting
# basic/mod.rs:222-235, linalg/mod.rs:692-725
_FMT = {"AddF": "({} + {})", "SubF": "({} - {})", "MulF": "({} * {})", "DivF": "({} / {})",
        "SinF": "sin({})", "CosF": "cos({})", "ExpF": "exp({})", "SqrF": "({})^2", "SqrtF": "sqrt({})",
        "LnF": "ln({})", "MakeVec2": "({}, {})", "MakeVec3": "({}, {}, {})", "GetXV2": "{}.x", "GetXV3": "{}.x",
        "GetYV2": "{}.y", "GetYV3": "{}.y", "GetZV3": "{}.z", "DotV2": "<{} \u2022 {}>", "DotV3": "<{} \u2022 {}>",
        "CrossV3": "({} x {})", "NormV2": "||{}||", "NormV3": "||{}||", "InverseM2": "{}^-1", "InverseM3": "{}^-1",
        "TransposeM2": "{}^T", "TransposeM3": "{}^T", "DetM2": "det({})", "DetM3": "det({})", "TraceM2": "tr({})",
        "TraceM3": "tr({})", "MakeMat2": "({}, {})", "MakeMat3": "({}, {}, {})"}
for _n in ("AddV2", "AddV3", "AddM2", "AddM3"):
    _FMT[_n] = "({} + {})"
for _n in ("SubV2", "SubV3", "SubM2", "SubM3"):
    _FMT[_n] = "({} - {})"
for _n in ("ScaleV2", "ScaleV3", "ScaleM2", "ScaleM3", "MulM2", "MulM3", "MulM2V2", "MulM3V3"):
    _FMT[_n] = "({} * {})"


def _fmt_scalar(c: I.Scalar) -> str:
    v = c.values
    if c.kind == I.FLOAT:
        return f"{v[0]:.4f}"
    if c.kind == I.MAT2:
        return "[{:.2f}, {:.2f}; {:.2f}, {:.2f}]".format(v[0], v[2], v[1], v[3])
    if c.kind == I.MAT3:
        return "[{:.2f}, {:.2f}, {:.2f}; {:.2f}, {:.2f}, {:.2f}; {:.2f}, {:.2f}, {:.2f}]".format(
            v[0], v[3], v[6], v[1], v[4], v[7], v[2], v[5], v[8])
    return "[" + ", ".join(f"{x:.2f}" for x in v) + "]"


def format_expr(nodes: Sequence[Node], constants: Sequence[I.Scalar]) -> str:
    """Infix text of an expression (format.rs:4-36)."""
    stack: List[str] = []
    for n in nodes:
        if n[0] == CONST:
            stack.append(_fmt_scalar(constants[n[1]]) if n[1] < len(constants) else f"C[{n[1]}]")
        elif n[0] == VAR:
            stack.append(f"X{n[1]}_{I.KIND_NAMES[n[2]]}")
        else:
            a = arity(n)
            args = [stack.pop() if stack else "?" for _ in range(a)][::-1]
            name = I.OP_NAMES[n[1]]
            stack.append(_FMT[name].format(*args))
    return stack.pop() if stack else "Empty expression"
