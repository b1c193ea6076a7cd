"""Instruction set, constants and compiled programs of rsr's stack VM.

Mirrors the reference's program format so that a population built on the
Rust side maps one-to-one onto the engine's C ABI:

* ``Instruction`` numbering follows the variant order of ``compose_engine!``
  (src/engine/domain.rs:46-63) with ``BasicOpCode`` (src/domains/basic/mod.rs:9-20)
  and ``LinalgOpCode`` (src/domains/linalg/mod.rs:9-51) appended in
  declaration order: 14 loads + 10 basic + 38 linalg = 62 opcodes.
* An instruction word is ``opcode | operand << 8``; the operand is the feature
  offset of a ``LoadVar*`` (u8) or the constant index of a ``LoadConst*`` (u16).
* ``Scalar`` kinds follow src/engine/eval/scalar.rs:4-12; the flat parameter
  order is that of ``Parameterized::flatten_params`` (src/engine/expr/program.rs:100-145).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

# --------------------------------------------------------------- opcodes
LOAD_NAMES = [
    "LoadVarF", "LoadConstF", "LoadVarB", "LoadConstB", "LoadVarI", "LoadConstI",
    "LoadVarV2", "LoadConstV2", "LoadVarV3", "LoadConstV3", "LoadVarM2", "LoadConstM2",
    "LoadVarM3", "LoadConstM3",
]
BASIC_NAMES = ["AddF", "SubF", "MulF", "DivF", "SinF", "CosF", "ExpF", "SqrF", "SqrtF", "LnF"]
LINALG_NAMES = [
    "MakeVec2", "MakeVec3", "GetXV2", "GetYV2", "GetXV3", "GetYV3", "GetZV3",
    "AddV2", "SubV2", "ScaleV2", "DotV2", "NormV2",
    "AddV3", "SubV3", "ScaleV3", "DotV3", "NormV3", "CrossV3",
    "MakeMat2", "AddM2", "SubM2", "ScaleM2", "MulM2", "MulM2V2", "DetM2", "TraceM2", "TransposeM2", "InverseM2",
    "MakeMat3", "AddM3", "SubM3", "ScaleM3", "MulM3", "MulM3V3", "DetM3", "TraceM3", "TransposeM3", "InverseM3",
]
OP_NAMES = LOAD_NAMES + BASIC_NAMES + LINALG_NAMES
N_OPCODES = len(OP_NAMES)
OP = {name: i for i, name in enumerate(OP_NAMES)}
globals().update({name: i for name, i in OP.items()})

# ------------------------------------------------------------ value types
# ValueType order (src/engine/eval/types.rs:2-10) == Scalar order (scalar.rs:4-12)
FLOAT, INT, BOOL, VEC2, VEC3, MAT2, MAT3 = range(7)
KIND_NAMES = ["Float", "Int", "Bool", "Vec2", "Vec3", "Mat2", "Mat3"]
KIND_WIDTH = [1, 0, 0, 2, 3, 4, 9]  # flat parameters per constant (program.rs:84-98)
TYPE_WIDTH = [1, 1, 1, 2, 3, 4, 9]  # feature slots per variable (dataset.rs:44-53)

_LOAD_TYPE = [FLOAT, FLOAT, BOOL, BOOL, INT, INT, VEC2, VEC2, VEC3, VEC3, MAT2, MAT2, MAT3, MAT3]

# (expected operand types, return type) per operator, from
# basic/mod.rs:198-217 and linalg/mod.rs:317-432.
_F, _V2, _V3, _M2, _M3 = FLOAT, VEC2, VEC3, MAT2, MAT3
SIGNATURE = {
    "AddF": ([_F, _F], _F), "SubF": ([_F, _F], _F), "MulF": ([_F, _F], _F), "DivF": ([_F, _F], _F),
    "SinF": ([_F], _F), "CosF": ([_F], _F), "ExpF": ([_F], _F), "SqrF": ([_F], _F), "SqrtF": ([_F], _F),
    "LnF": ([_F], _F),
    "MakeVec2": ([_F, _F], _V2), "MakeVec3": ([_F, _F, _F], _V3),
    "GetXV2": ([_V2], _F), "GetYV2": ([_V2], _F), "GetXV3": ([_V3], _F), "GetYV3": ([_V3], _F), "GetZV3": ([_V3], _F),
    "AddV2": ([_V2, _V2], _V2), "SubV2": ([_V2, _V2], _V2), "ScaleV2": ([_F, _V2], _V2),
    "DotV2": ([_V2, _V2], _F), "NormV2": ([_V2], _F),
    "AddV3": ([_V3, _V3], _V3), "SubV3": ([_V3, _V3], _V3), "ScaleV3": ([_F, _V3], _V3),
    "DotV3": ([_V3, _V3], _F), "NormV3": ([_V3], _F), "CrossV3": ([_V3, _V3], _V3),
    "MakeMat2": ([_V2, _V2], _M2), "AddM2": ([_M2, _M2], _M2), "SubM2": ([_M2, _M2], _M2),
    "ScaleM2": ([_F, _M2], _M2), "MulM2": ([_M2, _M2], _M2), "MulM2V2": ([_M2, _V2], _V2),
    "DetM2": ([_M2], _F), "TraceM2": ([_M2], _F), "TransposeM2": ([_M2], _M2), "InverseM2": ([_M2], _M2),
    "MakeMat3": ([_V3, _V3, _V3], _M3), "AddM3": ([_M3, _M3], _M3), "SubM3": ([_M3, _M3], _M3),
    "ScaleM3": ([_F, _M3], _M3), "MulM3": ([_M3, _M3], _M3), "MulM3V3": ([_M3, _V3], _V3),
    "DetM3": ([_M3], _F), "TraceM3": ([_M3], _F), "TransposeM3": ([_M3], _M3), "InverseM3": ([_M3], _M3),
}

# Unfused FP32 lane-operations per op, the algorithmic work unit used for
# roofline accounting (loads, Make*, Get*, Transpose* = 0).
FLOP_WEIGHT = {n: 0 for n in OP_NAMES}
FLOP_WEIGHT.update({
    "AddF": 1, "SubF": 1, "MulF": 1, "DivF": 1, "SqrF": 1, "SqrtF": 1, "SinF": 1, "CosF": 1, "ExpF": 1, "LnF": 1,
    "AddV2": 2, "SubV2": 2, "AddV3": 3, "SubV3": 3, "AddM2": 4, "SubM2": 4, "AddM3": 9, "SubM3": 9,
    "ScaleV2": 2, "ScaleV3": 3, "ScaleM2": 4, "ScaleM3": 9, "DotV2": 3, "DotV3": 5, "NormV2": 4, "NormV3": 6,
    "CrossV3": 9, "MulM2V2": 6, "MulM2": 12, "MulM3V3": 15, "MulM3": 45, "DetM2": 3, "DetM3": 14,
    "TraceM2": 1, "TraceM3": 2, "InverseM2": 8, "InverseM3": 51,
})
MSE_EPILOGUE_FLOPS = 3

# Differentiability (basic/mod.rs:260-262, linalg/mod.rs:493-495).
NON_DIFFERENTIABLE = {OP["InverseM2"], OP["InverseM3"]}


def word(opcode: int, operand: int = 0) -> int:
    """Encode one instruction word: opcode in bits 0-7, operand in bits 8-23."""
    if not 0 <= opcode < N_OPCODES:
        raise ValueError(f"opcode {opcode} out of range")
    if not 0 <= operand <= 0xFFFF:
        raise ValueError(f"operand {operand} out of range")
    return opcode | (operand << 8)


def decode(w: int) -> Tuple[int, int]:
    return w & 0xFF, (w >> 8) & 0xFFFF


def is_load(opcode: int) -> bool:
    return opcode < 14


def load_type(opcode: int) -> int:
    return _LOAD_TYPE[opcode]


def signature(opcode: int) -> Tuple[List[int], int]:
    """(operand types, result type) of an operator; loads return ([], type)."""
    if is_load(opcode):
        return [], _LOAD_TYPE[opcode]
    return SIGNATURE[OP_NAMES[opcode]]


def load_var(vtype: int, feature_offset: int) -> int:
    return word({FLOAT: 0, BOOL: 2, INT: 4, VEC2: 6, VEC3: 8, MAT2: 10, MAT3: 12}[vtype], feature_offset)


def load_const(vtype: int, const_index: int) -> int:
    return word({FLOAT: 1, BOOL: 3, INT: 5, VEC2: 7, VEC3: 9, MAT2: 11, MAT3: 13}[vtype], const_index)


def op(name: str) -> int:
    return word(OP[name])


# ------------------------------------------------------------- programs
@dataclass
class Scalar:
    """One constant of a program (scalar.rs:4-12): kind + component values.
    Mat2/Mat3 components are column-major, as the reference stores them."""
    kind: int
    values: Tuple[float, ...] = ()

    def __post_init__(self):
        self.values = tuple(float(np.float32(v)) for v in self.values)
        if len(self.values) != KIND_WIDTH[self.kind] and self.kind not in (INT, BOOL):
            raise ValueError(f"{KIND_NAMES[self.kind]} needs {KIND_WIDTH[self.kind]} values")

    @staticmethod
    def float(v: float) -> "Scalar":
        return Scalar(FLOAT, (v,))


@dataclass
class Program:
    """A compiled postfix program (src/engine/expr/program.rs:18-23)."""
    code: List[int]
    constants: List[Scalar] = field(default_factory=list)

    def param_count(self) -> int:
        return sum(KIND_WIDTH[c.kind] for c in self.constants)

    def flatten_params(self) -> np.ndarray:
        out = [v for c in self.constants for v in (c.values if KIND_WIDTH[c.kind] else ())]
        return np.asarray(out, dtype=np.float32)

    def unflatten_params(self, buf: Sequence[float]) -> None:
        ptr = 0
        for c in self.constants:
            w = KIND_WIDTH[c.kind]
            if w:
                c.values = tuple(float(np.float32(v)) for v in buf[ptr:ptr + w])
                ptr += w

    def kinds(self) -> np.ndarray:
        return np.asarray([c.kind for c in self.constants], dtype=np.uint8)

    def code_array(self) -> np.ndarray:
        return np.asarray(self.code, dtype=np.uint32)

    def flops_per_point(self) -> int:
        return sum(FLOP_WEIGHT[OP_NAMES[w & 0xFF]] for w in self.code) + MSE_EPILOGUE_FLOPS

    def is_differentiable(self) -> bool:
        return not any((w & 0xFF) in NON_DIFFERENTIABLE for w in self.code)


@dataclass
class PackedPrograms:
    """A population packed for the C ABI: concatenated code, constant kinds
    and flat parameters with (n+1)-entry offset arrays."""
    code: np.ndarray
    code_off: np.ndarray
    kinds: np.ndarray
    kind_off: np.ndarray
    params: np.ndarray
    param_off: np.ndarray

    @property
    def n(self) -> int:
        return len(self.code_off) - 1

    def program(self, i: int) -> Program:
        code = [int(w) for w in self.code[self.code_off[i]:self.code_off[i + 1]]]
        kinds = self.kinds[self.kind_off[i]:self.kind_off[i + 1]]
        flat = self.params[self.param_off[i]:self.param_off[i + 1]]
        consts, p = [], 0
        for k in kinds:
            w = KIND_WIDTH[int(k)]
            consts.append(Scalar(int(k), tuple(flat[p:p + w])))
            p += w
        return Program(code, consts)


def pack(programs: Sequence[Program]) -> PackedPrograms:
    code_off = np.zeros(len(programs) + 1, dtype=np.uint64)
    kind_off = np.zeros(len(programs) + 1, dtype=np.uint64)
    param_off = np.zeros(len(programs) + 1, dtype=np.uint64)
    codes, kinds, params = [], [], []
    for i, p in enumerate(programs):
        c, k, f = p.code_array(), p.kinds(), p.flatten_params()
        codes.append(c); kinds.append(k); params.append(f)
        code_off[i + 1] = code_off[i] + len(c)
        kind_off[i + 1] = kind_off[i] + len(k)
        param_off[i + 1] = param_off[i] + len(f)
    cat = lambda xs, dt: np.concatenate(xs).astype(dt) if xs and sum(map(len, xs)) else np.zeros(0, dt)
    return PackedPrograms(cat(codes, np.uint32), code_off, cat(kinds, np.uint8), kind_off,
                          cat(params, np.float32), param_off)
