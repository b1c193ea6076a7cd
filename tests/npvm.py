"""A second, vectorised restatement of the reference VM in numpy float32,
used by the tests to cross-check the C oracle op by op.

Follows src/domains/basic/eval.rs and src/domains/linalg/eval.rs operation by
operation; transcendentals call the oracle's Cephes restatement so that the
comparison is bit-exact.  Stacks start zeroed and the result is stack_f[0]
(src/engine/eval/evaluator.rs:20-150).
"""
import numpy as np

from oracle import binding as O
from rsr_b200 import isa as I

f32 = np.float32


def _t(name, x):
    return O.transcendental(name, x)


def eval_points(p: I.Program, X: np.ndarray) -> np.ndarray:
    """X: (n, num_features) float32 -> predictions (n,)."""
    n = X.shape[0]
    Z = lambda w: [np.zeros(n, f32) for _ in range(w)]
    st = {t: [Z(I.TYPE_WIDTH[t]) for _ in range(32)] for t in (I.FLOAT, I.VEC2, I.VEC3, I.MAT2, I.MAT3)}
    sp = {t: 0 for t in st}
    flat, acc = [], 0
    for c in p.constants:
        flat.append(acc)
        acc += I.KIND_WIDTH[c.kind]
    params = p.flatten_params()

    def push(t, v):
        st[t][sp[t]] = [np.asarray(c, f32) for c in v]
        sp[t] += 1

    def pop(t):
        sp[t] -= 1
        return st[t][sp[t]]

    for w in p.code:
        op, a = w & 0xFF, (w >> 8) & 0xFFFF
        name = I.OP_NAMES[op]
        if I.is_load(op):
            t = I.load_type(op)
            if t in (I.INT, I.BOOL):
                continue
            wd = I.TYPE_WIDTH[t]
            if op % 2 == 0:
                push(t, [X[:, a + i].copy() for i in range(wd)])
            else:
                if p.constants[a].kind == t:
                    st[t][sp[t]] = [np.full(n, params[flat[a] + i], f32) for i in range(wd)]
                sp[t] += 1
            continue
        F, V2, V3, M2, M3 = I.FLOAT, I.VEC2, I.VEC3, I.MAT2, I.MAT3
        if name in ("AddF", "SubF", "MulF", "DivF"):
            b, x = pop(F)[0], pop(F)[0]
            r = {"AddF": x + b, "SubF": x - b, "MulF": x * b, "DivF": x / b}[name]
            push(F, [r])
        elif name in ("SinF", "CosF", "ExpF", "LnF"):
            x = pop(F)[0]
            push(F, [_t({"SinF": "sin", "CosF": "cos", "ExpF": "exp", "LnF": "log"}[name], x)])
        elif name == "SqrF":
            x = pop(F)[0]; push(F, [x * x])
        elif name == "SqrtF":
            x = pop(F)[0]; push(F, [np.sqrt(x)])
        elif name == "MakeVec2":
            b, a_ = pop(F)[0], pop(F)[0]; push(V2, [a_, b])
        elif name == "MakeVec3":
            c, b, a_ = pop(F)[0], pop(F)[0], pop(F)[0]; push(V3, [a_, b, c])
        elif name.startswith("Get"):
            t = V2 if name.endswith("V2") else V3
            v = pop(t); push(F, [v["XYZ".index(name[3])]])
        elif name in ("AddV2", "SubV2", "AddV3", "SubV3", "AddM2", "SubM2", "AddM3", "SubM3"):
            t = {"V2": V2, "V3": V3, "M2": M2, "M3": M3}[name[-2:]]
            b, x = pop(t), pop(t)
            push(t, [(u + v) if name.startswith("Add") else (u - v) for u, v in zip(x, b)])
        elif name.startswith("Scale"):
            t = {"V2": V2, "V3": V3, "M2": M2, "M3": M3}[name[-2:]]
            v, s = pop(t), pop(F)[0]
            push(t, [u * s for u in v])
        elif name == "DotV2":
            b, x = pop(V2), pop(V2); push(F, [(x[0] * b[0]) + (x[1] * b[1])])
        elif name == "DotV3":
            b, x = pop(V3), pop(V3); push(F, [((x[0] * b[0]) + (x[1] * b[1])) + (x[2] * b[2])])
        elif name == "NormV2":
            x = pop(V2); push(F, [np.sqrt((x[0] * x[0]) + (x[1] * x[1]))])
        elif name == "NormV3":
            x = pop(V3); push(F, [np.sqrt(((x[0] * x[0]) + (x[1] * x[1])) + (x[2] * x[2]))])
        elif name == "CrossV3":
            b, x = pop(V3), pop(V3)
            push(V3, [x[1] * b[2] - x[2] * b[1], x[2] * b[0] - x[0] * b[2], x[0] * b[1] - x[1] * b[0]])
        elif name == "MakeMat2":
            c1, c0 = pop(V2), pop(V2); push(M2, [c0[0], c0[1], c1[0], c1[1]])
        elif name == "MakeMat3":
            c2, c1, c0 = pop(V3), pop(V3), pop(V3); push(M3, list(c0) + list(c1) + list(c2))
        elif name == "MulM2":
            b, x = pop(M2), pop(M2)
            push(M2, [x[0] * b[0] + x[2] * b[1], x[1] * b[0] + x[3] * b[1], x[0] * b[2] + x[2] * b[3],
                      x[1] * b[2] + x[3] * b[3]])
        elif name == "MulM2V2":
            v, m = pop(V2), pop(M2)
            push(V2, [m[0] * v[0] + m[2] * v[1], m[1] * v[0] + m[3] * v[1]])
        elif name == "DetM2":
            m = pop(M2); push(F, [(m[0] * m[3]) - (m[1] * m[2])])
        elif name == "TraceM2":
            m = pop(M2); push(F, [m[0] + m[3]])
        elif name == "TransposeM2":
            m = pop(M2); push(M2, [m[0], m[2], m[1], m[3]])
        elif name == "InverseM2":
            m = pop(M2)
            det = (m[0] * m[3]) - (m[1] * m[2])
            sing = np.abs(det) < f32(1e-9)
            inv = f32(1.0) / np.where(sing, f32(1.0), det)
            push(M2, [np.where(sing, f32(1), m[3] * inv), np.where(sing, f32(0), (-m[1]) * inv),
                      np.where(sing, f32(0), (-m[2]) * inv), np.where(sing, f32(1), m[0] * inv)])
        elif name == "MulM3":
            b, x = pop(M3), pop(M3)
            push(M3, [(x[r] * b[3 * c] + x[3 + r] * b[3 * c + 1]) + x[6 + r] * b[3 * c + 2]
                      for c in range(3) for r in range(3)])
        elif name == "MulM3V3":
            v, m = pop(V3), pop(M3)
            push(V3, [(m[r] * v[0] + m[3 + r] * v[1]) + m[6 + r] * v[2] for r in range(3)])
        elif name in ("DetM3", "InverseM3"):
            m = pop(M3)
            det = (m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7])) + \
                m[6] * (m[1] * m[5] - m[2] * m[4])
            if name == "DetM3":
                push(F, [det])
            else:
                sing = np.abs(det) < f32(1e-9)
                inv = f32(1.0) / np.where(sing, f32(1.0), det)
                cof = [m[4] * m[8] - m[5] * m[7], -(m[1] * m[8] - m[2] * m[7]), m[1] * m[5] - m[2] * m[4],
                       -(m[3] * m[8] - m[5] * m[6]), m[0] * m[8] - m[2] * m[6], -(m[0] * m[5] - m[2] * m[3]),
                       m[3] * m[7] - m[4] * m[6], -(m[0] * m[7] - m[1] * m[6]), m[0] * m[4] - m[1] * m[3]]
                push(M3, [np.where(sing, f32(1.0 if i % 4 == 0 else 0.0), c * inv) for i, c in enumerate(cof)])
        elif name == "TraceM3":
            m = pop(M3); push(F, [(m[0] + m[4]) + m[8]])
        elif name == "TransposeM3":
            m = pop(M3); push(M3, [m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]])
        else:
            raise ValueError(name)
    return st[I.FLOAT][0][0]
