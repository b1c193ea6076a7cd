"""A numpy emulator of the register adjoint's code (uops.h, kAdjHeaderWords):
the accumulator machine's forward sweep with its tape stores, then the
reverse sweep over the reverse entries, for every point of a dataset at
once.  It restates the rules kernels_adj.cu implements, so the CPU tests
can check an encoding's gradients against the dual-number oracle before any
device runs it.  Test infrastructure only; float32 values, float64 sums.
"""
from __future__ import annotations

import numpy as np

from oracle import binding as O
from rsr_b200 import evaluator as E

f32 = np.float32
BASE = [0, 32, 64, 104, 136]
WIDTH = [1, 2, 3, 4, 9]
NBIN = [6, 3, 5, 5, 5]
TAPE = [27, 59, 98, 131, 163]
SF, SV2, SV3, SM2, SM3 = range(5)


def block(kind):
    for t in (SM3, SM2, SV3, SV2, SF):
        if kind >= BASE[t]:
            return t
    return SF


def kv_scale(nb):
    return 3 + 3 * nb


def kv_dot(nb):
    return kv_scale(nb) + 4


def kv_norm(nb):
    return kv_dot(nb) + 3


def kv_mulm(nb, w):
    return kv_norm(nb) + 1 + w


def kv_make(nb, w):
    return kv_mulm(nb, w) + 4


def _sin(x):
    return _tr("sin", x)


def _cos(x):
    return _tr("cos", x)


def _tr(which, x):
    x = np.asarray(x, f32)
    n = len(x)
    pad = (-n) % 8
    y = O.transcendental(which, np.concatenate([x, np.zeros(pad, f32)]), simd=True)
    return y[:n]


def cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def mul_mat(a, b, n):  # column-major n x n
    out = [None] * (n * n)
    for c in range(n):
        for r in range(n):
            s = a[r] * b[n * c]
            for k in range(1, n):
                s = s + a[n * k + r] * b[n * c + k]
            out[n * c + r] = s
    return out


def mul_mat_vec(m, v, n):
    out = []
    for r in range(n):
        s = m[r] * v[0]
        for k in range(1, n):
            s = s + m[n * k + r] * v[k]
        out.append(s)
    return out


def det(m, n):
    if n == 2:
        return m[0] * m[3] - m[1] * m[2]
    return (m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7])) + \
        m[6] * (m[1] * m[5] - m[2] * m[4])


def cofactor(m, n, r, c):
    if n == 2:
        return [m[3], -m[2], -m[1], m[0]][2 * c + r]
    r1, r2, c1, c2 = (r + 1) % 3, (r + 2) % 3, (c + 1) % 3, (c + 2) % 3
    return m[3 * c1 + r1] * m[3 * c2 + r2] - m[3 * c2 + r1] * m[3 * c1 + r2]


def inverse(m, n):
    """The reference's inverse (linalg/eval.rs:316-329, 476-506): adjugate
    times 1/det, identity where |det| < 1e-9."""
    d = det(m, n)
    sing = np.abs(d) < f32(1e-9)
    inv = f32(1) / np.where(sing, f32(1), d)
    if n == 2:
        c = [m[3], -m[1], -m[2], m[0]]
        out = [x * inv for x in c]
    else:
        c = [m[4] * m[8] - m[5] * m[7], m[1] * m[8] - m[2] * m[7], m[1] * m[5] - m[2] * m[4],
             m[3] * m[8] - m[5] * m[6], m[0] * m[8] - m[2] * m[6], m[0] * m[5] - m[2] * m[3],
             m[3] * m[7] - m[4] * m[6], m[0] * m[7] - m[1] * m[6], m[0] * m[4] - m[1] * m[3]]
        out = [(-c[i] if i & 1 else c[i]) * inv for i in range(9)]
    return [np.where(sing, f32(1) if i % (n + 1) == 0 else f32(0), out[i]).astype(f32) for i in range(n * n)]


def transpose(m, n):
    return [m[n * (i % n) + i // n] for i in range(n * n)]


def _is_unary(t, k):
    if t == SF:
        return 21 <= k < 27
    if t in (SV2, SV3):
        return kv_norm(NBIN[t]) <= k <= kv_norm(NBIN[t]) + WIDTH[t]
    return 22 <= k <= 25


def run(program, ds, alias_stacks=True, form=5):
    """Gradient of the MSE w.r.t. the first min(32, P) flat parameters and
    the MSE, by the register adjoint's code; (mse, grad[32]).  form=1 runs
    the register kernel's accumulator form instead (fused loads,
    no tape, no reverse sweep) and returns the MSE alone."""
    if form == 1:
        words = E.encoding(program, ds.num_features, 1)
        if len(words) == 0:
            raise ValueError("no accumulator form")
        fwd = [(int(w), 0xFFFFFFFF) for w in words]
        rev = []
    else:
        enc = E.encoding(program, ds.num_features, 5)
        if enc[0] == 0xFFFFFFFF:
            raise ValueError("no register adjoint form")
        code = enc[7:]
        n_fwd, n_rev = int(code[0]), int(code[1])
        # forward entries: (micro-op word, tape stores before | after << 16)
        fwd = [(int(code[2 + 2 * i]), int(code[3 + 2 * i])) for i in range(n_fwd)]
        r0 = 2 + 2 * n_fwd
        rev = [(int(code[r0 + 2 * i]), int(code[r0 + 1 + 2 * i])) for i in range(n_rev)]
    npts = ds.num_batches * 8
    ff = np.asarray(ds.feature_flat, f32).reshape(ds.num_batches, ds.num_features, 8)
    X = [ff[:, f, :].reshape(-1) for f in range(ds.num_features)]
    y = np.asarray(ds.target_batches, f32)
    consts = np.asarray(program.flatten_params(), f32)
    C = lambda i: np.full(npts, consts[i], f32)
    zero = np.zeros(npts, f32)
    A = [[zero] * WIDTH[t] for t in range(5)]
    S = [dict() for _ in range(5)]
    tape = {}

    def fetch(t, src, arg, w):
        if src == 0:
            return [X[arg + c] for c in range(w)]
        if src == 1:
            return [C(arg + c) for c in range(w)]
        return list(S[t][arg])

    def forward_op(kind, arg, t, k, W, nb):
        if _is_unary(t, k) and (arg >> 12) & 3:  # the operand's load, fused into the op (accumulator form)
            src1, off = (arg >> 12) & 3, arg & 0xFFF
            A[t] = [X[off + c] if src1 == 1 else C(off + c) for c in range(W)]
        if k == 0:
            A[t] = [X[arg + c] for c in range(W)]
        elif k == 1:
            A[t] = [C(arg + c) for c in range(W)]
        elif k == 2:
            S[t][arg & 15] = list(A[t])
            lt = (arg >> 4) & 7   # a load fused into the PUSH (uops.h push_load_arg)
            if lt:
                off, W2 = (arg >> 8) & 0xFFF, WIDTH[lt - 1]
                A[lt - 1] = [C(off + c) if (arg >> 7) & 1 else X[off + c] for c in range(W2)]

        elif k < 3 + 3 * nb:
            j, src = (k - 3) // 3, (k - 3) % 3
            B = fetch(t, src, arg, W)
            a = A[t]
            if j == 0:
                A[t] = [a[c] + B[c] for c in range(W)]
            elif j == 1:
                A[t] = [a[c] - B[c] for c in range(W)]
            elif j == 2:
                A[t] = [B[c] - a[c] for c in range(W)]
            elif t == SF:
                A[t] = [[a[0] * B[0], a[0] / B[0], B[0] / a[0]][j - 3]]
            elif t == SV3:
                A[t] = cross(a, B) if j == 3 else cross(B, a)
            else:
                n = 2 if t == SM2 else 3
                A[t] = mul_mat(a, B, n) if j == 3 else mul_mat(B, a, n)
        elif t == SF:
            u, a = k - 21, A[SF][0]
            A[SF] = [[_sin(a), _cos(a), _tr("exp", a), a * a, np.sqrt(a), _tr("log", a)][u]]
        elif t in (SV2, SV3):
            ks, kd, kn, km, kk = kv_scale(nb), kv_dot(nb), kv_norm(nb), kv_mulm(nb, W), kv_make(nb, W)
            if ks <= k < ks + 4:
                s = A[SF][0] if k == ks else fetch(SF, k - ks - 1, arg, 1)[0]
                A[t] = [A[t][c] * s for c in range(W)]
            elif kd <= k < kd + 3:
                B = fetch(t, k - kd, arg, W)
                d = A[t][0] * B[0] + A[t][1] * B[1]
                if W == 3:
                    d = d + A[t][2] * B[2]
                A[SF] = [d]
            elif k == kn:
                a = A[t]
                d = a[0] * a[0] + a[1] * a[1]
                if W == 3:
                    d = d + a[2] * a[2]
                A[SF] = [np.sqrt(d)]
            elif kn < k <= kn + W:
                A[SF] = [A[t][k - kn - 1]]
            elif km <= k < km + 4:
                tm, n = (SM2, 2) if W == 2 else (SM3, 3)
                M = A[tm] if k == km else fetch(tm, k - km - 1, arg, n * n)
                A[t] = mul_mat_vec(M, A[t], n)
            elif k == kk:
                A[t] = [S[SF][arg + c][0] for c in range(W - 1)] + [A[SF][0]]
        else:
            n = 2 if t == SM2 else 3
            tv = SV2 if n == 2 else SV3
            if 18 <= k < 22:
                s = A[SF][0] if k == 18 else fetch(SF, k - 19, arg, 1)[0]
                A[t] = [A[t][c] * s for c in range(W)]
            elif k == 22:
                A[SF] = [det(A[t], n)]
            elif k == 23:
                A[SF] = [A[t][0] + A[t][3]] if n == 2 else [(A[t][0] + A[t][4]) + A[t][8]]
            elif k == 24:
                A[t] = transpose(A[t], n)
            elif k == 25:
                A[t] = inverse(A[t], n)
            elif k == 26:
                cols = [S[tv][arg + c] for c in range(n - 1)] + [A[tv]]
                A[t] = [cols[c][r] for c in range(n) for r in range(n)]

    for word, tapes in fwd:
        kind, arg = word & 0xFF, word >> 8
        t = block(kind)
        k, W, nb = kind - BASE[t], WIDTH[t], NBIN[t]
        if kind == TAPE[t]:
            for c in range(W):
                tape[arg + c] = A[t][c]
            continue
        if tapes & 0xFFFF != 0xFFFF:   # the op's type's accumulator, stored before the op
            for c in range(W):
                tape[(tapes & 0xFFFF) + c] = A[t][c]
        forward_op(kind, arg, t, k, W, nb)
        if tapes >> 16 != 0xFFFF:      # and after it
            for c in range(W):
                tape[(tapes >> 16) + c] = A[t][c]

    pred = A[SF][0]
    valid = np.arange(npts) < ds.num_batches * 8
    diff = pred - y
    sse = float(np.sum(diff.astype(np.float64) ** 2))
    if form == 1:
        return sse / ds.num_samples
    # reverse sweep
    G = [[zero] * WIDTH[t] for t in range(5)]
    G[SF] = [(f32(2) * diff).astype(f32)]
    # a spilled value's adjoint takes its forward slot: the one micro-op that
    # pops the value reads it (in both sweeps) before its reverse writes the
    # adjoint, and nothing reads the slot's forward value after that
    GS = S if alias_stacks else [dict() for _ in range(5)]
    grad = np.zeros(32)
    def T(ref, w):  # a tape slot, or a feature / constant reference (uops.h kTapeRefX, kTapeRefC)
        if ref & 0x8000:
            return [X[(ref & 0x3FFF) + c] for c in range(w)]
        if ref & 0x4000:
            return [C((ref & 0x3FFF) + c) for c in range(w)]
        return [tape[ref + c] for c in range(w)]

    def to_const(arg, g, w):
        for c in range(w):
            if arg + c < 32:
                grad[arg + c] += float(np.sum(g[c][valid].astype(np.float64)))

    def send(t, src, arg, g, w):  # adjoint of a second operand
        if src == 1:
            to_const(arg, g, w)
        elif src == 2:
            GS[t][arg] = g

    for w0, w1 in rev:
        kind, arg = w0 & 0xFF, w0 >> 8
        ta, tb = w1 & 0xFFFF, w1 >> 16
        t = block(kind)
        k, W, nb = kind - BASE[t], WIDTH[t], NBIN[t]
        g = G[t]
        if k == 0:
            G[t] = [zero] * W
        elif k == 1:
            to_const(arg, g, W)
            G[t] = [zero] * W
        elif k == 2:
            lt = (arg >> 4) & 7
            if lt:  # the fused load ran after the PUSH: reverse it first
                if (arg >> 7) & 1:
                    to_const(arg >> 8, G[lt - 1], WIDTH[lt - 1])
                G[lt - 1] = [zero] * WIDTH[lt - 1]
                g = G[t]
            G[t] = [g[c] + GS[t][arg & 15][c] for c in range(W)]
        elif k < 3 + 3 * nb:
            j, src = (k - 3) // 3, (k - 3) % 3
            if j == 0:
                send(t, src, arg, list(g), W)
            elif j == 1:
                send(t, src, arg, [-x for x in g], W)
            elif j == 2:
                send(t, src, arg, list(g), W)
                G[t] = [-x for x in g]
            else:
                B = fetch(t, src, arg, W)
                if t == SF:
                    if j == 3:
                        send(t, src, arg, [g[0] * T(ta, 1)[0]], 1)
                        G[t] = [g[0] * B[0]]
                    elif j == 4:
                        q = g[0] / B[0]
                        send(t, src, arg, [-(q * T(ta, 1)[0])], 1)
                        G[t] = [q]
                    else:
                        q = g[0] / T(ta, 1)[0]
                        send(t, src, arg, [q], 1)
                        G[t] = [-(q * T(tb, 1)[0])]
                elif t == SV3:
                    a = T(ta, 3)
                    if j == 3:
                        send(t, src, arg, cross(g, a), 3)
                        G[t] = cross(B, g)
                    else:
                        send(t, src, arg, cross(a, g), 3)
                        G[t] = cross(g, B)
                else:
                    n = 2 if t == SM2 else 3
                    a = T(ta, n * n)
                    gt = transpose(g, n)
                    if j == 3:   # O = A B: dA = G B^T, dB = A^T G
                        send(t, src, arg, mul_mat(transpose(a, n), g, n), n * n)
                        G[t] = mul_mat(g, transpose(B, n), n)
                    else:        # O = B A: dB = G A^T, dA = B^T G
                        send(t, src, arg, mul_mat(g, transpose(a, n), n), n * n)
                        G[t] = mul_mat(transpose(B, n), g, n)
                    del gt
        elif t == SF:
            u = k - 21
            a = T(ta, 1)[0]
            G[SF] = [[g[0] * _cos(a), g[0] * (-_sin(a)), g[0] * a, g[0] * (f32(2) * a),
                      g[0] / (f32(2) * a), g[0] / a][u]]
        elif t in (SV2, SV3):
            ks, kd, kn, km, kk = kv_scale(nb), kv_dot(nb), kv_norm(nb), kv_mulm(nb, W), kv_make(nb, W)
            if ks <= k < ks + 4:
                a = T(ta, W)
                s = T(tb, 1)[0] if k == ks else fetch(SF, k - ks - 1, arg, 1)[0]
                gs = np.zeros(len(zero), f32)
                for c in range(W):
                    gs = gs + g[c] * a[c]
                if k == ks:
                    G[SF] = [G[SF][0] + gs]
                else:
                    send(SF, k - ks - 1, arg, [gs], 1)
                G[t] = [g[c] * s for c in range(W)]
            elif kd <= k < kd + 3:
                a = T(ta, W)
                B = fetch(t, k - kd, arg, W)
                gf = G[SF][0]
                G[t] = [g[c] + gf * B[c] for c in range(W)]
                send(t, k - kd, arg, [gf * a[c] for c in range(W)], W)
                G[SF] = [zero]
            elif k == kn:
                a = T(tb, W)
                d = a[0] * a[0] + a[1] * a[1]   # the norm, recomputed in the forward's operation order
                if W == 3:
                    d = d + a[2] * a[2]
                q = G[SF][0] / np.sqrt(d)
                G[t] = [g[c] + q * a[c] for c in range(W)]
                G[SF] = [zero]
            elif kn < k <= kn + W:
                c0 = k - kn - 1
                G[t] = [g[c] + G[SF][0] if c == c0 else g[c] for c in range(W)]
                G[SF] = [zero]
            elif km <= k < km + 4:
                tm, n = (SM2, 2) if W == 2 else (SM3, 3)
                v = T(ta, W)
                M = T(tb, n * n) if k == km else fetch(tm, k - km - 1, arg, n * n)
                gm = [g[r] * v[c] for c in range(n) for r in range(n)]
                if k == km:
                    G[tm] = [G[tm][i] + gm[i] for i in range(n * n)]
                else:
                    send(tm, k - km - 1, arg, gm, n * n)
                nv = []
                for c in range(n):
                    s = zero
                    for r in range(n):
                        s = s + M[n * c + r] * g[r]
                    nv.append(s)
                G[t] = nv
            elif k == kk:
                G[SF] = [G[SF][0] + g[W - 1]]
                for c in range(W - 1):
                    GS[SF][arg + c] = [g[c]]
                G[t] = [zero] * W
        else:
            n = 2 if t == SM2 else 3
            tv = SV2 if n == 2 else SV3
            if 18 <= k < 22:
                a = T(ta, W)
                s = T(tb, 1)[0] if k == 18 else fetch(SF, k - 19, arg, 1)[0]
                gs = np.zeros(len(zero), f32)
                for c in range(W):
                    gs = gs + g[c] * a[c]
                if k == 18:
                    G[SF] = [G[SF][0] + gs]
                else:
                    send(SF, k - 19, arg, [gs], 1)
                G[t] = [g[c] * s for c in range(W)]
            elif k == 22:
                m = T(ta, W)
                gf = G[SF][0]
                G[t] = [g[n * c + r] + gf * cofactor(m, n, r, c) for c in range(n) for r in range(n)]
                G[SF] = [zero]
            elif k == 23:
                gf = G[SF][0]
                G[t] = [g[i] + gf if i % (n + 1) == 0 else g[i] for i in range(W)]
                G[SF] = [zero]
            elif k == 24:
                G[t] = transpose(g, n)
            elif k == 25:
                o, m = T(ta, W), T(tb, W)
                sing = np.abs(det(m, n)) < f32(1e-9)
                h = mul_mat(transpose(o, n), g, n)
                d = mul_mat(h, transpose(o, n), n)
                G[t] = [np.where(sing, f32(0), -x).astype(f32) for x in d]
            elif k == 26:
                G[tv] = [G[tv][r] + g[n * (n - 1) + r] for r in range(n)]
                for c in range(n - 1):
                    GS[tv][arg + c] = [g[n * c + r] for r in range(n)]
                G[t] = [zero] * W
    return sse / ds.num_samples, grad / ds.num_samples
