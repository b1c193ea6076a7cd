// kernels_adj.cu -- the register adjoint: MSE and d(MSE)/d(constants) with
// the forward and the reverse sweep both on accumulator registers.
//
// Replaces compute_mse_with_gradient (src/engine/eval/evaluator.rs:177-224)
// and its one dual-number pass per flat parameter (eval_simd_dual,
// evaluator.rs:228-388) for the programs the accumulator machine takes.
// Per tile of 32*P points a warp runs
//   forward  the accumulator form (acc_ops.cuh) with a load after a PUSH
//            fused into the PUSH and every PUSH to its own stack slot; the
//            forward values the reverse rules read go to a per-warp tape in
//            shared memory, stored by the op's own entry (before or after
//            the op) or by a TAPE micro-op;
//   seed     G_F = 2 (pred - y) on counted points (evaluator.rs:207);
//   reverse  the reverse entries (uops.h, kAdjHeaderWords): each maps the
//            adjoint accumulators G_t of the micro-op's output to those of
//            its inputs.  A second operand's adjoint goes to the constant
//            sums (LoadConst), to the adjoint stack slot of its PUSH (a
//            spilled value, which takes the value's own slot), or nowhere
//            (a feature).
// The reverse rules follow autodiff.rs's forward rules (product and quotient
// rules, g/(2 sqrt x), norms through sqrt of dot); InverseM2/M3, whose dual
// rule is a no-op in the reference (src/domains/linalg/mod.rs:643,687), get
// the exact adjoint -A^-T G A^-T, zero on the singular branch.  The tape is
// recorded and consumed tile by tile: the population x points x length tape
// is never stored.  The encoder's tape slot conventions are listed with
// AdjEmitter (encoder.cpp).
#include <cuda_runtime.h>
#include <float.h>

#include "acc_ops.cuh"
#include "kernels.h"
#include "kernels_common.cuh"

namespace rsr {

constexpr uint32_t kAdjParams = 32;

// The tape lives in tensor memory (tmem.cuh): one block per SM allocates
// all 512 columns of its SM's 128 lanes; warp w owns lanes 32 (w % 4) ..
// +31, one lane per thread, and the (w / 4)-th run of a.tmem_cols columns
// (512 / (warps / 4)); a tape slot is P consecutive columns of the thread's
// lane.  The launch pads each block's shared memory to more than half an
// SM's (enqueue_plan), so no two blocks that allocate share an SM and the
// allocation never waits.

// Reverse-sweep access: the forward machine's operand fetches (features,
// constants, forward stack values), the adjoint stacks, the tape and the
// lane's gradient sums.
template <int P>
struct RevIO : AccIO<P> {
    // adjoint stacks in the interleaved lane layout (blocks of 32*P floats),
    // at this lane's first value
    float *gstk[N_STACKS];  // adjoint stacks, block (slot*W + c)
    uint32_t tm;            // tensor-memory tape: this warp's lanes, column 0
    float *gacc;            // this lane's f32 gradient sums: gacc[k*32]
    uint32_t valid;         // bit q: value q of the lane is a counted point
    // a tape reference (uops.h, kTapeRefX): a tape slot, or the feature or
    // constant the forward value was loaded from
    __device__ __forceinline__ Vf<P> T(uint32_t ref) const {
        if (ref & kTapeRefX) return this->X(ref & kTapeRefIndex);
        if (ref & kTapeRefC) return this->C(ref & kTapeRefIndex);
        return tm_ld<P>(tm + ref * (uint32_t)P);
    }
    __device__ __forceinline__ void put_tape(uint32_t slot, const Vf<P> &v) const {
        tm_st<P>(tm + slot * (uint32_t)P, v);
    }
    template <int W>
    __device__ __forceinline__ Vf<P> GS(int t, uint32_t slot, int c) const {
        return lds_lane<P>(gstk[t] + (slot * W + c) * 32u * P);
    }
    template <int W>
    __device__ __forceinline__ void put_g(int t, uint32_t slot, int c, const Vf<P> &v) const {
        sts_lane<P>(gstk[t] + (slot * W + c) * 32u * P, v);
    }
    // adds the lane's counted points of g to the sum of flat parameter k
    // (points past the dataset's end may carry 0*inf = NaN adjoints)
    __device__ __forceinline__ void grad_add(uint32_t k, const Vf<P> &g) const {
        if (k >= kAdjParams) return;
        float s = 0.0f;
#pragma unroll
        for (int q = 0; q < P; ++q)
            if ((valid >> q) & 1u) s = s + g.v[q];
        gacc[k * 32] += s;
    }
};

// kStackWidth for device code
__device__ __forceinline__ constexpr uint32_t type_width(int t) {
    return t == SF ? 1u : t == SV2 ? 2u : t == SV3 ? 3u : t == SM2 ? 4u : 9u;
}

template <int P, int W>
__device__ __forceinline__ void zero_acc(Vf<P> *G) {
#pragma unroll
    for (int c = 0; c < W; ++c) G[c] = splat<P>(0.0f);
}

template <int P, int W>
__device__ __forceinline__ void load_tape(Vf<P> *v, const RevIO<P> &io, uint32_t slot) {
#pragma unroll
    for (int c = 0; c < W; ++c) v[c] = io.T(slot + c);
}

// The adjoint of a second operand from source SRC: a constant's goes to the
// parameter sums, a spilled value's to its adjoint stack slot (its PUSH adds
// it back), a feature's nowhere.
template <int P, int W, int SRC>
__device__ __forceinline__ void send(const RevIO<P> &io, int t, uint32_t arg, const Vf<P> *gb) {
    if constexpr (SRC == SRC_C) {
#pragma unroll
        for (int c = 0; c < W; ++c) io.grad_add(arg + c, gb[c]);
    } else if constexpr (SRC == SRC_S) {
#pragma unroll
        for (int c = 0; c < W; ++c) io.template put_g<W>(t, arg, c, gb[c]);
    }
}

// out(r,c) = sum_j G(r,j) B(c,j) = (G B^T)(r,c), column-major N x N.
template <int P, int N>
__device__ __forceinline__ void mm_nt(const Vf<P> *G, const Vf<P> *B, Vf<P> *out) {
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
        for (int c = 0; c < N; ++c) {
            Vf<P> s = splat<P>(0.0f);
#pragma unroll
            for (int j = 0; j < N; ++j) s = s + G[N * j + r] * B[N * j + c];
            out[N * c + r] = s;
        }
}
// out(r,c) = sum_j A(j,r) G(j,c) = (A^T G)(r,c).
template <int P, int N>
__device__ __forceinline__ void mm_tn(const Vf<P> *A, const Vf<P> *G, Vf<P> *out) {
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
        for (int c = 0; c < N; ++c) {
            Vf<P> s = splat<P>(0.0f);
#pragma unroll
            for (int j = 0; j < N; ++j) s = s + A[N * r + j] * G[N * c + j];
            out[N * c + r] = s;
        }
}

// Reverse of a load into the accumulator of type t: a constant's adjoint
// goes to the parameter sums, and the value the load overwrote is dead.
template <int PROF, int P, int t>
__device__ __forceinline__ void rev_load_t(Acc<PROF, P> &g, const RevIO<P> &io, uint32_t is_const, uint32_t off) {
    if constexpr (((kProfileTypes[PROF] >> t) & 1u) != 0u) {
        constexpr int W = kStackWidth[t];
        Vf<P> *G = acc_of<PROF, P, t>(g);
        if (is_const) {
#pragma unroll
            for (int c = 0; c < W; ++c) io.grad_add(off + c, G[c]);
        }
        zero_acc<P, W>(G);
    }
}
template <int PROF, int P>
__device__ __forceinline__ void rev_load_any(Acc<PROF, P> &g, const RevIO<P> &io, uint32_t t, uint32_t is_const,
                                             uint32_t off) {
    switch (t) {
        case SF: rev_load_t<PROF, P, SF>(g, io, is_const, off); break;
        case SV2: rev_load_t<PROF, P, SV2>(g, io, is_const, off); break;
        case SV3: rev_load_t<PROF, P, SV3>(g, io, is_const, off); break;
        case SM2: rev_load_t<PROF, P, SM2>(g, io, is_const, off); break;
        default: rev_load_t<PROF, P, SM3>(g, io, is_const, off); break;
    }
}

// Reverse of one micro-op of kind K: g holds the adjoints of the machine's
// accumulators after the micro-op and is left holding those before it.
template <int PROF, int P, int K>
__device__ __forceinline__ void rev_op(Acc<PROF, P> &g, const RevIO<P> &io, uint32_t arg, uint32_t w1) {
    constexpr int t = K >= K_M3 ? SM3 : K >= K_M2 ? SM2 : K >= K_V3 ? SV3 : K >= K_V2 ? SV2 : SF;
    if constexpr (((kProfileTypes[PROF] >> t) & 1u) != 0u) {
        constexpr int W = kStackWidth[t];
        constexpr int k = K - kBlockBase[t];
        constexpr int nb = kBinOps[t];
        Vf<P> *G = acc_of<PROF, P, t>(g);
        const uint32_t ta = w1 & 0xFFFFu, tb = w1 >> 16;
        if constexpr (k == KV_LDX) {
            zero_acc<P, W>(G);
        } else if constexpr (k == KV_LDC) {
#pragma unroll
            for (int c = 0; c < W; ++c) io.grad_add(arg + c, G[c]);
            zero_acc<P, W>(G);
        } else if constexpr (k == KV_PUSH) {
            // a load fused into the PUSH ran after it: reverse it first
            const uint32_t lt = (arg >> 4) & 7u, slot = arg & 15u;
            if (lt) rev_load_any<PROF, P>(g, io, lt - 1u, (arg >> 7) & 1u, (arg >> 8) & ((1u << kLdOffsetBits) - 1u));
#pragma unroll
            for (int c = 0; c < W; ++c) G[c] = G[c] + io.template GS<W>(t, slot, c);
        } else if constexpr (k >= KV_BIN && k < KV_BIN + 3 * nb) {
            constexpr int j = (k - KV_BIN) / 3, src = (k - KV_BIN) % 3;
            constexpr int op = bin_code<t, j>();
            if constexpr (op == BIN_ADD) {
                send<P, W, src>(io, t, arg, G);
            } else if constexpr (op == BIN_SUB || op == BIN_RSUB) {
                Vf<P> n[W];
#pragma unroll
                for (int c = 0; c < W; ++c) n[c] = -G[c];
                if constexpr (op == BIN_SUB) {
                    send<P, W, src>(io, t, arg, n);
                } else {
                    send<P, W, src>(io, t, arg, G);
#pragma unroll
                    for (int c = 0; c < W; ++c) G[c] = n[c];
                }
            } else if constexpr (op == BIN_MUL) {        // a * b: tape a
                Vf<P> b;
                fetch<P, 1, src>(&b, io, t, arg);
                const Vf<P> gb = G[0] * io.T(ta);
                send<P, 1, src>(io, t, arg, &gb);
                G[0] = G[0] * b;
            } else if constexpr (op == BIN_DIV) {        // a / b: tape the quotient
                Vf<P> b;
                fetch<P, 1, src>(&b, io, t, arg);
                const Vf<P> q = G[0] / b;
                const Vf<P> gb = -(q * io.T(ta));
                send<P, 1, src>(io, t, arg, &gb);
                G[0] = q;
            } else if constexpr (op == BIN_RDIV) {       // b / a: tape a, the quotient
                const Vf<P> q = G[0] / io.T(ta);
                send<P, 1, src>(io, t, arg, &q);
                G[0] = -(q * io.T(tb));
            } else if constexpr (op == BIN_CROSS || op == BIN_RCROSS) {  // tape a
                Vf<P> a[3], b[3], gb[3];
                load_tape<P, 3>(a, io, ta);
                fetch<P, 3, src>(b, io, t, arg);
                if constexpr (op == BIN_CROSS) {   // o = a x b: da = b x g, db = g x a
                    cross3(G, a, gb);
                    cross3(b, G, G);
                } else {                           // o = b x a: db = a x g, da = g x b
                    cross3(a, G, gb);
                    cross3(G, b, G);
                }
                send<P, 3, src>(io, t, arg, gb);
            } else {                                     // matrix products: tape a
                constexpr int N = W == 4 ? 2 : 3;
                Vf<P> a[W], b[W], gb[W], ga[W];
                load_tape<P, W>(a, io, ta);
                fetch<P, W, src>(b, io, t, arg);
                if constexpr (op == BIN_MMUL) {    // o = a b: da = g b^T, db = a^T g
                    mm_tn<P, N>(a, G, gb);
                    mm_nt<P, N>(G, b, ga);
                } else {                           // o = b a: db = g a^T, da = b^T g
                    mm_nt<P, N>(G, a, gb);
                    mm_tn<P, N>(b, G, ga);
                }
                send<P, W, src>(io, t, arg, gb);
#pragma unroll
                for (int c = 0; c < W; ++c) G[c] = ga[c];
            }
        } else if constexpr (t == SF) {                  // unary: sin cos exp sqr sqrt ln
            constexpr int u = k - (K_F_UN - K_F);
            const Vf<P> v = io.T(ta);  // the operand, or the result for exp and sqrt
            if constexpr (u == 0) G[0] = G[0] * vcos(v);
            else if constexpr (u == 1) G[0] = G[0] * (-vsin(v));
            else if constexpr (u == 2) G[0] = G[0] * v;
            else if constexpr (u == 3) G[0] = G[0] * (splat<P>(2.0f) * v);
            else if constexpr (u == 4) G[0] = G[0] / (splat<P>(2.0f) * v);
            else if constexpr (u == 5) G[0] = G[0] / v;
        } else if constexpr (t == SV2 || t == SV3) {
            constexpr int ks = kv_scale(nb), kd = kv_dot(nb), kn = kv_norm(nb), km = kv_mulm(nb, W),
                          kk = kv_make(nb, W);
            if constexpr (k >= ks && k < ks + 4) {       // SCALE {A X C S}: tape the vector (and A_F)
                Vf<P> a[W], s;
                load_tape<P, W>(a, io, ta);
                if constexpr (k == ks) s = io.T(tb);
                else fetch<P, 1, k - ks - 1>(&s, io, SF, arg);
                Vf<P> gs = splat<P>(0.0f);
#pragma unroll
                for (int c = 0; c < W; ++c) gs = gs + G[c] * a[c];
                if constexpr (k == ks) g.F[0] = g.F[0] + gs;
                else send<P, 1, k - ks - 1>(io, SF, arg, &gs);
#pragma unroll
                for (int c = 0; c < W; ++c) G[c] = G[c] * s;
            } else if constexpr (k >= kd && k < kd + 3) { // DOT {X C S}: tape the vector
                Vf<P> a[W], b[W], gb[W];
                load_tape<P, W>(a, io, ta);
                fetch<P, W, k - kd>(b, io, t, arg);
                const Vf<P> gf = g.F[0];
#pragma unroll
                for (int c = 0; c < W; ++c) {
                    G[c] = G[c] + gf * b[c];
                    gb[c] = gf * a[c];
                }
                send<P, W, k - kd>(io, t, arg, gb);
                g.F[0] = splat<P>(0.0f);
            } else if constexpr (k == kn) {              // NORM: tape the vector; the norm is recomputed
                Vf<P> v[W];
                load_tape<P, W>(v, io, tb);
                Vf<P> nrm;
                if constexpr (W == 2) nrm = norm2(v); else nrm = norm3(v);  // the forward's value, bit for bit
                const Vf<P> q = g.F[0] / nrm;
#pragma unroll
                for (int c = 0; c < W; ++c) G[c] = G[c] + q * v[c];
                g.F[0] = splat<P>(0.0f);
            } else if constexpr (k > kn && k <= kn + W) { // GET x/y/z
                G[k - kn - 1] = G[k - kn - 1] + g.F[0];
                g.F[0] = splat<P>(0.0f);
            } else if constexpr (k >= km && k < km + 4) { // MULM {A X C S}: tape the vector (and A_M)
                constexpr int tm = W == 2 ? SM2 : SM3;
                constexpr int MW = W * W;
                if constexpr (((kProfileTypes[PROF] >> tm) & 1u) != 0u || k != km) {
                    Vf<P> v[W], m[MW], gm[MW];
                    load_tape<P, W>(v, io, ta);
                    if constexpr (k == km) load_tape<P, MW>(m, io, tb);
                    else fetch<P, MW, k - km - 1>(m, io, tm, arg);
#pragma unroll
                    for (int c = 0; c < W; ++c)
#pragma unroll
                        for (int r = 0; r < W; ++r) gm[W * c + r] = G[r] * v[c];
                    if constexpr (k == km) {
                        if constexpr (((kProfileTypes[PROF] >> tm) & 1u) != 0u) {
                            Vf<P> *GM = acc_of<PROF, P, tm>(g);
#pragma unroll
                            for (int i = 0; i < MW; ++i) GM[i] = GM[i] + gm[i];
                        }
                    } else {
                        send<P, MW, k - km - 1>(io, tm, arg, gm);
                    }
                    Vf<P> nv[W];
#pragma unroll
                    for (int c = 0; c < W; ++c) {
                        Vf<P> s = splat<P>(0.0f);
#pragma unroll
                        for (int r = 0; r < W; ++r) s = s + m[W * c + r] * G[r];
                        nv[c] = s;
                    }
#pragma unroll
                    for (int c = 0; c < W; ++c) G[c] = nv[c];
                }
            } else if constexpr (k == kk) {              // MAKE from F stack slots + A_F
                g.F[0] = g.F[0] + G[W - 1];
#pragma unroll
                for (int c = 0; c + 1 < W; ++c) io.template put_g<1>(SF, arg + c, 0, G[c]);
                zero_acc<P, W>(G);
            }
        } else {  // M2 / M3
            constexpr int N = W == 4 ? 2 : 3;
            constexpr int tv = W == 4 ? SV2 : SV3;
            if constexpr (k >= KM_SCALE && k < KM_SCALE + 4) {
                Vf<P> a[W], s;
                load_tape<P, W>(a, io, ta);
                if constexpr (k == KM_SCALE) s = io.T(tb);
                else fetch<P, 1, k - KM_SCALE - 1>(&s, io, SF, arg);
                Vf<P> gs = splat<P>(0.0f);
#pragma unroll
                for (int c = 0; c < W; ++c) gs = gs + G[c] * a[c];
                if constexpr (k == KM_SCALE) g.F[0] = g.F[0] + gs;
                else send<P, 1, k - KM_SCALE - 1>(io, SF, arg, &gs);
#pragma unroll
                for (int c = 0; c < W; ++c) G[c] = G[c] * s;
            } else if constexpr (k == KM_DET) {          // tape the matrix
                Vf<P> m[W];
                load_tape<P, W>(m, io, ta);
                const Vf<P> gf = g.F[0];
                if constexpr (N == 2) {
                    G[0] = G[0] + gf * m[3];
                    G[3] = G[3] + gf * m[0];
                    G[1] = G[1] + (-(gf * m[2]));
                    G[2] = G[2] + (-(gf * m[1]));
                } else {
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                            const Vf<P> cof = m[3 * c1 + r1] * m[3 * c2 + r2] - m[3 * c2 + r1] * m[3 * c1 + r2];
                            G[3 * c + r] = G[3 * c + r] + gf * cof;
                        }
                }
                g.F[0] = splat<P>(0.0f);
            } else if constexpr (k == KM_TRACE) {
#pragma unroll
                for (int i = 0; i < N; ++i) G[(N + 1) * i] = G[(N + 1) * i] + g.F[0];
                g.F[0] = splat<P>(0.0f);
            } else if constexpr (k == KM_TRANSPOSE) {
                Vf<P> tr[W];
#pragma unroll
                for (int r = 0; r < N; ++r)
#pragma unroll
                    for (int c = 0; c < N; ++c) tr[N * r + c] = G[N * c + r];
#pragma unroll
                for (int i = 0; i < W; ++i) G[i] = tr[i];
            } else if constexpr (k == KM_INVERSE) {      // tape the inverse, the matrix
                Vf<P> o[W], m[W], h[W];
                load_tape<P, W>(o, io, ta);
                load_tape<P, W>(m, io, tb);
                Vf<P> det;
                if constexpr (N == 2) det = det_m2(m); else det = det_m3(m);
                // h = O^T G, then dA = -(h O^T), zero where singular
#pragma unroll
                for (int i = 0; i < N; ++i)
#pragma unroll
                    for (int l = 0; l < N; ++l) {
                        Vf<P> s = splat<P>(0.0f);
#pragma unroll
                        for (int q = 0; q < N; ++q) s = s + o[N * i + q] * G[N * l + q];
                        h[N * l + i] = s;
                    }
#pragma unroll
                for (int i = 0; i < N; ++i)
#pragma unroll
                    for (int j = 0; j < N; ++j) {
                        Vf<P> s = splat<P>(0.0f);
#pragma unroll
                        for (int l = 0; l < N; ++l) s = s + h[N * l + i] * o[N * l + j];
                        Vf<P> d;
#pragma unroll
                        for (int q = 0; q < P; ++q) d.v[q] = fabsf(det.v[q]) < 1e-9f ? 0.0f : -s.v[q];
                        m[N * j + i] = d;  // m is no longer needed
                    }
#pragma unroll
                for (int i = 0; i < W; ++i) G[i] = m[i];
            } else if constexpr (k == KM_MAKE) {         // columns: vector stack slots + A_V
                if constexpr (((kProfileTypes[PROF] >> tv) & 1u) != 0u) {
                    Vf<P> *GV = acc_of<PROF, P, tv>(g);
#pragma unroll
                    for (int r = 0; r < N; ++r) GV[r] = GV[r] + G[N * (N - 1) + r];
#pragma unroll
                    for (int col = 0; col + 1 < N; ++col)
#pragma unroll
                        for (int r = 0; r < N; ++r) io.template put_g<N>(tv, arg + col, r, G[N * col + r]);
                }
                zero_acc<P, W>(G);
            }
        }
    }
}

// Forward: a micro-op of kind K, or a TAPE store of its block's accumulator.
template <int PROF, int P, int t>
__device__ __forceinline__ void tape_store(Acc<PROF, P> &a, const RevIO<P> &io, uint32_t slot) {
    if constexpr (((kProfileTypes[PROF] >> t) & 1u) != 0u) {
        constexpr int W = kStackWidth[t];
        const Vf<P> *A = acc_of<PROF, P, t>(a);
#pragma unroll
        for (int c = 0; c < W; ++c) io.put_tape(slot + c, A[c]);
    }
}

// A forward entry: the op's type's accumulator stored to the tape before
// and/or after the op (uops.h, kNoTape).
template <int PROF, int P, int K>
__device__ __forceinline__ void fwd_op(Acc<PROF, P> &a, const RevIO<P> &io, uint32_t arg, uint32_t tapes) {
    constexpr int t = K >= K_M3 ? SM3 : K >= K_M2 ? SM2 : K >= K_V3 ? SV3 : K >= K_V2 ? SV2 : SF;
    if ((tapes & kNoTape) != kNoTape) tape_store<PROF, P, t>(a, io, tapes & kNoTape);
    acc_op<PROF, P, K>(a, io, arg);
    if ((tapes >> 16) != kNoTape) tape_store<PROF, P, t>(a, io, tapes >> 16);
}

#define RSR_F(K) case (K): fwd_op<PROF, P, (K)>(a, io, arg, tapes); break;
#define RSR_R(K) case (K): rev_op<PROF, P, (K)>(g, io, arg, w1); break;
#define RSR_X4(M, K) M(K) M(K + 1) M(K + 2) M(K + 3)
#define RSR_X9(M, K) RSR_X4(M, K) RSR_X4(M, K + 4) M(K + 8)
#define RSR_X27(M, K) RSR_X9(M, K) RSR_X9(M, K + 9) RSR_X9(M, K + 18)
#define RSR_X34(M, K) RSR_X27(M, K) RSR_X4(M, K + 27) M(K + 31) M(K + 32) M(K + 33)
// The kinds of each profile's blocks (F 0..26, V2 32..58, V3 64..97, M2
// 104..130, M3 136..162): a profile's switch lists only its own, and an
// instance leaves out the handler sets its launch's programs do not use
// (OMIT bit 0: the unary Float ops; bit 1, F+V3: the mat-vec products whose
// matrix is a feature, a constant or a spilled value), as the register
// kernel's instances do.
#define RSR_ADJ_F(M) RSR_X27(M, K_F)
#define RSR_ADJ_F_NU(M) RSR_X9(M, K_F) RSR_X9(M, K_F + 9) M(K_F + 18) M(K_F + 19) M(K_F + 20)
#define RSR_ADJ_V3(M) RSR_X34(M, K_V3)
#define RSR_ADJ_V3_NM(M) RSR_X27(M, K_V3) M(K_V3 + 27) M(K_V3 + 28) M(K_V3 + 29) M(K_V3 + 33)
static_assert(kv_mulm(5, 3) == 29 && kv_make(5, 3) == 33, "Vec3 block: mat-vec kinds at 29..32");
#define RSR_SWITCH(M, EXTRA)                                                                          \
    if constexpr (PROF == P_F && (OMIT & 1)) {                                                        \
        switch (kind) { EXTRA RSR_ADJ_F_NU(M) default: break; }                                       \
    } else if constexpr (PROF == P_F) {                                                               \
        switch (kind) { EXTRA RSR_ADJ_F(M) default: break; }                                          \
    } else if constexpr (PROF == P_FV3 && (OMIT & 3) == 3) {                                          \
        switch (kind) { EXTRA RSR_ADJ_F_NU(M) RSR_ADJ_V3_NM(M) default: break; }                      \
    } else if constexpr (PROF == P_FV3 && (OMIT & 1)) {                                               \
        switch (kind) { EXTRA RSR_ADJ_F_NU(M) RSR_ADJ_V3(M) default: break; }                         \
    } else if constexpr (PROF == P_FV3 && (OMIT & 2)) {                                               \
        switch (kind) { EXTRA RSR_ADJ_F(M) RSR_ADJ_V3_NM(M) default: break; }                         \
    } else if constexpr (PROF == P_FV3) {                                                             \
        switch (kind) { EXTRA RSR_ADJ_F(M) RSR_ADJ_V3(M) default: break; }                            \
    } else if constexpr (PROF == P_FV2M2 && (OMIT & 1)) {                                             \
        switch (kind) { EXTRA RSR_ADJ_F_NU(M) RSR_X27(M, K_V2) RSR_X27(M, K_M2) default: break; }     \
    } else if constexpr (PROF == P_FV2M2) {                                                           \
        switch (kind) { EXTRA RSR_ADJ_F(M) RSR_X27(M, K_V2) RSR_X27(M, K_M2) default: break; }        \
    } else {                                                                                          \
        switch (kind) { EXTRA RSR_ADJ_F(M) RSR_ADJ_V3(M) RSR_X27(M, K_M3) default: break; }           \
    }
#define RSR_TAPES                                                            \
    case kTapeKind[SF]: tape_store<PROF, P, SF>(a, io, arg); break;          \
    case kTapeKind[SV2]: tape_store<PROF, P, SV2>(a, io, arg); break;        \
    case kTapeKind[SV3]: tape_store<PROF, P, SV3>(a, io, arg); break;        \
    case kTapeKind[SM2]: tape_store<PROF, P, SM2>(a, io, arg); break;        \
    case kTapeKind[SM3]: tape_store<PROF, P, SM3>(a, io, arg); break;
#define RSR_NONE

// Forward entries are (word, tape stores); the next entry is read while the
// current one runs.
template <int PROF, int P, int OMIT>
__device__ __forceinline__ void run_forward(Acc<PROF, P> &a, const RevIO<P> &io, const uint32_t *code, uint32_t n) {
    uint32_t w = code[0], tapes = code[1];
    for (uint32_t pc = 0; pc < n; ++pc) {
        const uint32_t wn = code[2 * pc + 2], tn = code[2 * pc + 3];
        const uint32_t arg = w >> 8, kind = w & 0xFFu;
        RSR_SWITCH(RSR_F, RSR_TAPES)
        w = wn;
        tapes = tn;
    }
}

// The next entry is read while the current one runs (the code ends with two
// pad words).
template <int PROF, int P, int OMIT>
__device__ __forceinline__ void run_reverse(Acc<PROF, P> &g, const RevIO<P> &io, const uint32_t *rev, uint32_t n) {
    uint32_t w0 = rev[0], w1 = rev[1];
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t w0n = rev[2 * i + 2], w1n = rev[2 * i + 3];
        const uint32_t arg = w0 >> 8, kind = w0 & 0xFFu;
        RSR_SWITCH(RSR_R, RSR_NONE)
        w0 = w0n;
        w1 = w1n;
    }
}

#undef RSR_NONE
#undef RSR_TAPES
#undef RSR_SWITCH
#undef RSR_ADJ_F
#undef RSR_ADJ_F_NU
#undef RSR_ADJ_V3
#undef RSR_ADJ_V3_NM
#undef RSR_X34
#undef RSR_X27
#undef RSR_X9
#undef RSR_X4
#undef RSR_R
#undef RSR_F

// Block-cooperative persistent kernel, one block per SM: its warps take the
// tiles of one work item (one program on a chunk of points).  Shared
// memory: block header (code | constants | meta | cross-warp sums), then
// one region per warp: stacks (then adjoint stacks) | gradient sums | Kahan
// state.  The tape is in tensor memory, a.tmem_cols columns per warp.
// Warps of a block of instance (PROF, P), one block per SM: a multiple of
// 4, at most 16.  More warps than the instance's registers allow unspilled
// pay: the extra warps hide more of the dispatch latency than the spill
// costs.  F+V3 at 8 points per lane: 168 registers at 12 warps, 128 with
// ~250 bytes of spill at 16 (vector workload gradient 17.7 ms against 22.4
// ms); F+V2+M2 and F+V3+M3 at 4 points likewise at 16 and 12 warps (matrix
// workload 17.0 against 18.7 ms).
template <int PROF, int P>
__host__ __device__ constexpr int adj_warps() {
    if constexpr (PROF == P_FV3M3) return P >= 4 ? 12 : 16;
    else return 16;
}

template <int PROF, int P, int OMIT>
__global__ void __launch_bounds__(adj_warps<PROF, P>() * 32, 1) adj_eval_kernel(const LaunchArgs a) {
    extern __shared__ __align__(16) float smem[];
    if (a.run_if && *a.run_if == 0u) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    uint32_t *scode = reinterpret_cast<uint32_t *>(smem);
    float *sconst = smem + ((a.smem_code_words + 2u + 3u) & ~3u);  // code and its two pad words
    uint32_t *meta = reinterpret_cast<uint32_t *>(sconst + ((a.smem_const_floats + 3u) & ~3u));  // [0] item, [1] tape
    double *red = reinterpret_cast<double *>(meta + 4);  // [part][warp][1 + kAdjParams]
    float *wbase = smem + a.block_hdr_floats + (size_t)warp * a.region_floats;

    // the block takes all of the SM's tensor memory; warp w owns lanes
    // 32 (w % 4) .. +31 (its quadrant) and the (w / 4)-th share of columns
    if (warp == 0) tm_alloc(&meta[1], 512u);
    tm_fence_before_sync();
    __syncthreads();
    tm_fence_after_sync();
    RevIO<P> io;
    io.consts = sconst;
    io.tm = meta[1] + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(warp >> 2) * a.tmem_cols;

    for (;;) {
        if (threadIdx.x == 0) meta[0] = atomicAdd(a.item_counter, 1u);
        __syncthreads();
        const uint32_t item_id = meta[0];
        if (item_id >= a.n_items) break;
        const WorkItem it = a.items[item_id];
        if (a.active && !a.active[it.prog_begin]) {
            __syncthreads();  // meta[0] is rewritten by the next item fetch
            continue;
        }
        const ProgDesc pd = a.progs[it.prog_begin];
        // this program's warp region: stacks | sums (n_tape: stack depths,
        // 5 bits per type); the launch's region_floats is the largest of its
        // programs'
        {
            const uint32_t l0 = lane_point<P>(lane, 0);
            uint32_t off = 0;
            // A spilled value's adjoint takes the value's own slot: the one
            // micro-op that pops the value reads it into registers (in both
            // sweeps) before its reverse writes the adjoint, and no later
            // reverse step reads the forward value (every PUSH has its own slot).
#pragma unroll
            for (int t = 0; t < N_STACKS; ++t) {
                io.stk[t] = wbase + off + l0;
                io.gstk[t] = io.stk[t];
                off += ((pd.n_tape >> (5 * t)) & 31u) * type_width(t) * 32u * P;
            }
            io.gacc = wbase + off + lane;
        }
        const uint32_t np = min(pd.n_consts, kAdjParams);
        float *kahan = io.gacc - lane + np * 32u;  // [2][32], after the program's own gradient sums
        for (uint32_t i = threadIdx.x; i < pd.uop_len; i += blockDim.x) scode[i] = __ldg(a.code + pd.uop_off + i);
        if (threadIdx.x == 0) scode[pd.uop_len] = scode[pd.uop_len + 1] = 0u;  // prefetch pads of the loops
        for (uint32_t i = threadIdx.x; i < pd.n_consts; i += blockDim.x) sconst[i] = __ldg(a.consts + pd.const_off + i);
        for (uint32_t k = 0; k < np; ++k) io.gacc[k * 32] = 0.0f;
        kahan[lane] = 0.0f;
        kahan[32 + lane] = 0.0f;
        __syncthreads();
        const DatasetDesc ds = a.datasets[pd.dataset];
        io.stride = (uint32_t)ds.stride;
        const uint32_t n_fwd = scode[0], n_rev = scode[1];
        const uint32_t *fwd = scode + kAdjHeaderWords, *rev = fwd + 2 * n_fwd;
        // The item's parts (kPartPoints points each) one after another; a
        // warp takes the same tiles of a part, and sums them the same way,
        // whatever the item's size, so a program's partial sums do not
        // depend on how its batch was cut into items.
        constexpr uint32_t part_tiles = kPartPoints / (32u * P);
        const uint32_t n_parts = (it.tile_end - it.tile_begin + part_tiles - 1) / part_tiles;
        for (uint32_t part = 0; part < n_parts; ++part) {
            const uint32_t part_end = min(it.tile_end, it.tile_begin + (part + 1) * part_tiles);
            for (uint32_t tile = it.tile_begin + part * part_tiles + warp; tile < part_end; tile += nw) {
                const uint64_t t0 = (uint64_t)tile * (32u * P);
                const uint64_t p0 = t0 + lane_point<P>(lane, 0);
                io.xl = ds.x + p0;
                uint32_t valid = 0;
#pragma unroll
                for (int q = 0; q < P; ++q) valid |= (t0 + lane_point<P>(lane, q) < ds.n_eval ? 1u : 0u) << q;
                io.valid = valid;
                Acc<PROF, P> acc;
                run_forward<PROF, P, OMIT>(acc, io, fwd, n_fwd);
                tm_wait_st();  // the tape stores land before the reverse sweep reads them
                const Vf<P> y = load_lane<P>(ds.y + p0);
                Acc<PROF, P> g;
                g.F[0] = splat<P>(0.0f);
                if constexpr (Types<PROF>::V2) zero_acc<P, 2>(g.V2);
                if constexpr (Types<PROF>::V3) zero_acc<P, 3>(g.V3);
                if constexpr (Types<PROF>::M2) zero_acc<P, 4>(g.M2);
                if constexpr (Types<PROF>::M3) zero_acc<P, 9>(g.M3);
                Kahan ks;
                ks.s = kahan[lane];
                ks.c = kahan[32 + lane];
#pragma unroll
                for (int q = 0; q < P; ++q) {
                    const bool ok = (valid >> q) & 1u;
                    const float d = acc.F[0].v[q] - y.v[q];
                    if (ok) ks.add(d * d);
                    g.F[0].v[q] = ok ? 2.0f * d : 0.0f;  // d(diff^2)/d pred, as in evaluator.rs:207
                }
                kahan[lane] = ks.s;
                kahan[32 + lane] = ks.c;
                run_reverse<PROF, P, OMIT>(g, io, rev, n_rev);
            }
            // the warp's sums of this part in f64, then a fresh start for the next
            {
                // sums 0 (squared errors) .. np (gradient), four warp sums
                // at a time, each as warp_sum adds
                double *wred = red + ((size_t)part * nw + warp) * (1 + kAdjParams);
                Kahan ks;
                ks.s = kahan[lane];
                ks.c = kahan[32 + lane];
                for (uint32_t i0 = 0; i0 <= np; i0 += 4) {
                    double v[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint32_t i = i0 + j;
                        v[j] = i == 0 ? (double)ks.value() : i <= np ? (double)io.gacc[(i - 1) * 32] : 0.0;
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                        for (int j = 0; j < 4; ++j) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
                    if (lane == 0)
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if (i0 + j <= np) wred[i0 + j] = v[j];
                }
                for (uint32_t k = 0; k < np; ++k) io.gacc[k * 32] = 0.0f;
                kahan[lane] = 0.0f;
                kahan[32 + lane] = 0.0f;
            }
        }
        // each part's sums across warps in a fixed order (the sums of the
        // parameters past the program's own are 0)
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < n_parts * (1 + kAdjParams); t += blockDim.x) {
            const uint32_t part = t / (1 + kAdjParams), k = t % (1 + kAdjParams);
            double s = 0.0;
            if (k <= np)
                for (int w = 0; w < nw; ++w) s += red[((size_t)part * nw + w) * (1 + kAdjParams) + k];
            a.partials[(size_t)(pd.part_off + it.chunk + part) * (1 + kAdjParams) + k] = s;
        }
        __syncthreads();
    }
    // every thread left the loop together (after the item fetch's barrier)
    tm_fence_before_sync();
    __syncthreads();
    if (warp == 0) tm_dealloc(meta[1], 512u);
}

// ------------------------------------------------------------- launchers
// Shared-memory layout (floats).  Block header: code (+2 pads) | constants |
// meta (4 words) | cross-warp sums (parts x warps x 33 doubles).  Per warp: stacks
// (per type; the reverse sweep's adjoint stacks in the same slots) |
// gradient sums (one row of 32 per parameter, at most 32) | Kahan state (2 x
// 32), each program's own sizes (the kernel lays the region out per item);
// warp_floats is the largest region of the launch.  The tape is in tensor
// memory (a.tmem_cols columns a warp).
uint32_t adj_warp_floats(const uint32_t *stack_depth, int P, uint32_t n_params) {
    uint32_t slots = 0;  // the stacks, whose slots the adjoints reuse
    for (int t = 0; t < N_STACKS; ++t) slots += stack_depth[t] * (uint32_t)kStackWidth[t];
    const uint32_t np = n_params < kAdjParams ? n_params : kAdjParams;
    return (slots * 32u * (uint32_t)P + np * 32u + 2u * 32u + 3u) & ~3u;
}

uint32_t adj_pack_depth(const uint32_t *stack_depth) {
    uint32_t v = 0;
    for (int t = 0; t < N_STACKS; ++t) v |= (stack_depth[t] & 31u) << (5 * t);
    return v;
}

void adj_layout(uint32_t code_words, uint32_t const_floats, uint32_t warp_floats, int nw, uint32_t parts,
                LaunchArgs *a) {
    a->block_hdr_floats = ((code_words + 2u + 3u) & ~3u) + ((const_floats + 3u) & ~3u) + 4u +
                          2u * parts * (uint32_t)nw * (1u + kAdjParams);
    a->region_floats = warp_floats;
    a->tmem_cols = 512u / ((uint32_t)nw / 4u);
}

size_t adj_smem_bytes(uint32_t code_words, uint32_t const_floats, uint32_t warp_floats, int nw, uint32_t parts) {
    LaunchArgs a{};
    adj_layout(code_words, const_floats, warp_floats, nw, parts, &a);
    return ((size_t)a.block_hdr_floats + (size_t)a.region_floats * (uint32_t)nw) * 4u;
}

template <int PROF, int P, int OMIT>
static cudaError_t launch_adj_pp(const LaunchArgs &a, uint32_t grid, size_t smem, cudaStream_t st) {
    auto k = adj_eval_kernel<PROF, P, OMIT>;
    static std::atomic<uint64_t> limit_raised{0};
    cudaError_t e = raise_smem_limit(k, limit_raised);
    if (e != cudaSuccess) return e;
    k<<<grid, adj_warps<PROF, P>() * 32, smem, st>>>(a);
    return cudaGetLastError();
}

// Loads one instance ahead of its first real launch (an empty launch: run_if
// points at a zero word, every thread returns at its first check).
template <int PROF, int P, int OMIT>
static cudaError_t adj_preload_pp(const uint32_t *zero, cudaStream_t st) {
    LaunchArgs none{};
    none.run_if = zero;
    return launch_adj_pp<PROF, P, OMIT>(none, 1, 0, st);
}

bool adj_supported(int profile) { return profile >= P_F && profile <= P_FV3M3; }

// P = 8 exists for the F and F+V3 profiles only (the others would spill).
int adj_max_p(int profile) { return profile == P_F || profile == P_FV3 ? 8 : 4; }

// The instances that exist: (profile, P) as above; OMIT 0..3 for F+V3,
// 0..1 for F and F+V2+M2, 0 for F+V3+M3.  `what` picks the launcher, the
// block size or the preload of instance (PROF, P, omit).
enum AdjWhat { ADJ_LAUNCH, ADJ_WARPS, ADJ_PRELOAD };
struct AdjCall {
    AdjWhat what;
    const LaunchArgs *a;
    uint32_t grid;
    size_t smem;
    cudaStream_t st;
    const uint32_t *zero;
    int occ = 0;  // ADJ_WARPS: the instance's warps per block
};

template <int PROF, int P, int OMIT>
static cudaError_t adj_do(AdjCall &c) {
    if (c.what == ADJ_LAUNCH) return launch_adj_pp<PROF, P, OMIT>(*c.a, c.grid, c.smem, c.st);
    if (c.what == ADJ_WARPS) {
        c.occ = adj_warps<PROF, P>();
        return cudaSuccess;
    }
    return adj_preload_pp<PROF, P, OMIT>(c.zero, c.st);
}

template <int PROF, int P>
static cudaError_t adj_do_omit(AdjCall &c, unsigned omit) {
    if constexpr (PROF == P_FV3) {
        switch (omit & 3u) {
            case 3: return adj_do<PROF, P, 3>(c);
            case 2: return adj_do<PROF, P, 2>(c);
            case 1: return adj_do<PROF, P, 1>(c);
            default: return adj_do<PROF, P, 0>(c);
        }
    } else if constexpr (PROF == P_F || PROF == P_FV2M2) {
        return omit & 1u ? adj_do<PROF, P, 1>(c) : adj_do<PROF, P, 0>(c);
    } else {
        return adj_do<PROF, P, 0>(c);
    }
}

static cudaError_t adj_dispatch(AdjCall &c, int profile, int P, unsigned omit) {
    if (P >= 8) {
        if (profile == P_F) return adj_do_omit<P_F, 8>(c, omit);
        if (profile == P_FV3) return adj_do_omit<P_FV3, 8>(c, omit);
        return cudaErrorInvalidValue;
    }
    switch (profile * 2 + (P >= 4 ? 1 : 0)) {
        case 0: return adj_do_omit<P_F, 2>(c, omit);
        case 1: return adj_do_omit<P_F, 4>(c, omit);
        case 2: return adj_do_omit<P_FV3, 2>(c, omit);
        case 3: return adj_do_omit<P_FV3, 4>(c, omit);
        case 4: return adj_do_omit<P_FV2M2, 2>(c, omit);
        case 5: return adj_do_omit<P_FV2M2, 4>(c, omit);
        case 6: return adj_do_omit<P_FV3M3, 2>(c, omit);
        case 7: return adj_do_omit<P_FV3M3, 4>(c, omit);
        default: return cudaErrorInvalidValue;
    }
}

unsigned adj_omittable(int profile) {
    return profile == P_FV3 ? 3u : profile == P_F || profile == P_FV2M2 ? 1u : 0u;
}

cudaError_t launch_adj(const LaunchArgs &a, int profile, int P, unsigned omit, uint32_t grid, size_t smem,
                       cudaStream_t st) {
    AdjCall c{ADJ_LAUNCH, &a, grid, smem, st, nullptr};
    return adj_dispatch(c, profile, P, omit);
}

int adj_block_warps(int profile, int P) {
    AdjCall c{ADJ_WARPS, nullptr, 0, 0, nullptr, nullptr};
    return adj_dispatch(c, profile, P, 0u) == cudaSuccess ? c.occ : 0;
}

cudaError_t preload_adj(const uint32_t *zero, cudaStream_t st) {
    AdjCall c{ADJ_PRELOAD, nullptr, 0, 0, st, zero};
    for (int profile = P_F; profile <= P_FV3M3; ++profile)
        for (int P = 2; P <= adj_max_p(profile); P *= 2)
            for (unsigned omit = 0; omit <= adj_omittable(profile); ++omit) {
                const cudaError_t e = adj_dispatch(c, profile, P, omit);
                if (e != cudaSuccess) return e;
            }
    return cudaSuccess;
}

}  // namespace rsr
