// acc_ops.cuh -- the accumulator machine of the register kernels: value
// registers of each type, operand fetches and one handler per micro-op kind
// (uops.h, accumulator form).  Shared by the evaluation kernel
// (kernels_reg.cu) and the forward sweep of the register adjoint
// (kernels_adj.cu).
//
// Each value type of the reference VM (state.rs:12-37) has one accumulator
// register set holding P data points per lane: A_F, A_V2[2], A_V3[3],
// A_M2[4], A_M3[9].  A micro-op combines an accumulator with a feature, a
// constant, a value spilled to a per-type stack in shared memory (slot fixed
// by the encoder), or another type's accumulator.
#pragma once
#include "kernels_common.cuh"
#include "tmem.cuh"

namespace rsr {

template <int PROF>
struct Types {
    static constexpr uint32_t T = kProfileTypes[PROF];
    static constexpr bool V2 = (T >> SV2) & 1u, V3 = (T >> SV3) & 1u, M2 = (T >> SM2) & 1u, M3 = (T >> SM3) & 1u;
};

template <int PROF, int P>
struct Acc {
    Vf<P> F[1];
    Vf<P> V2[Types<PROF>::V2 ? 2 : 1];
    Vf<P> V3[Types<PROF>::V3 ? 3 : 1];
    Vf<P> M2[Types<PROF>::M2 ? 4 : 1];
    Vf<P> M3[Types<PROF>::M3 ? 9 : 1];
};

// Operand sources of one lane.  Per-lane values (features, stack slots) use
// the interleaved lane layout (kernels_common.cuh): a feature's tile and a
// stack slot component are each one block of 32*P floats.
template <int P>
struct AccIO {
    const float *xl;        // feature 0 of the current tile, at this lane's first point
    uint32_t stride;        // floats between features
    const float *consts;
    float *stk[N_STACKS];   // per-type stacks, block (slot*W + c), at this lane's first value
    __device__ __forceinline__ Vf<P> X(uint32_t f) const { return load_lane<P>(xl + (size_t)f * stride); }
    __device__ __forceinline__ Vf<P> C(uint32_t i) const { return splat<P>(consts[i]); }
    template <int W>
    __device__ __forceinline__ Vf<P> S(int t, uint32_t slot, int c) const {
        return lds_lane<P>(stk[t] + (slot * W + c) * 32u * P);
    }
    template <int W>
    __device__ __forceinline__ void put(int t, uint32_t slot, int c, const Vf<P> &v) const {
        sts_lane<P>(stk[t] + (slot * W + c) * 32u * P, v);
    }
};

template <int PROF, int P, int t>
__device__ __forceinline__ Vf<P> *acc_of(Acc<PROF, P> &a) {
    if constexpr (t == SF) return a.F;
    else if constexpr (t == SV2) return a.V2;
    else if constexpr (t == SV3) return a.V3;
    else if constexpr (t == SM2) return a.M2;
    else return a.M3;
}

// Second operand of width W from a feature, a constant or a stack slot of type t.
template <int P, int W, int SRC>
__device__ __forceinline__ void fetch(Vf<P> *b, const AccIO<P> &io, int t, uint32_t arg) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
        if constexpr (SRC == SRC_X) b[c] = io.X(arg + c);
        else if constexpr (SRC == SRC_C) b[c] = io.C(arg + c);
        else b[c] = io.template S<W>(t, arg, c);
    }
}

// a = a op b (or b op a for the R-forms), op an AccBin code.
template <int P, int W, int OP>
__device__ __forceinline__ void apply_bin(Vf<P> *a, const Vf<P> *b) {
    if constexpr (OP == BIN_ADD) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = a[i] + b[i];
    } else if constexpr (OP == BIN_SUB) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = a[i] - b[i];
    } else if constexpr (OP == BIN_RSUB) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = b[i] - a[i];
    } else if constexpr (OP == BIN_MUL) {
        a[0] = a[0] * b[0];
    } else if constexpr (OP == BIN_DIV) {
        a[0] = a[0] / b[0];
    } else if constexpr (OP == BIN_RDIV) {
        a[0] = b[0] / a[0];
    } else if constexpr (OP == BIN_CROSS) {
        cross3(a, b, a);
    } else if constexpr (OP == BIN_RCROSS) {
        cross3(b, a, a);
    } else if constexpr (OP == BIN_MMUL) {
        if constexpr (W == 4) mul_m2(a, b, a); else mul_m3(a, b, a);
    } else {
        if constexpr (W == 4) mul_m2(b, a, a); else mul_m3(b, a, a);
    }
}

template <int t, int j>
__host__ __device__ constexpr int bin_code() {
    if constexpr (t == SF) {
        return j == 0 ? BIN_ADD : j == 1 ? BIN_SUB : j == 2 ? BIN_RSUB : j == 3 ? BIN_MUL : j == 4 ? BIN_DIV : BIN_RDIV;
    } else if constexpr (t == SV2) {
        return j == 0 ? BIN_ADD : j == 1 ? BIN_SUB : BIN_RSUB;
    } else if constexpr (t == SV3) {
        return j == 0 ? BIN_ADD : j == 1 ? BIN_SUB : j == 2 ? BIN_RSUB : j == 3 ? BIN_CROSS : BIN_RCROSS;
    } else {
        return j == 0 ? BIN_ADD : j == 1 ? BIN_SUB : j == 2 ? BIN_RSUB : j == 3 ? BIN_MMUL : BIN_RMMUL;
    }
}

// Load a feature (or a constant) into the accumulator of runtime type t
// (one of the profile's): the load fused after a PUSH.
template <int PROF, int P, int t>
__device__ __forceinline__ void load_t(Acc<PROF, P> &a, const AccIO<P> &io, uint32_t is_const, uint32_t off) {
    if constexpr (((kProfileTypes[PROF] >> t) & 1u) != 0u) {
        constexpr int W = kStackWidth[t];
        Vf<P> *A = acc_of<PROF, P, t>(a);
        if (is_const) fetch<P, W, SRC_C>(A, io, t, off);
        else fetch<P, W, SRC_X>(A, io, t, off);
    }
}
template <int PROF, int P>
__device__ __forceinline__ void load_any(Acc<PROF, P> &a, const AccIO<P> &io, uint32_t t, uint32_t is_const,
                                         uint32_t off) {
    switch (t) {
        case SF: load_t<PROF, P, SF>(a, io, is_const, off); break;
        case SV2: load_t<PROF, P, SV2>(a, io, is_const, off); break;
        case SV3: load_t<PROF, P, SV3>(a, io, is_const, off); break;
        case SM2: load_t<PROF, P, SM2>(a, io, is_const, off); break;
        default: load_t<PROF, P, SM3>(a, io, is_const, off); break;
    }
}

// Optional operand load in front of a unary op (uops.h, unary_load_arg).
template <int P, int W>
__device__ __forceinline__ void unary_prefix(Vf<P> *A, const AccIO<P> &io, int t, uint32_t arg) {
    const uint32_t src1 = (arg >> 12) & 3u;
    if (src1 == 1u) fetch<P, W, SRC_X>(A, io, t, arg & 0xFFFu);
    else if (src1 == 2u) fetch<P, W, SRC_C>(A, io, t, arg & 0xFFFu);
}

// One accumulator micro-op of kind K.
template <int PROF, int P, int K>
__device__ __forceinline__ void acc_op(Acc<PROF, P> &a, const AccIO<P> &io, uint32_t arg) {
    constexpr int t = K >= K_M3 ? SM3 : K >= K_M2 ? SM2 : K >= K_V3 ? SV3 : K >= K_V2 ? SV2 : SF;
    if constexpr (((kProfileTypes[PROF] >> t) & 1u) != 0u) {
        constexpr int W = kStackWidth[t];
        constexpr int k = K - kBlockBase[t];
        constexpr int nb = kBinOps[t];
        Vf<P> *A = acc_of<PROF, P, t>(a);
        if constexpr (k == KV_LDX) {
            fetch<P, W, SRC_X>(A, io, t, arg);
        } else if constexpr (k == KV_LDC) {
            fetch<P, W, SRC_C>(A, io, t, arg);
        } else if constexpr (k == KV_PUSH) {
            const uint32_t slot = arg & 15u, lt = (arg >> 4) & 7u;
#pragma unroll
            for (int c = 0; c < W; ++c) io.template put<W>(t, slot, c, A[c]);
            if (lt) load_any<PROF, P>(a, io, lt - 1u, (arg >> 7) & 1u, (arg >> 8) & ((1u << kLdOffsetBits) - 1u));
        } else if constexpr (k >= KV_BIN && k < KV_BIN + 3 * nb) {
            constexpr int j = (k - KV_BIN) / 3, src = (k - KV_BIN) % 3;
            Vf<P> b[W];
            fetch<P, W, src>(b, io, t, arg);
            apply_bin<P, W, bin_code<t, j>()>(A, b);
        } else if constexpr (t == SF) {
            constexpr int u = k - (K_F_UN - K_F);
            unary_prefix<P, 1>(A, io, t, arg);
            if constexpr (u == 0) A[0] = vsin(A[0]);
            else if constexpr (u == 1) A[0] = vcos(A[0]);
            else if constexpr (u == 2) A[0] = vexp(A[0]);
            else if constexpr (u == 3) A[0] = A[0] * A[0];
            else if constexpr (u == 4) A[0] = vsqrt(A[0]);
            else if constexpr (u == 5) A[0] = vlog(A[0]);
        } else if constexpr (t == SV2 || t == SV3) {
            constexpr int ks = kv_scale(nb), kd = kv_dot(nb), kn = kv_norm(nb), km = kv_mulm(nb, W),
                          kk = kv_make(nb, W);
            if constexpr (k >= ks && k < ks + 4) {                // SCALE {A X C S}
                Vf<P> s;
                if constexpr (k == ks) s = a.F[0];
                else if constexpr (k == ks + 1) s = io.X(arg);
                else if constexpr (k == ks + 2) s = io.C(arg);
                else s = io.template S<1>(SF, arg, 0);
#pragma unroll
                for (int c = 0; c < W; ++c) A[c] = A[c] * s;
            } else if constexpr (k >= kd && k < kd + 3) {         // DOT {X C S} -> A_F
                Vf<P> b[W];
                fetch<P, W, k - kd>(b, io, t, arg);
                if constexpr (W == 2) a.F[0] = dot2(A, b); else a.F[0] = dot3(A, b);
            } else if constexpr (k == kn) {                       // NORM -> A_F
                unary_prefix<P, W>(A, io, t, arg);
                if constexpr (W == 2) a.F[0] = norm2(A); else a.F[0] = norm3(A);
            } else if constexpr (k > kn && k <= kn + W) {         // GET x/y/z -> A_F
                unary_prefix<P, W>(A, io, t, arg);
                a.F[0] = A[k - kn - 1];
            } else if constexpr (k >= km && k < km + 4) {         // MULM {A X C S}: A = M * A
                constexpr int tm = W == 2 ? SM2 : SM3;
                constexpr int MW = W * W;
                if constexpr (((kProfileTypes[PROF] >> tm) & 1u) != 0u || k != km) {
                    Vf<P> m[MW];
                    if constexpr (k == km) {
                        if constexpr (((kProfileTypes[PROF] >> tm) & 1u) != 0u) {
                            Vf<P> *M = acc_of<PROF, P, tm>(a);
#pragma unroll
                            for (int c = 0; c < MW; ++c) m[c] = M[c];
                        }
                    } else if constexpr (k == km + 1) {
                        fetch<P, MW, SRC_X>(m, io, tm, arg);
                    } else if constexpr (k == km + 2) {
                        fetch<P, MW, SRC_C>(m, io, tm, arg);
                    } else {
                        fetch<P, MW, SRC_S>(m, io, tm, arg);
                    }
                    if constexpr (W == 2) mul_m2v2(m, A, A); else mul_m3v3(m, A, A);
                }
            } else if constexpr (k == kk) {                       // MAKE from F stack + A_F
#pragma unroll
                for (int c = 0; c + 1 < W; ++c) A[c] = io.template S<1>(SF, arg + c, 0);
                A[W - 1] = a.F[0];
            }
        } else {  // M2 / M3
            constexpr int N = W == 4 ? 2 : 3;
            constexpr int tv = W == 4 ? SV2 : SV3;
            if constexpr (k >= KM_SCALE && k < KM_SCALE + 4) {
                Vf<P> s;
                if constexpr (k == KM_SCALE) s = a.F[0];
                else if constexpr (k == KM_SCALE + 1) s = io.X(arg);
                else if constexpr (k == KM_SCALE + 2) s = io.C(arg);
                else s = io.template S<1>(SF, arg, 0);
#pragma unroll
                for (int c = 0; c < W; ++c) A[c] = A[c] * s;
            } else if constexpr (k == KM_DET) {
                unary_prefix<P, W>(A, io, t, arg);
                if constexpr (N == 2) a.F[0] = det_m2(A); else a.F[0] = det_m3(A);
            } else if constexpr (k == KM_TRACE) {
                unary_prefix<P, W>(A, io, t, arg);
                if constexpr (N == 2) a.F[0] = trace_m2(A); else a.F[0] = trace_m3(A);
            } else if constexpr (k == KM_TRANSPOSE) {
                unary_prefix<P, W>(A, io, t, arg);
                if constexpr (N == 2) transpose_m2(A, A); else transpose_m3(A, A);
            } else if constexpr (k == KM_INVERSE) {
                unary_prefix<P, W>(A, io, t, arg);
                if constexpr (N == 2) inverse_m2(A, A); else inverse_m3(A, A);
            } else if constexpr (k == KM_MAKE) {                  // columns: stack slots + A_V
                if constexpr (((kProfileTypes[PROF] >> tv) & 1u) != 0u) {
                    Vf<P> *V = acc_of<PROF, P, tv>(a);
#pragma unroll
                    for (int col = 0; col + 1 < N; ++col)
#pragma unroll
                        for (int r = 0; r < N; ++r) A[N * col + r] = io.template S<N>(tv, arg + col, r);
#pragma unroll
                    for (int r = 0; r < N; ++r) A[N * (N - 1) + r] = V[r];
                }
            }
        }
    }
}

}  // namespace rsr
