// kernels_grad.cu -- reverse-mode adjoint kernel: MSE and d(MSE)/d(constants)
// of a program in one forward and one reverse sweep per tile of points.
//
// Replaces compute_mse_with_gradient (src/engine/eval/evaluator.rs:177-224),
// which runs one dual-number forward pass per flat parameter
// (eval_simd_dual, evaluator.rs:228-388).  The tape is the program's SSA slot
// file (every live value has its own slots) in shared memory, recorded for
// one tile of 32*P points and consumed by the reverse sweep right away: the
// whole population x points x length tape is never stored, it is recomputed
// tile by tile.
//
// Reverse rules follow the forward rules of src/engine/eval/autodiff.rs; for
// InverseM2/M3, whose dual dispatch is a no-op in the reference
// (src/domains/linalg/mod.rs:643,687), the adjoint is the exact one,
// dA = -A^-T G A^-T, and zero on the singular branch (|det| < 1e-9), whose
// value is a constant identity.
#include <cuda_runtime.h>
#include <float.h>

#include "kernels.h"
#include "kernels_common.cuh"

namespace rsr {

__host__ __device__ __forceinline__ uint32_t align4g(uint32_t v) { return (v + 3u) & ~3u; }
constexpr uint32_t kGradParams = 32;

// Per-profile kernels: an opcode whose value type the profile lacks gets a
// case label outside the opcode range, so its handler is dropped and the
// kernel's code (and its instruction-cache footprint) shrinks.
#define RSR_PROFILE_TYPES(PROF)                                                    \
    constexpr uint32_t kTypes = kProfileTypes[PROF];                               \
    constexpr bool HV2 = (kTypes >> SV2) & 1u, HV3 = (kTypes >> SV3) & 1u;         \
    constexpr bool HM2 = (kTypes >> SM2) & 1u, HM3 = (kTypes >> SM3) & 1u;         \
    (void)HV2; (void)HV3; (void)HM2; (void)HM3;
#define RSR_GATE(OP, HAS) ((HAS) ? (int)(OP) : 0x1000 + (int)(OP))

template <int P>
struct TapeCtx {
    Vf<P> *val;   // [slot][lane]
    Vf<P> *adj;   // [slot][lane]
    const float *consts;
    const float *x;
    uint64_t stride, p0;
    uint64_t n_eval;   // points counted (num_batches * 8)
    int lane;
    // a value slot with kTapeFeature set is a feature column, read in place
    __device__ __forceinline__ Vf<P> V(uint32_t s) const {
        return (s & kTapeFeature) ? X(s & (kTapeFeature - 1u)) : val[s * 32 + lane];
    }
    __device__ __forceinline__ void SV(uint32_t s, const Vf<P> &v) const { val[s * 32 + lane] = v; }
    __device__ __forceinline__ Vf<P> A(uint32_t s) const { return adj[s * 32 + lane]; }
    // adds a contribution to adjoint slot s (a feature's goes to the sink)
    __device__ __forceinline__ void AddA(uint32_t s, const Vf<P> &v) const {
        Vf<P> &r = adj[s * 32 + lane];
        r = r + v;
    }
    __device__ __forceinline__ void ClearA(uint32_t s, uint32_t width) const {
        for (uint32_t i = 0; i < width; ++i) adj[(s + i) * 32 + lane] = splat<P>(0.0f);
    }
    __device__ __forceinline__ Vf<P> X(uint32_t f) const { return load_pts<P>(x + f * stride + p0); }
};

// Element-wise vector/matrix ops with the width known at compile time, so
// that their operands stay in registers.
template <int P, int W, bool SUB>
__device__ __forceinline__ void fwd_addsub(const TapeCtx<P> &t, uint32_t o, uint32_t i0, uint32_t i1) {
#pragma unroll
    for (int i = 0; i < W; ++i) t.SV(o + i, SUB ? t.V(i0 + i) - t.V(i1 + i) : t.V(i0 + i) + t.V(i1 + i));
}
template <int P, int W>
__device__ __forceinline__ void fwd_scale(const TapeCtx<P> &t, uint32_t o, uint32_t i0, uint32_t i1) {
    const Vf<P> s = t.V(i0);
#pragma unroll
    for (int i = 0; i < W; ++i) t.SV(o + i, t.V(i1 + i) * s);
}

// Forward value of one tape instruction (same semantics as the slot kernel).
template <int PROF, int P, bool NU>
__device__ __forceinline__ void tape_forward(const TapeCtx<P> &t, const uint32_t *w) {
    RSR_PROFILE_TYPES(PROF)
    constexpr bool HU = !NU;  // the launch has unary Float ops
    const uint32_t op = w[0] & 0xFFu, aux = (w[0] >> 8) & 0xFFFFFu;
    const uint32_t o = w[1] & 0xFFFFu, i0 = w[2] & 0xFFFFu, i1 = w[3] & 0xFFFFu, i2 = w[4] & 0xFFFFu;
    Vf<P> A[9], B[9], R[9];
    auto Ln = [&](Vf<P> *d, uint32_t s, int n) { for (int i = 0; i < n; ++i) d[i] = t.V(s + i); };
    auto Sn = [&](uint32_t s, const Vf<P> *v, int n) { for (int i = 0; i < n; ++i) t.SV(s + i, v[i]); };
    switch (op) {
        case SLOT_NOP: {  // stale constant slot: copy of the aliased value, or zero
            const uint32_t w = aux >> 1;
            for (uint32_t i = 0; i < w; ++i) t.SV(o + i, (aux & 1u) ? t.V(i0 + i) : splat<P>(0.0f));
            break;
        }
        case LOAD_VAR_F: t.SV(o, t.X(aux)); break;
        case RSR_GATE(LOAD_VAR_V2, HV2): for (int i = 0; i < 2; ++i) t.SV(o + i, t.X(aux + i)); break;
        case RSR_GATE(LOAD_VAR_V3, HV3): for (int i = 0; i < 3; ++i) t.SV(o + i, t.X(aux + i)); break;
        case RSR_GATE(LOAD_VAR_M2, HM2): for (int i = 0; i < 4; ++i) t.SV(o + i, t.X(aux + i)); break;
        case RSR_GATE(LOAD_VAR_M3, HM3): for (int i = 0; i < 9; ++i) t.SV(o + i, t.X(aux + i)); break;
        case LOAD_CONST_F: t.SV(o, splat<P>(t.consts[aux])); break;
        case RSR_GATE(LOAD_CONST_V2, HV2): for (int i = 0; i < 2; ++i) t.SV(o + i, splat<P>(t.consts[aux + i])); break;
        case RSR_GATE(LOAD_CONST_V3, HV3): for (int i = 0; i < 3; ++i) t.SV(o + i, splat<P>(t.consts[aux + i])); break;
        case RSR_GATE(LOAD_CONST_M2, HM2): for (int i = 0; i < 4; ++i) t.SV(o + i, splat<P>(t.consts[aux + i])); break;
        case RSR_GATE(LOAD_CONST_M3, HM3): for (int i = 0; i < 9; ++i) t.SV(o + i, splat<P>(t.consts[aux + i])); break;
        case ADD_F: t.SV(o, t.V(i0) + t.V(i1)); break;
        case SUB_F: t.SV(o, t.V(i0) - t.V(i1)); break;
        case MUL_F: t.SV(o, t.V(i0) * t.V(i1)); break;
        case DIV_F: t.SV(o, t.V(i0) / t.V(i1)); break;
        case RSR_GATE(SIN_F, HU): t.SV(o, vsin(t.V(i0))); break;
        case RSR_GATE(COS_F, HU): t.SV(o, vcos(t.V(i0))); break;
        case RSR_GATE(EXP_F, HU): t.SV(o, vexp(t.V(i0))); break;
        case RSR_GATE(SQR_F, HU): { Vf<P> a = t.V(i0); t.SV(o, a * a); break; }
        case RSR_GATE(SQRT_F, HU): t.SV(o, vsqrt(t.V(i0))); break;
        case RSR_GATE(LN_F, HU): t.SV(o, vlog(t.V(i0))); break;
        case MAKE_VEC2: A[0] = t.V(i0); A[1] = t.V(i1); Sn(o, A, 2); break;
        case MAKE_VEC3: A[0] = t.V(i0); A[1] = t.V(i1); A[2] = t.V(i2); Sn(o, A, 3); break;
        case RSR_GATE(GET_X_V2, HV2): case RSR_GATE(GET_X_V3, HV3): t.SV(o, t.V(i0)); break;
        case RSR_GATE(GET_Y_V2, HV2): case RSR_GATE(GET_Y_V3, HV3): t.SV(o, t.V(i0 + 1)); break;
        case RSR_GATE(GET_Z_V3, HV3): t.SV(o, t.V(i0 + 2)); break;
        case RSR_GATE(ADD_V2, HV2): fwd_addsub<P, 2, false>(t, o, i0, i1); break;
        case RSR_GATE(ADD_V3, HV3): fwd_addsub<P, 3, false>(t, o, i0, i1); break;
        case RSR_GATE(ADD_M2, HM2): fwd_addsub<P, 4, false>(t, o, i0, i1); break;
        case RSR_GATE(ADD_M3, HM3): fwd_addsub<P, 9, false>(t, o, i0, i1); break;
        case RSR_GATE(SUB_V2, HV2): fwd_addsub<P, 2, true>(t, o, i0, i1); break;
        case RSR_GATE(SUB_V3, HV3): fwd_addsub<P, 3, true>(t, o, i0, i1); break;
        case RSR_GATE(SUB_M2, HM2): fwd_addsub<P, 4, true>(t, o, i0, i1); break;
        case RSR_GATE(SUB_M3, HM3): fwd_addsub<P, 9, true>(t, o, i0, i1); break;
        case RSR_GATE(SCALE_V2, HV2): fwd_scale<P, 2>(t, o, i0, i1); break;
        case RSR_GATE(SCALE_V3, HV3): fwd_scale<P, 3>(t, o, i0, i1); break;
        case RSR_GATE(SCALE_M2, HM2): fwd_scale<P, 4>(t, o, i0, i1); break;
        case RSR_GATE(SCALE_M3, HM3): fwd_scale<P, 9>(t, o, i0, i1); break;
        case RSR_GATE(DOT_V2, HV2): Ln(A, i0, 2); Ln(B, i1, 2); t.SV(o, dot2(A, B)); break;
        case RSR_GATE(DOT_V3, HV3): Ln(A, i0, 3); Ln(B, i1, 3); t.SV(o, dot3(A, B)); break;
        case RSR_GATE(NORM_V2, HV2): Ln(A, i0, 2); t.SV(o, norm2(A)); break;
        case RSR_GATE(NORM_V3, HV3): Ln(A, i0, 3); t.SV(o, norm3(A)); break;
        case RSR_GATE(CROSS_V3, HV3): Ln(A, i0, 3); Ln(B, i1, 3); cross3(A, B, R); Sn(o, R, 3); break;
        case RSR_GATE(MAKE_MAT2, HM2): Ln(A, i0, 2); Ln(A + 2, i1, 2); Sn(o, A, 4); break;
        case RSR_GATE(MUL_M2, HM2): Ln(A, i0, 4); Ln(B, i1, 4); mul_m2(A, B, R); Sn(o, R, 4); break;
        case RSR_GATE(MUL_M2V2, HM2): Ln(A, i0, 4); Ln(B, i1, 2); mul_m2v2(A, B, R); Sn(o, R, 2); break;
        case RSR_GATE(DET_M2, HM2): Ln(A, i0, 4); t.SV(o, det_m2(A)); break;
        case RSR_GATE(TRACE_M2, HM2): Ln(A, i0, 4); t.SV(o, trace_m2(A)); break;
        case RSR_GATE(TRANSPOSE_M2, HM2): Ln(A, i0, 4); transpose_m2(A, R); Sn(o, R, 4); break;
        case RSR_GATE(INVERSE_M2, HM2): Ln(A, i0, 4); inverse_m2(A, R); Sn(o, R, 4); break;
        case RSR_GATE(MAKE_MAT3, HM3): Ln(A, i0, 3); Ln(A + 3, i1, 3); Ln(A + 6, i2, 3); Sn(o, A, 9); break;
        case RSR_GATE(MUL_M3, HM3): Ln(A, i0, 9); Ln(B, i1, 9); mul_m3(A, B, R); Sn(o, R, 9); break;
        case RSR_GATE(MUL_M3V3, HM3): Ln(A, i0, 9); Ln(B, i1, 3); mul_m3v3(A, B, R); Sn(o, R, 3); break;
        case RSR_GATE(DET_M3, HM3): Ln(A, i0, 9); t.SV(o, det_m3(A)); break;
        case RSR_GATE(TRACE_M3, HM3): Ln(A, i0, 9); t.SV(o, trace_m3(A)); break;
        case RSR_GATE(TRANSPOSE_M3, HM3): Ln(A, i0, 9); transpose_m3(A, R); Sn(o, R, 9); break;
        case RSR_GATE(INVERSE_M3, HM3): Ln(A, i0, 9); inverse_m3(A, R); Sn(o, R, 9); break;
        default: break;
    }
}

// dA = -O^T G O^T for O = A^-1 (N x N, column-major), zero where singular.
template <int P, int N>
__device__ __forceinline__ void inverse_adjoint(const TapeCtx<P> &t, uint32_t vo, uint32_t ao, uint32_t v0, uint32_t a0) {
    if (v0 & kTapeFeature) return;  // a feature matrix keeps no adjoint
    Vf<P> O[N * N], G[N * N], H[N * N], M[N * N];
    for (int i = 0; i < N * N; ++i) { O[i] = t.V(vo + i); G[i] = t.A(ao + i); M[i] = t.V(v0 + i); }
    Vf<P> det;
    if constexpr (N == 2) det = det_m2(M); else det = det_m3(M);
    // H = O^T G : H(i,l) = sum_k O(k,i) G(k,l)
    for (int i = 0; i < N; ++i)
        for (int l = 0; l < N; ++l) {
            Vf<P> s = splat<P>(0.0f);
            for (int k = 0; k < N; ++k) s = s + O[N * i + k] * G[N * l + k];
            H[N * l + i] = s;
        }
    // dA(i,j) = -sum_l H(i,l) O(j,l)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            Vf<P> s = splat<P>(0.0f);
            for (int l = 0; l < N; ++l) s = s + H[N * l + i] * O[N * l + j];
            Vf<P> d;
#pragma unroll
            for (int k = 0; k < P; ++k) d.v[k] = fabsf(det.v[k]) < 1e-9f ? 0.0f : -s.v[k];
            t.AddA(a0 + N * j + i, d);
        }
}

// O = A B (N x N, column-major): dA = G B^T, dB = A^T G.
template <int P, int N>
__device__ __forceinline__ void rev_mulm(const TapeCtx<P> &t, uint32_t vo, uint32_t ao, uint32_t v0, uint32_t a0, uint32_t v1,
                                         uint32_t a1) {
    // a feature matrix keeps no adjoint
    const bool keep_a = !(v0 & kTapeFeature), keep_b = !(v1 & kTapeFeature);
    Vf<P> Am[N * N], Bm[N * N], G[N * N];
#pragma unroll
    for (int i = 0; i < N * N; ++i) { Am[i] = t.V(v0 + i); Bm[i] = t.V(v1 + i); G[i] = t.A(ao + i); }
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
        for (int c = 0; c < N; ++c) {
            Vf<P> da = splat<P>(0.0f), db = splat<P>(0.0f);
#pragma unroll
            for (int j = 0; j < N; ++j) {
                da = da + G[N * j + r] * Bm[N * j + c];   // G(r,j) B(c,j)
                db = db + Am[N * r + j] * G[N * c + j];   // A(j,r) G(j,c)
            }
            if (keep_a) t.AddA(a0 + N * c + r, da);
            if (keep_b) t.AddA(a1 + N * c + r, db);
        }
}
// o = M v: dM(r,c) += g_r v_c, dv_c += sum_r M(r,c) g_r.
template <int P, int N>
__device__ __forceinline__ void rev_mulmv(const TapeCtx<P> &t, uint32_t vo, uint32_t ao, uint32_t v0, uint32_t a0, uint32_t v1,
                                          uint32_t a1) {
    Vf<P> g[N], v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) { g[i] = t.A(ao + i); v[i] = t.V(v1 + i); }
    if (!(v0 & kTapeFeature)) {  // a feature matrix keeps no adjoint
#pragma unroll
        for (int c = 0; c < N; ++c)
#pragma unroll
            for (int r = 0; r < N; ++r) t.AddA(a0 + N * c + r, g[r] * v[c]);
    }
#pragma unroll
    for (int c = 0; c < N; ++c) {
        Vf<P> dv = splat<P>(0.0f);
#pragma unroll
        for (int r = 0; r < N; ++r) dv = dv + t.V(v0 + N * c + r) * g[r];
        t.AddA(a1 + c, dv);
    }
}

// Reverse sweep of one tape instruction.  gacc: this lane's f32 gradient
// contributions of the tile (summed over its P points).
template <int PROF, int P, bool NU>
__device__ __forceinline__ void tape_reverse(const TapeCtx<P> &t, const uint32_t *w, float *gacc_lane) {
    RSR_PROFILE_TYPES(PROF)
    constexpr bool HU = !NU;
    const uint32_t op = w[0] & 0xFFu, aux = (w[0] >> 8) & 0xFFFFFu;
    const uint32_t vo = w[1] & 0xFFFFu, ao = w[1] >> 16;
    const uint32_t v0 = w[2] & 0xFFFFu, v1 = w[3] & 0xFFFFu;
    const uint32_t a0 = (w[2] >> 16) & ~kTapeZeroFirst, a1 = (w[3] >> 16) & ~kTapeZeroFirst,
                   a2 = (w[4] >> 16) & ~kTapeZeroFirst;
    // inputs whose adjoint gets its first contribution here: clear their
    // slots, which may still hold an earlier value (widths: a copy's own
    // width, else one nibble per input)
    if ((w[2] | w[3] | w[4]) & (kTapeZeroFirst << 16)) {
        if (op == SLOT_NOP) {
            if (w[2] & (kTapeZeroFirst << 16)) t.ClearA(a0, aux >> 1);
        } else {
            if (w[2] & (kTapeZeroFirst << 16)) t.ClearA(a0, aux & 0xFu);
            if (w[3] & (kTapeZeroFirst << 16)) t.ClearA(a1, (aux >> 4) & 0xFu);
            if (w[4] & (kTapeZeroFirst << 16)) t.ClearA(a2, (aux >> 8) & 0xFu);
        }
    }
    switch (op) {
        case SLOT_NOP:
            if (aux & 1u) for (uint32_t i = 0; i < (aux >> 1); ++i) t.AddA(a0 + i, t.A(ao + i));
            break;
        case LOAD_VAR_F: case RSR_GATE(LOAD_VAR_V2, HV2): case RSR_GATE(LOAD_VAR_V3, HV3): case RSR_GATE(LOAD_VAR_M2, HM2): case RSR_GATE(LOAD_VAR_M3, HM3): break;
        case LOAD_CONST_F: case RSR_GATE(LOAD_CONST_V2, HV2): case RSR_GATE(LOAD_CONST_V3, HV3): case RSR_GATE(LOAD_CONST_M2, HM2): case RSR_GATE(LOAD_CONST_M3, HM3): {
            const int w = op == LOAD_CONST_F ? 1 : op == LOAD_CONST_V2 ? 2 : op == LOAD_CONST_V3 ? 3
                        : op == LOAD_CONST_M2 ? 4 : 9;
            for (int i = 0; i < w; ++i) {
                if (aux + i >= kGradParams) break;
                const Vf<P> g = t.A(ao + i);
                float s = 0.0f;
#pragma unroll
                for (int k = 0; k < P; ++k)  // points past the dataset's end may carry 0*inf = NaN adjoints
                    if (t.p0 + k < t.n_eval) s = s + g.v[k];
                gacc_lane[(aux + i) * 32] += s;
            }
            break;
        }
        case ADD_F: { const Vf<P> g = t.A(ao); t.AddA(a0, g); t.AddA(a1, g); break; }
        case SUB_F: { const Vf<P> g = t.A(ao); t.AddA(a0, g); t.AddA(a1, -g); break; }
        case MUL_F: { const Vf<P> g = t.A(ao); t.AddA(a0, g * t.V(v1)); t.AddA(a1, g * t.V(v0)); break; }
        case DIV_F: {
            const Vf<P> q = t.A(ao) / t.V(v1);
            t.AddA(a0, q);
            t.AddA(a1, -(q * t.V(vo)));
            break;
        }
        case RSR_GATE(SIN_F, HU): t.AddA(a0, t.A(ao) * vcos(t.V(v0))); break;
        case RSR_GATE(COS_F, HU): t.AddA(a0, t.A(ao) * (-vsin(t.V(v0)))); break;
        case RSR_GATE(EXP_F, HU): t.AddA(a0, t.A(ao) * t.V(vo)); break;
        case RSR_GATE(SQR_F, HU): t.AddA(a0, t.A(ao) * (splat<P>(2.0f) * t.V(v0))); break;
        case RSR_GATE(SQRT_F, HU): t.AddA(a0, t.A(ao) / (splat<P>(2.0f) * t.V(vo))); break;
        case RSR_GATE(LN_F, HU): t.AddA(a0, t.A(ao) / t.V(v0)); break;
        case MAKE_VEC2: t.AddA(a0, t.A(ao)); t.AddA(a1, t.A(ao + 1)); break;
        case MAKE_VEC3: t.AddA(a0, t.A(ao)); t.AddA(a1, t.A(ao + 1)); t.AddA(a2, t.A(ao + 2)); break;
        case RSR_GATE(GET_X_V2, HV2): case RSR_GATE(GET_X_V3, HV3): t.AddA(a0, t.A(ao)); break;
        case RSR_GATE(GET_Y_V2, HV2): case RSR_GATE(GET_Y_V3, HV3): t.AddA(a0 + 1, t.A(ao)); break;
        case RSR_GATE(GET_Z_V3, HV3): t.AddA(a0 + 2, t.A(ao)); break;
        case RSR_GATE(ADD_V2, HV2): case RSR_GATE(ADD_V3, HV3): case RSR_GATE(ADD_M2, HM2): case RSR_GATE(ADD_M3, HM3): case RSR_GATE(SUB_V2, HV2): case RSR_GATE(SUB_V3, HV3): case RSR_GATE(SUB_M2, HM2): case RSR_GATE(SUB_M3, HM3): {
            const bool sub = op == SUB_V2 || op == SUB_V3 || op == SUB_M2 || op == SUB_M3;
            const int w = (op == ADD_V2 || op == SUB_V2) ? 2 : (op == ADD_V3 || op == SUB_V3) ? 3
                        : (op == ADD_M2 || op == SUB_M2) ? 4 : 9;
            for (int i = 0; i < w; ++i) {
                const Vf<P> g = t.A(ao + i);
                t.AddA(a0 + i, g);
                t.AddA(a1 + i, sub ? -g : g);
            }
            break;
        }
        case RSR_GATE(SCALE_V2, HV2): case RSR_GATE(SCALE_V3, HV3): case RSR_GATE(SCALE_M2, HM2): case RSR_GATE(SCALE_M3, HM3): {
            const int w = op == SCALE_V2 ? 2 : op == SCALE_V3 ? 3 : op == SCALE_M2 ? 4 : 9;
            const Vf<P> s = t.V(v0);
            Vf<P> ds = splat<P>(0.0f);
            for (int i = 0; i < w; ++i) {
                const Vf<P> g = t.A(ao + i);
                ds = ds + g * t.V(v1 + i);
                t.AddA(a1 + i, g * s);
            }
            t.AddA(a0, ds);
            break;
        }
        case RSR_GATE(DOT_V2, HV2): case RSR_GATE(DOT_V3, HV3): {
            const int w = op == DOT_V2 ? 2 : 3;
            const Vf<P> g = t.A(ao);
            for (int i = 0; i < w; ++i) {
                const Vf<P> a = t.V(v0 + i), b = t.V(v1 + i);
                t.AddA(a0 + i, g * b);
                t.AddA(a1 + i, g * a);
            }
            break;
        }
        case RSR_GATE(NORM_V2, HV2): case RSR_GATE(NORM_V3, HV3): {
            const int w = op == NORM_V2 ? 2 : 3;
            const Vf<P> q = t.A(ao) / t.V(vo);
            for (int i = 0; i < w; ++i) t.AddA(a0 + i, q * t.V(v0 + i));
            break;
        }
        case RSR_GATE(CROSS_V3, HV3): {  // o = a x b: da += b x g, db += g x a
            Vf<P> a[3], b[3], g[3], da[3], db[3];
            for (int i = 0; i < 3; ++i) { a[i] = t.V(v0 + i); b[i] = t.V(v1 + i); g[i] = t.A(ao + i); }
            cross3(b, g, da);
            cross3(g, a, db);
            for (int i = 0; i < 3; ++i) { t.AddA(a0 + i, da[i]); t.AddA(a1 + i, db[i]); }
            break;
        }
        case RSR_GATE(MAKE_MAT2, HM2):
            t.AddA(a0, t.A(ao)); t.AddA(a0 + 1, t.A(ao + 1)); t.AddA(a1, t.A(ao + 2)); t.AddA(a1 + 1, t.A(ao + 3));
            break;
        case RSR_GATE(MAKE_MAT3, HM3):
            for (int i = 0; i < 3; ++i) { t.AddA(a0 + i, t.A(ao + i)); t.AddA(a1 + i, t.A(ao + 3 + i)); t.AddA(a2 + i, t.A(ao + 6 + i)); }
            break;
        case RSR_GATE(MUL_M2, HM2): rev_mulm<P, 2>(t, vo, ao, v0, a0, v1, a1); break;
        case RSR_GATE(MUL_M3, HM3): rev_mulm<P, 3>(t, vo, ao, v0, a0, v1, a1); break;
        case RSR_GATE(MUL_M2V2, HM2): rev_mulmv<P, 2>(t, vo, ao, v0, a0, v1, a1); break;
        case RSR_GATE(MUL_M3V3, HM3): rev_mulmv<P, 3>(t, vo, ao, v0, a0, v1, a1); break;
        case RSR_GATE(DET_M2, HM2): {
            const Vf<P> g = t.A(ao);
            t.AddA(a0, g * t.V(v0 + 3));
            t.AddA(a0 + 3, g * t.V(v0));
            t.AddA(a0 + 1, -(g * t.V(v0 + 2)));
            t.AddA(a0 + 2, -(g * t.V(v0 + 1)));
            break;
        }
        case RSR_GATE(DET_M3, HM3): {  // d det / d m(r,c) = cofactor C(r,c)
            const Vf<P> g = t.A(ao);
            Vf<P> m[9];
            for (int i = 0; i < 9; ++i) m[i] = t.V(v0 + i);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
                    const Vf<P> cof = m[3 * c1 + r1] * m[3 * c2 + r2] - m[3 * c2 + r1] * m[3 * c1 + r2];
                    t.AddA(a0 + 3 * c + r, g * cof);
                }
            break;
        }
        case RSR_GATE(TRACE_M2, HM2): { const Vf<P> g = t.A(ao); t.AddA(a0, g); t.AddA(a0 + 3, g); break; }
        case RSR_GATE(TRACE_M3, HM3): { const Vf<P> g = t.A(ao); t.AddA(a0, g); t.AddA(a0 + 4, g); t.AddA(a0 + 8, g); break; }
        case RSR_GATE(TRANSPOSE_M2, HM2): case RSR_GATE(TRANSPOSE_M3, HM3): {
            const int N = op == TRANSPOSE_M2 ? 2 : 3;
            for (int r = 0; r < N; ++r)
                for (int c = 0; c < N; ++c) t.AddA(a0 + N * r + c, t.A(ao + N * c + r));
            break;
        }
        case RSR_GATE(INVERSE_M2, HM2): inverse_adjoint<P, 2>(t, vo, ao, v0, a0); break;
        case RSR_GATE(INVERSE_M3, HM3): inverse_adjoint<P, 3>(t, vo, ao, v0, a0); break;
        default: break;
    }
}

// NU: no program of the launch has a unary Float op (sin, cos, exp, sqr,
// sqrt, ln), so their forward and reverse handlers are left out.
template <int PROF, int P, bool NU>
__global__ void __launch_bounds__(kGradThreads, 16) grad_kernel(const LaunchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t item_id = blockIdx.x * (blockDim.x >> 5) + warp;
    if (item_id >= a.n_items) return;
    if (a.run_if && *a.run_if == 0u) return;
    const uint32_t cw = align4g(a.smem_code_words), cf = align4g(a.smem_const_floats);
    const uint32_t gp = min(kGradParams, a.smem_const_floats);
    const uint32_t region = cw + cf + gp * 32u + (a.smem_slots + a.smem_adj_slots) * 32u * P;
    float *base = smem + (size_t)warp * region;
    uint32_t *scode = reinterpret_cast<uint32_t *>(base);
    float *sconst = base + cw;
    float *gacc = sconst + cf;  // [param][lane] f32 gradient sums of this item's tiles
    Vf<P> *val = reinterpret_cast<Vf<P> *>(gacc + gp * 32u);
    Vf<P> *adj = val;  // values and adjoints share the slot file

    const WorkItem it = a.items[item_id];
    if (a.active && !a.active[it.prog_begin]) return;
    const ProgDesc pd = a.progs[it.prog_begin];
    const DatasetDesc ds = a.datasets[pd.dataset];
    for (uint32_t i = lane; i < pd.uop_len; i += 32) scode[i] = __ldg(a.code + pd.uop_off + i);
    for (uint32_t i = lane; i < pd.n_consts; i += 32) sconst[i] = __ldg(a.consts + pd.const_off + i);
    const uint32_t np = min(pd.n_consts, kGradParams);
    for (uint32_t k = 0; k < np; ++k) gacc[k * 32 + lane] = 0.0f;
    __syncwarp();
    const uint32_t result = scode[0], result_adj = scode[1];
    const uint32_t *code = scode + 2;
    const uint32_t n_nodes = (pd.uop_len - 2) / 5;
    TapeCtx<P> t{val, adj, sconst, ds.x, ds.stride, 0, ds.n_eval, lane};
    Kahan sse;
    for (uint32_t tile = it.tile_begin; tile < it.tile_end; ++tile) {
        t.p0 = (uint64_t)tile * (32u * P) + (uint64_t)lane * P;
        for (uint32_t i = 0; i < n_nodes; ++i) tape_forward<PROF, P, NU>(t, code + 5 * i);
        const Vf<P> pred = result == 0xFFFFFFFFu ? splat<P>(0.0f) : t.V(result);
        const Vf<P> y = load_pts<P>(ds.y + t.p0);
        Vf<P> seed;
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const bool valid = t.p0 + k < ds.n_eval;
            const float d = pred.v[k] - y.v[k];
            if (valid) sse.add(d * d);
            seed.v[k] = valid ? 2.0f * d : 0.0f;  // d(diff^2)/d pred, as in evaluator.rs:207
        }
        if (result == 0xFFFFFFFFu) continue;
        adj[result_adj * 32 + lane] = seed;  // the first contribution
        // reverse sweep; constant loads add their adjoints to gacc
        for (uint32_t i = n_nodes; i-- > 0;) tape_reverse<PROF, P, NU>(t, code + 5 * i, gacc + lane);
    }
    double *out = a.partials + (size_t)(pd.part_off + it.chunk) * (1 + kGradParams);
    const double s = warp_sum(sse.value());
    if (lane == 0) out[0] = s;
    for (uint32_t k = 0; k < kGradParams; ++k) {
        const double g = k < np ? warp_sum((double)gacc[k * 32 + lane]) : 0.0;
        if (lane == 0) out[1 + k] = g;
    }
}

// compute_mse_with_gradient epilogue (evaluator.rs:211-223).
__global__ void finalize_grad_kernel(const ProgDesc *progs, const DatasetDesc *datasets, const double *partials,
                                     uint32_t n_progs, float *mse_out, float *grad_out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_progs) return;
    const ProgDesc pd = progs[p];
    const double n = (double)datasets[pd.dataset].num_samples;
    double s = 0.0, g[kGradParams];
    for (int k = 0; k < (int)kGradParams; ++k) g[k] = 0.0;
    for (uint32_t c = 0; c < pd.n_parts; ++c) {
        const double *q = partials + (size_t)(pd.part_off + c) * (1 + kGradParams);
        s += q[0];
        for (int k = 0; k < (int)kGradParams; ++k) g[k] += q[1 + k];
    }
    float m = (float)(s / n);
    const bool bad = !(s <= (double)FLT_MAX) || !isfinite(m);
    mse_out[p] = bad ? FLT_MAX : m;
    const uint32_t np = min(pd.n_consts, kGradParams);
    for (uint32_t k = 0; k < kGradParams; ++k) grad_out[(size_t)p * kGradParams + k] = (bad || k >= np) ? 0.0f : (float)(g[k] / n);
}

template <int PROF, int P, bool NU>
static cudaError_t launch_grad_p(const LaunchArgs &a, uint32_t wpb, size_t smem, cudaStream_t st) {
    auto k = grad_kernel<PROF, P, NU>;
    static std::atomic<uint64_t> limit_raised{0};
    cudaError_t e = raise_smem_limit(k, limit_raised);
    if (e != cudaSuccess) return e;
    k<<<(a.n_items + wpb - 1) / wpb, wpb * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int PROF, bool NU>
static cudaError_t launch_grad_prof(const LaunchArgs &a, uint32_t wpb, size_t smem, cudaStream_t st) {
    return a.progs_per_warp >= 4 ? launch_grad_p<PROF, 4, NU>(a, wpb, smem, st)
         : a.progs_per_warp >= 2 ? launch_grad_p<PROF, 2, NU>(a, wpb, smem, st)
                                 : launch_grad_p<PROF, 1, NU>(a, wpb, smem, st);
}

// Kernels without the unary Float handlers exist for the F and F+V3 profiles.
bool grad_has_no_unary(int profile) { return profile == P_F || profile == P_FV3; }

cudaError_t launch_grad(const LaunchArgs &a, int profile, bool no_unary, uint32_t wpb, size_t smem, cudaStream_t st) {
    switch (profile) {
        case P_F: return no_unary ? launch_grad_prof<P_F, true>(a, wpb, smem, st)
                                  : launch_grad_prof<P_F, false>(a, wpb, smem, st);
        case P_FV3: return no_unary ? launch_grad_prof<P_FV3, true>(a, wpb, smem, st)
                                    : launch_grad_prof<P_FV3, false>(a, wpb, smem, st);
        case P_FV2M2: return launch_grad_prof<P_FV2M2, false>(a, wpb, smem, st);
        case P_FV3M3: return launch_grad_prof<P_FV3M3, false>(a, wpb, smem, st);
        default: return launch_grad_prof<P_ALL, false>(a, wpb, smem, st);
    }
}

// Loads every instance and the epilogue ahead of their first real launches:
// empty launches that return at once (one item, whose warp stops at run_if,
// a zero word; no programs for the epilogue).
template <int PROF, bool NU>
static cudaError_t preload_grad_prof(const uint32_t *zero, cudaStream_t st) {
    LaunchArgs none{};
    none.n_items = 1;
    none.run_if = zero;
    cudaError_t e;
    for (uint32_t ppw : {1u, 2u, 4u}) {
        none.progs_per_warp = ppw;
        if ((e = launch_grad_prof<PROF, NU>(none, 1, 0, st)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t preload_grad(const uint32_t *zero, cudaStream_t st) {
    const cudaError_t r[] = {preload_grad_prof<P_F, true>(zero, st),      preload_grad_prof<P_F, false>(zero, st),
                             preload_grad_prof<P_FV3, true>(zero, st),    preload_grad_prof<P_FV3, false>(zero, st),
                             preload_grad_prof<P_FV2M2, false>(zero, st), preload_grad_prof<P_FV3M3, false>(zero, st),
                             preload_grad_prof<P_ALL, false>(zero, st)};
    for (cudaError_t e : r)
        if (e != cudaSuccess) return e;
    finalize_grad_kernel<<<1, 32, 0, st>>>(nullptr, nullptr, nullptr, 0u, nullptr, nullptr);  // n_progs = 0
    return cudaGetLastError();
}

size_t grad_smem_per_warp(uint32_t code_words, uint32_t const_floats, uint32_t val_slots, uint32_t adj_slots,
                          int P) {
    const uint32_t gp = const_floats < kGradParams ? const_floats : kGradParams;
    return ((size_t)align4g(code_words) + align4g(const_floats) + gp * 32u +
            ((size_t)val_slots + adj_slots) * 32u * (size_t)P) * 4u;
}

cudaError_t launch_finalize_grad(const ProgDesc *progs, const DatasetDesc *ds, const double *partials, uint32_t n,
                                 float *mse_out, float *grad_out, cudaStream_t st) {
    finalize_grad_kernel<<<(n + 127) / 128, 128, 0, st>>>(progs, ds, partials, n, mse_out, grad_out);
    return cudaGetLastError();
}

}  // namespace rsr
