// kernels_reg.cu -- the register-stack interpreter (batched persistent
// kernel).
//
// Each typed stack of the reference VM (state.rs:12-37) is an array of
// P-point values held in registers.  A register cannot be indexed at run
// time, so the stack position is part of the dispatch: every micro-op word
// selects one (kind, position) case of a dense switch, and each case is
// straight-line code on fixed registers.  The encoder keeps positions small
// by evaluating subtrees in the order that needs the fewest slots, which
// leaves every value bit-identical to the reference's.
//
// The kernel is persistent: warps pull work items (a group of programs on a
// chunk of point tiles) from a global counter, so uneven program lengths and
// uneven dataset sizes balance across the GPU.  All programs of an item run
// on each tile while its features are hot in L1.
#include <cuda_runtime.h>

#include "kernels.h"
#include "kernels_common.cuh"

namespace rsr {

template <int N> struct AtLeast1 { static constexpr int v = N > 0 ? N : 1; };

template <int PROF, int P>
struct RegState {
    static constexpr int DF = kProfiles[PROF].cap[SF];
    static constexpr int DV2 = kProfiles[PROF].cap[SV2];
    static constexpr int DV3 = kProfiles[PROF].cap[SV3];
    static constexpr int DM2 = kProfiles[PROF].cap[SM2];
    static constexpr int DM3 = kProfiles[PROF].cap[SM3];
    static constexpr int NT = kProfiles[PROF].n_transfer;
    Vf<P> F[AtLeast1<DF>::v];
    Vf<P> V2[AtLeast1<DV2>::v][2];
    Vf<P> V3[AtLeast1<DV3>::v][3];
    Vf<P> M2[AtLeast1<DM2>::v][4];
    Vf<P> M3[AtLeast1<DM3>::v][9];
    Vf<P> T[AtLeast1<NT>::v];
};

template <int P>
struct RegIO {
    const float *x;
    uint64_t stride;
    uint64_t p0;
    const float *consts;
    __device__ __forceinline__ Vf<P> X(uint32_t f) const { return load_pts<P>(x + f * stride + p0); }
    __device__ __forceinline__ Vf<P> C(uint32_t i) const { return splat<P>(consts[i]); }
    __device__ __forceinline__ void Xn(Vf<P> *d, uint32_t f, int n) const {
#pragma unroll
        for (int i = 0; i < n; ++i) d[i] = X(f + i);
    }
    __device__ __forceinline__ void Cn(Vf<P> *d, uint32_t c, int n) const {
#pragma unroll
        for (int i = 0; i < n; ++i) d[i] = C(c + i);
    }
};

template <int P, int W>
__device__ __forceinline__ void vcopy(Vf<P> *d, const Vf<P> *s) {
#pragma unroll
    for (int i = 0; i < W; ++i) d[i] = s[i];
}

// Same-stack binary operations of width W: a = a op b, op selected by OPK:
// 0 add, 1 sub, 2 reversed sub (b - a), 3 cross, 4 reversed cross,
// 5 mat-mul (M2 if W == 4, M3 if W == 9), 6 reversed mat-mul.
template <int P, int W, int OPK>
__device__ __forceinline__ void bin_op(Vf<P> *a, const Vf<P> *b) {
    if constexpr (OPK == 0) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = a[i] + b[i];
    } else if constexpr (OPK == 1) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = a[i] - b[i];
    } else if constexpr (OPK == 2) {
#pragma unroll
        for (int i = 0; i < W; ++i) a[i] = b[i] - a[i];
    } else if constexpr (OPK == 3) {
        cross3(a, b, a);
    } else if constexpr (OPK == 4) {
        cross3(b, a, a);
    } else if constexpr (OPK == 5) {
        if constexpr (W == 4) mul_m2(a, b, a); else mul_m3(a, b, a);
    } else {
        if constexpr (W == 4) mul_m2(b, a, a); else mul_m3(b, a, a);
    }
}

// One register micro-op (kind K at stack position S).
template <int PROF, int P, int K, int S>
__device__ __forceinline__ void uop(RegState<PROF, P> &st, const RegIO<P> &io, uint32_t arg) {
    using St = RegState<PROF, P>;
    constexpr int DF = St::DF, DV2 = St::DV2, DV3 = St::DV3, DM2 = St::DM2, DM3 = St::DM3, NT = St::NT;
    // ------------------------------------------------------------ F stack
    if constexpr (K <= U_F_LN) {
        if constexpr (S < DF) {
            Vf<P> &a = st.F[S];
            if constexpr (K == U_F_LDX) a = io.X(arg);
            else if constexpr (K == U_F_LDC) a = io.C(arg);
            else if constexpr (K == U_F_FROM_T0) a = st.T[0];
            else if constexpr (K == U_F_TO_T0) st.T[0] = a;
            else if constexpr (K == U_F_TO_T1) { if constexpr (NT > 1) st.T[1] = a; }
            else if constexpr (K == U_F_TO_T2) { if constexpr (NT > 2) st.T[2] = a; }
            else if constexpr (K >= U_F_ADD && K <= U_F_RDIV) {
                if constexpr (S + 1 < DF) {
                    const Vf<P> &b = st.F[S + 1];
                    if constexpr (K == U_F_ADD) a = a + b;
                    else if constexpr (K == U_F_SUB) a = a - b;
                    else if constexpr (K == U_F_RSUB) a = b - a;
                    else if constexpr (K == U_F_MUL) a = a * b;
                    else if constexpr (K == U_F_DIV) a = a / b;
                    else a = b / a;
                }
            } else if constexpr (K >= U_F_ADDX && K <= U_F_RDIVC) {
                constexpr int k6 = (K - U_F_ADDX) % 6;
                const Vf<P> b = (K <= U_F_RDIVX) ? io.X(arg) : io.C(arg);
                if constexpr (k6 == 0) a = a + b;
                else if constexpr (k6 == 1) a = a - b;
                else if constexpr (k6 == 2) a = b - a;
                else if constexpr (k6 == 3) a = a * b;
                else if constexpr (k6 == 4) a = a / b;
                else a = b / a;
            } else if constexpr (K == U_F_SIN) a = vsin(a);
            else if constexpr (K == U_F_COS) a = vcos(a);
            else if constexpr (K == U_F_EXP) a = vexp(a);
            else if constexpr (K == U_F_SQR) a = a * a;
            else if constexpr (K == U_F_SQRT) a = vsqrt(a);
            else if constexpr (K == U_F_LN) a = vlog(a);
        }
    }
    // ----------------------------------------------------------- V2 stack
    else if constexpr (K >= U_V2_LDX && K <= U_V2_MULMC) {
        if constexpr (S < DV2) {
            Vf<P> *a = st.V2[S];
            if constexpr (K == U_V2_LDX) io.Xn(a, arg, 2);
            else if constexpr (K == U_V2_LDC) io.Cn(a, arg, 2);
            else if constexpr (K == U_V2_FROM_T) { if constexpr (NT >= 2) vcopy<P, 2>(a, st.T); }
            else if constexpr (K == U_V2_TO_T0) { if constexpr (NT >= 2) vcopy<P, 2>(st.T, a); }
            else if constexpr (K == U_V2_TO_T2) { if constexpr (NT >= 4) vcopy<P, 2>(st.T + 2, a); }
            else if constexpr (K >= U_V2_ADD && K <= U_V2_RSUB) {
                if constexpr (S + 1 < DV2) bin_op<P, 2, K - U_V2_ADD>(a, st.V2[S + 1]);
            } else if constexpr (K >= U_V2_ADDX && K <= U_V2_RSUBC) {
                Vf<P> b[2];
                if constexpr (K <= U_V2_RSUBX) io.Xn(b, arg, 2); else io.Cn(b, arg, 2);
                bin_op<P, 2, (K - U_V2_ADDX) % 3>(a, b);
            } else if constexpr (K == U_V2_SCALE_T || K == U_V2_SCALE_X || K == U_V2_SCALE_C) {
                const Vf<P> s = K == U_V2_SCALE_T ? st.T[0] : K == U_V2_SCALE_X ? io.X(arg) : io.C(arg);
                a[0] = a[0] * s; a[1] = a[1] * s;
            } else if constexpr (K == U_V2_DOT_T) {
                if constexpr (S + 1 < DV2) st.T[0] = dot2(a, st.V2[S + 1]);
            } else if constexpr (K == U_V2_DOTX_T || K == U_V2_DOTC_T) {
                Vf<P> b[2];
                if constexpr (K == U_V2_DOTX_T) io.Xn(b, arg, 2); else io.Cn(b, arg, 2);
                st.T[0] = dot2(a, b);
            } else if constexpr (K == U_V2_NORM_T) st.T[0] = norm2(a);
            else if constexpr (K == U_V2_GETX_T) st.T[0] = a[0];
            else if constexpr (K == U_V2_GETY_T) st.T[0] = a[1];
            else if constexpr (K == U_V2_MULM_T) { if constexpr (NT >= 4) mul_m2v2(st.T, a, a); }
            else if constexpr (K == U_V2_MULMX || K == U_V2_MULMC) {
                Vf<P> m[4];
                if constexpr (K == U_V2_MULMX) io.Xn(m, arg, 4); else io.Cn(m, arg, 4);
                mul_m2v2(m, a, a);
            }
        }
    }
    // ----------------------------------------------------------- V3 stack
    else if constexpr (K >= U_V3_LDX && K <= U_V3_MULMC) {
        if constexpr (S < DV3) {
            Vf<P> *a = st.V3[S];
            if constexpr (K == U_V3_LDX) io.Xn(a, arg, 3);
            else if constexpr (K == U_V3_LDC) io.Cn(a, arg, 3);
            else if constexpr (K == U_V3_FROM_T) { if constexpr (NT >= 3) vcopy<P, 3>(a, st.T); }
            else if constexpr (K == U_V3_TO_T0) { if constexpr (NT >= 3) vcopy<P, 3>(st.T, a); }
            else if constexpr (K == U_V3_TO_T3) { if constexpr (NT >= 6) vcopy<P, 3>(st.T + 3, a); }
            else if constexpr (K == U_V3_TO_T6) { if constexpr (NT >= 9) vcopy<P, 3>(st.T + 6, a); }
            else if constexpr (K >= U_V3_ADD && K <= U_V3_RCROSS) {
                if constexpr (S + 1 < DV3) bin_op<P, 3, K - U_V3_ADD>(a, st.V3[S + 1]);
            } else if constexpr (K >= U_V3_ADDX && K <= U_V3_RCROSSC) {
                Vf<P> b[3];
                if constexpr (K <= U_V3_RCROSSX) io.Xn(b, arg, 3); else io.Cn(b, arg, 3);
                bin_op<P, 3, (K - U_V3_ADDX) % 5>(a, b);
            } else if constexpr (K == U_V3_SCALE_T || K == U_V3_SCALE_X || K == U_V3_SCALE_C) {
                const Vf<P> s = K == U_V3_SCALE_T ? st.T[0] : K == U_V3_SCALE_X ? io.X(arg) : io.C(arg);
                a[0] = a[0] * s; a[1] = a[1] * s; a[2] = a[2] * s;
            } else if constexpr (K == U_V3_DOT_T) {
                if constexpr (S + 1 < DV3) st.T[0] = dot3(a, st.V3[S + 1]);
            } else if constexpr (K == U_V3_DOTX_T || K == U_V3_DOTC_T) {
                Vf<P> b[3];
                if constexpr (K == U_V3_DOTX_T) io.Xn(b, arg, 3); else io.Cn(b, arg, 3);
                st.T[0] = dot3(a, b);
            } else if constexpr (K == U_V3_NORM_T) st.T[0] = norm3(a);
            else if constexpr (K == U_V3_GETX_T) st.T[0] = a[0];
            else if constexpr (K == U_V3_GETY_T) st.T[0] = a[1];
            else if constexpr (K == U_V3_GETZ_T) st.T[0] = a[2];
            else if constexpr (K == U_V3_MULM_T) { if constexpr (NT >= 9) mul_m3v3(st.T, a, a); }
            else if constexpr (K == U_V3_MULMX || K == U_V3_MULMC) {
                Vf<P> m[9];
                if constexpr (K == U_V3_MULMX) io.Xn(m, arg, 9); else io.Cn(m, arg, 9);
                mul_m3v3(m, a, a);
            }
        }
    }
    // ------------------------------------------------------- M2 / M3 stacks
    else if constexpr (K >= U_M2_LDX && K <= U_M3_INVERSE) {
        constexpr bool is3 = K >= U_M3_LDX;
        constexpr int W = is3 ? 9 : 4;
        constexpr int D = is3 ? DM3 : DM2;
        constexpr int k = K - (is3 ? U_M3_LDX : U_M2_LDX);  // offset within the M block
        if constexpr (S < D) {
            Vf<P> *a;
            if constexpr (is3) a = st.M3[S]; else a = st.M2[S];
            if constexpr (k == 0) io.Xn(a, arg, W);
            else if constexpr (k == 1) io.Cn(a, arg, W);
            else if constexpr (k == 2) { if constexpr (NT >= W) vcopy<P, W>(a, st.T); }
            else if constexpr (k == 3) { if constexpr (NT >= W) vcopy<P, W>(st.T, a); }
            else if constexpr (k >= 4 && k <= 8) {  // ADD SUB RSUB MUL RMUL (stack)
                if constexpr (S + 1 < D) {
                    Vf<P> *b;
                    if constexpr (is3) b = st.M3[S + 1]; else b = st.M2[S + 1];
                    constexpr int opk = k == 4 ? 0 : k == 5 ? 1 : k == 6 ? 2 : k == 7 ? 5 : 6;
                    bin_op<P, W, opk>(a, b);
                }
            } else if constexpr (k >= 9 && k <= 18) {  // X and C forms
                Vf<P> b[W];
                if constexpr (k <= 13) io.Xn(b, arg, W); else io.Cn(b, arg, W);
                constexpr int j = (k - 9) % 5;
                constexpr int opk = j == 0 ? 0 : j == 1 ? 1 : j == 2 ? 2 : j == 3 ? 5 : 6;
                bin_op<P, W, opk>(a, b);
            } else if constexpr (k >= 19 && k <= 21) {  // SCALE_T / X / C
                const Vf<P> s = k == 19 ? st.T[0] : k == 20 ? io.X(arg) : io.C(arg);
#pragma unroll
                for (int i = 0; i < W; ++i) a[i] = a[i] * s;
            } else if constexpr (k == 22) {
                if constexpr (is3) st.T[0] = det_m3(a); else st.T[0] = det_m2(a);
            } else if constexpr (k == 23) {
                if constexpr (is3) st.T[0] = trace_m3(a); else st.T[0] = trace_m2(a);
            } else if constexpr (k == 24) {
                if constexpr (is3) transpose_m3(a, a); else transpose_m2(a, a);
            } else if constexpr (k == 25) {
                if constexpr (is3) inverse_m3(a, a); else inverse_m2(a, a);
            }
        }
    }
}

#define RSR_C(K, S) case ((K) << 3) | (S): uop<PROF, P, (K), (S)>(st, io, arg); break;
#define RSR_K(K) RSR_C(K, 0) RSR_C(K, 1) RSR_C(K, 2) RSR_C(K, 3) RSR_C(K, 4) RSR_C(K, 5) RSR_C(K, 6) RSR_C(K, 7)

// Runs one program (register form) on this lane's P points.  One flat
// switch over (kind, position); cases of stacks the profile does not hold
// compile to nothing.
template <int PROF, int P>
__device__ __forceinline__ void run_program(RegState<PROF, P> &st, const RegIO<P> &io, const uint32_t *code,
                                            uint32_t len) {
    uint32_t w = code[0];
    for (uint32_t pc = 0; pc < len; ++pc) {
        const uint32_t wn = code[pc + 1];
        const uint32_t arg = w >> 11;
        switch (w & 0x7FFu) {
            RSR_K(U_F_LDX) RSR_K(U_F_LDC) RSR_K(U_F_FROM_T0) RSR_K(U_F_TO_T0) RSR_K(U_F_TO_T1) RSR_K(U_F_TO_T2)
            RSR_K(U_F_ADD) RSR_K(U_F_SUB) RSR_K(U_F_RSUB) RSR_K(U_F_MUL) RSR_K(U_F_DIV) RSR_K(U_F_RDIV)
            RSR_K(U_F_ADDX) RSR_K(U_F_SUBX) RSR_K(U_F_RSUBX) RSR_K(U_F_MULX) RSR_K(U_F_DIVX) RSR_K(U_F_RDIVX)
            RSR_K(U_F_ADDC) RSR_K(U_F_SUBC) RSR_K(U_F_RSUBC) RSR_K(U_F_MULC) RSR_K(U_F_DIVC) RSR_K(U_F_RDIVC)
            RSR_K(U_F_SIN) RSR_K(U_F_COS) RSR_K(U_F_EXP) RSR_K(U_F_SQR) RSR_K(U_F_SQRT) RSR_K(U_F_LN)
            RSR_K(U_V2_LDX) RSR_K(U_V2_LDC) RSR_K(U_V2_FROM_T) RSR_K(U_V2_TO_T0) RSR_K(U_V2_TO_T2)
            RSR_K(U_V2_ADD) RSR_K(U_V2_SUB) RSR_K(U_V2_RSUB) RSR_K(U_V2_ADDX) RSR_K(U_V2_SUBX)
            RSR_K(U_V2_RSUBX) RSR_K(U_V2_ADDC) RSR_K(U_V2_SUBC) RSR_K(U_V2_RSUBC)
            RSR_K(U_V2_SCALE_T) RSR_K(U_V2_SCALE_X) RSR_K(U_V2_SCALE_C)
            RSR_K(U_V2_DOT_T) RSR_K(U_V2_DOTX_T) RSR_K(U_V2_DOTC_T) RSR_K(U_V2_NORM_T)
            RSR_K(U_V2_GETX_T) RSR_K(U_V2_GETY_T) RSR_K(U_V2_MULM_T) RSR_K(U_V2_MULMX) RSR_K(U_V2_MULMC)
            RSR_K(U_V3_LDX) RSR_K(U_V3_LDC) RSR_K(U_V3_FROM_T) RSR_K(U_V3_TO_T0) RSR_K(U_V3_TO_T3)
            RSR_K(U_V3_TO_T6) RSR_K(U_V3_ADD) RSR_K(U_V3_SUB) RSR_K(U_V3_RSUB) RSR_K(U_V3_CROSS)
            RSR_K(U_V3_RCROSS) RSR_K(U_V3_ADDX) RSR_K(U_V3_SUBX) RSR_K(U_V3_RSUBX)
            RSR_K(U_V3_CROSSX) RSR_K(U_V3_RCROSSX) RSR_K(U_V3_ADDC) RSR_K(U_V3_SUBC)
            RSR_K(U_V3_RSUBC) RSR_K(U_V3_CROSSC) RSR_K(U_V3_RCROSSC)
            RSR_K(U_V3_SCALE_T) RSR_K(U_V3_SCALE_X) RSR_K(U_V3_SCALE_C)
            RSR_K(U_V3_DOT_T) RSR_K(U_V3_DOTX_T) RSR_K(U_V3_DOTC_T) RSR_K(U_V3_NORM_T)
            RSR_K(U_V3_GETX_T) RSR_K(U_V3_GETY_T) RSR_K(U_V3_GETZ_T)
            RSR_K(U_V3_MULM_T) RSR_K(U_V3_MULMX) RSR_K(U_V3_MULMC)
            RSR_K(U_M2_LDX) RSR_K(U_M2_LDC) RSR_K(U_M2_FROM_T) RSR_K(U_M2_TO_T)
            RSR_K(U_M2_ADD) RSR_K(U_M2_SUB) RSR_K(U_M2_RSUB) RSR_K(U_M2_MUL) RSR_K(U_M2_RMUL)
            RSR_K(U_M2_ADDX) RSR_K(U_M2_SUBX) RSR_K(U_M2_RSUBX) RSR_K(U_M2_MULX) RSR_K(U_M2_RMULX)
            RSR_K(U_M2_ADDC) RSR_K(U_M2_SUBC) RSR_K(U_M2_RSUBC) RSR_K(U_M2_MULC) RSR_K(U_M2_RMULC)
            RSR_K(U_M2_SCALE_T) RSR_K(U_M2_SCALE_X) RSR_K(U_M2_SCALE_C)
            RSR_K(U_M2_DET_T) RSR_K(U_M2_TRACE_T) RSR_K(U_M2_TRANSPOSE) RSR_K(U_M2_INVERSE)
            RSR_K(U_M3_LDX) RSR_K(U_M3_LDC) RSR_K(U_M3_FROM_T) RSR_K(U_M3_TO_T)
            RSR_K(U_M3_ADD) RSR_K(U_M3_SUB) RSR_K(U_M3_RSUB) RSR_K(U_M3_MUL) RSR_K(U_M3_RMUL)
            RSR_K(U_M3_ADDX) RSR_K(U_M3_SUBX) RSR_K(U_M3_RSUBX) RSR_K(U_M3_MULX) RSR_K(U_M3_RMULX)
            RSR_K(U_M3_ADDC) RSR_K(U_M3_SUBC) RSR_K(U_M3_RSUBC) RSR_K(U_M3_MULC) RSR_K(U_M3_RMULC)
            RSR_K(U_M3_SCALE_T) RSR_K(U_M3_SCALE_X) RSR_K(U_M3_SCALE_C)
            RSR_K(U_M3_DET_T) RSR_K(U_M3_TRACE_T) RSR_K(U_M3_TRANSPOSE) RSR_K(U_M3_INVERSE)
            default: break;
        }
        w = wn;
    }
}

#undef RSR_K
#undef RSR_C

__host__ __device__ __forceinline__ uint32_t align4r(uint32_t v) { return (v + 3u) & ~3u; }

constexpr uint32_t kMaxProgsPerWarp = 8;

template <int PROF, int P>
__global__ void __launch_bounds__(kRegThreads) reg_eval_kernel(const LaunchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t region = align4r(a.smem_code_words) + align4r(a.smem_const_floats) + 2u * 32u * kMaxProgsPerWarp;
    float *base = smem + (size_t)warp * region;
    uint32_t *scode = reinterpret_cast<uint32_t *>(base);
    float *sconst = base + align4r(a.smem_code_words);
    float *sacc = sconst + align4r(a.smem_const_floats);  // [g][2][32] Kahan state
    __shared__ uint32_t meta[kRegThreads / 32][kMaxProgsPerWarp][3];  // code off, len, const off

    for (;;) {
        uint32_t item_id = 0;
        if (lane == 0) item_id = atomicAdd(a.item_counter, 1u);
        item_id = __shfl_sync(0xffffffffu, item_id, 0);
        if (item_id >= a.n_items) break;
        const WorkItem it = a.items[item_id];
        const uint32_t G = it.n_progs;
        // stage the programs of this item
        uint32_t coff = 0, koff = 0;
        for (uint32_t g = 0; g < G; ++g) {
            const ProgDesc pd = a.progs[it.prog_begin + g];
            for (uint32_t i = lane; i < pd.uop_len; i += 32) scode[coff + i] = __ldg(a.code + pd.uop_off + i);
            if (lane == 0) scode[coff + pd.uop_len] = 0u;  // prefetch pad
            for (uint32_t i = lane; i < pd.n_consts; i += 32) sconst[koff + i] = __ldg(a.consts + pd.const_off + i);
            if (lane == 0) { meta[warp][g][0] = coff; meta[warp][g][1] = pd.uop_len; meta[warp][g][2] = koff; }
            sacc[(g * 2) * 32 + lane] = 0.0f;
            sacc[(g * 2 + 1) * 32 + lane] = 0.0f;
            coff += pd.uop_len + 1;
            koff += pd.n_consts;
        }
        __syncwarp();
        const ProgDesc pd0 = a.progs[it.prog_begin];
        const DatasetDesc ds = a.datasets[pd0.dataset];
        RegState<PROF, P> st;
        RegIO<P> io{ds.x, ds.stride, 0, sconst};
        for (uint32_t tile = it.tile_begin; tile < it.tile_end; ++tile) {
            io.p0 = (uint64_t)tile * (32u * P) + (uint64_t)lane * P;
            const Vf<P> y = load_pts<P>(ds.y + io.p0);
            for (uint32_t g = 0; g < G; ++g) {
                io.consts = sconst + meta[warp][g][2];
                run_program<PROF, P>(st, io, scode + meta[warp][g][0], meta[warp][g][1]);
                const Vf<P> pred = st.F[0];
                if (a.mode == MODE_POINTS) {
                    store_pts<P>(a.points_out + (uint64_t)(it.prog_begin + g) * a.points_stride + io.p0, pred, io.p0,
                                 ds.n_eval);
                } else {
                    Kahan acc;
                    acc.s = sacc[(g * 2) * 32 + lane];
                    acc.c = sacc[(g * 2 + 1) * 32 + lane];
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        if (io.p0 + k < ds.n_eval) {
                            const float d = pred.v[k] - y.v[k];
                            acc.add(d * d);
                        }
                    }
                    sacc[(g * 2) * 32 + lane] = acc.s;
                    sacc[(g * 2 + 1) * 32 + lane] = acc.c;
                }
            }
        }
        if (a.mode == MODE_MSE) {
            for (uint32_t g = 0; g < G; ++g) {
                Kahan acc;
                acc.s = sacc[(g * 2) * 32 + lane];
                acc.c = sacc[(g * 2 + 1) * 32 + lane];
                const double s = warp_sum(acc.value());
                if (lane == 0) a.partials[a.progs[it.prog_begin + g].part_off + it.chunk] = s;
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------- launchers
template <int PROF, int P>
static cudaError_t launch_reg_pp(const LaunchArgs &a, uint32_t grid, cudaStream_t st) {
    auto k = reg_eval_kernel<PROF, P>;
    const size_t smem = reg_smem_per_warp(a.smem_code_words, a.smem_const_floats) * (kRegThreads / 32);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, kRegThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int PROF>
static cudaError_t launch_reg_prof(const LaunchArgs &a, int P, uint32_t grid, cudaStream_t st) {
    switch (P) {
        case 1: return launch_reg_pp<PROF, 1>(a, grid, st);
        case 2: return launch_reg_pp<PROF, 2>(a, grid, st);
        default:
            if constexpr (PROF == P_ALL) return launch_reg_pp<PROF, 2>(a, grid, st);
            else return launch_reg_pp<PROF, 4>(a, grid, st);
    }
}

cudaError_t launch_reg(const LaunchArgs &a, int profile, int P, uint32_t grid, cudaStream_t st) {
    switch (profile) {
        case P_F: return P == 8 ? launch_reg_pp<P_F, 8>(a, grid, st) : launch_reg_prof<P_F>(a, P, grid, st);
        case P_FV3: return launch_reg_prof<P_FV3>(a, P, grid, st);
        case P_FV2M2: return launch_reg_prof<P_FV2M2>(a, P, grid, st);
        case P_FV3M3: return launch_reg_prof<P_FV3M3>(a, P, grid, st);
        default: return launch_reg_prof<P_ALL>(a, P, grid, st);
    }
}

size_t reg_smem_per_warp(uint32_t code_words, uint32_t const_floats) {
    return ((size_t)align4r(code_words) + align4r(const_floats) + 2u * 32u * kMaxProgsPerWarp) * 4u;
}

template <int PROF, int P>
static int occ(size_t smem) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, reg_eval_kernel<PROF, P>, kRegThreads, smem);
    return n;
}

int reg_max_blocks_per_sm(int profile, int P) {
    const size_t smem = reg_smem_per_warp(512, 256) * (kRegThreads / 32);
    switch (profile) {
        case P_F: return P == 8 ? occ<P_F, 8>(smem) : P == 4 ? occ<P_F, 4>(smem) : P == 2 ? occ<P_F, 2>(smem) : occ<P_F, 1>(smem);
        case P_FV3: return P >= 4 ? occ<P_FV3, 4>(smem) : P == 2 ? occ<P_FV3, 2>(smem) : occ<P_FV3, 1>(smem);
        case P_FV2M2: return P >= 4 ? occ<P_FV2M2, 4>(smem) : P == 2 ? occ<P_FV2M2, 2>(smem) : occ<P_FV2M2, 1>(smem);
        case P_FV3M3: return P >= 4 ? occ<P_FV3M3, 4>(smem) : P == 2 ? occ<P_FV3M3, 2>(smem) : occ<P_FV3M3, 1>(smem);
        default: return P >= 2 ? occ<P_ALL, 2>(smem) : occ<P_ALL, 1>(smem);
    }
}

}  // namespace rsr
