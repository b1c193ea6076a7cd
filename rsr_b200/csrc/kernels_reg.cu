// kernels_reg.cu -- the batched register kernel: an accumulator machine.
//
// Each value type of the reference VM (state.rs:12-37) has one accumulator
// register set holding P data points per lane: A_F, A_V2[2], A_V3[3],
// A_M2[4], A_M3[9].  Micro-ops (uops.h, accumulator form) combine an
// accumulator with a feature, a constant, a value spilled to a per-type
// stack in shared memory (slot fixed by the encoder), or another type's
// accumulator, so dispatch is on the micro-op kind alone (about 140 cases,
// one code block each) and values never leave registers except for spills.
//
// The kernel is persistent: warps pull work items (up to 8 programs sharing a
// dataset, on a chunk of point tiles) from a global counter, so uneven
// program lengths and dataset sizes balance across the 148 SMs; all programs
// of an item run on each tile while its features are hot in L1.
#include <cuda_runtime.h>

#include "kernels.h"
#include "kernels_common.cuh"

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

template <int P>
struct AccIO {
    const float *xl;        // this lane's first point of feature 0 in the current tile
    uint32_t stride;        // floats between features
    const float *consts;
    Vf<P> *stk[N_STACKS];   // per-type shared-memory stacks of this lane: [(slot*W + c)*32]
    __device__ __forceinline__ Vf<P> X(uint32_t f) const { return load_pts<P>(xl + (size_t)f * stride); }
    __device__ __forceinline__ Vf<P> C(uint32_t i) const { return splat<P>(consts[i]); }
    template <int W>
    __device__ __forceinline__ Vf<P> &S(int t, uint32_t slot, int c) const { return stk[t][(slot * W + c) * 32]; }
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
            for (int c = 0; c < W; ++c) io.template S<W>(t, slot, c) = A[c];
            if (lt) load_any<PROF, P>(a, io, lt - 1u, (arg >> 7) & 1u, arg >> 8);
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

#define RSR_C(K) case (K): acc_op<PROF, P, (K)>(a, io, arg); break;
#define RSR_C4(K) RSR_C(K) RSR_C(K + 1) RSR_C(K + 2) RSR_C(K + 3)
#define RSR_C9(K) RSR_C4(K) RSR_C4(K + 4) RSR_C(K + 8)
#define RSR_C27(K) RSR_C9(K) RSR_C9(K + 9) RSR_C9(K + 18)
#define RSR_BLOCK_F RSR_C27(K_F)     // 0..26
#define RSR_BLOCK_F_NU RSR_C9(K_F) RSR_C9(K_F + 9) RSR_C(K_F + 18) RSR_C(K_F + 19) RSR_C(K_F + 20)  // 0..20
static_assert(K_F_UN == K_F + 21 && K_F_END == K_F + 27, "Float block: 21 kinds, then the 6 unary ones");
// Vec3 block without the mat-vec kinds whose matrix is a feature, a constant
// or a spilled value (64 + 30..32)
#define RSR_BLOCK_V3_NM RSR_C27(K_V3) RSR_C(K_V3 + 27) RSR_C(K_V3 + 28) RSR_C(K_V3 + 29) RSR_C(K_V3 + 33)
static_assert(kv_mulm(5, 3) == 29 && kv_make(5, 3) == 33, "Vec3 block: mat-vec kinds at 29..32");
// Vec3 block as the F+V3 profile can meet it: a mat-vec with a spilled matrix
// (64 + 32) needs a Mat3 accumulator, which that profile does not have
#define RSR_BLOCK_V3_F RSR_C27(K_V3) RSR_C4(K_V3 + 27) RSR_C(K_V3 + 31) RSR_C(K_V3 + 33)
#define RSR_BLOCK_V2 RSR_C27(K_V2)   // 32..58
#define RSR_BLOCK_V3 RSR_C27(K_V3) RSR_C4(K_V3 + 27) RSR_C(K_V3 + 31) RSR_C(K_V3 + 32) RSR_C(K_V3 + 33)  // 64..97
#define RSR_BLOCK_M2 RSR_C27(K_M2)   // 104..130
#define RSR_BLOCK_M3 RSR_C27(K_M3)   // 136..162

// Runs one program (accumulator form) on this lane's P points; the result
// is left in A_F.  OMIT: handlers left out of the kernel because no program
// of the launch needs them -- bit 0: the unary Float ops (sin, cos, exp,
// sqr, sqrt, ln); bit 1 (F+V3 profile): mat-vec products whose matrix is a
// feature, a constant or a spilled value.
template <int PROF, int P, int OMIT>
__device__ __forceinline__ void run_program(Acc<PROF, P> &a, const AccIO<P> &io, const uint32_t *code,
                                            uint32_t len) {
    // Each profile's switch lists only its own types' kinds, so the branch
    // tree the compiler builds for it is as shallow as the profile allows.
    uint32_t w = code[0];
    for (uint32_t pc = 0; pc < len; ++pc) {
        const uint32_t wn = code[pc + 1];
        const uint32_t arg = w >> 8;
        const uint32_t kind = w & 0xFFu;
        constexpr bool NU = (OMIT & 1) != 0, NM = (OMIT & 2) != 0;
        if constexpr (PROF == P_F && NU) {
            switch (kind) { RSR_BLOCK_F_NU default: break; }
        } else if constexpr (PROF == P_F) {
            switch (kind) { RSR_BLOCK_F default: break; }
        } else if constexpr (PROF == P_FV3 && NU && NM) {
            switch (kind) { RSR_BLOCK_F_NU RSR_BLOCK_V3_NM default: break; }
        } else if constexpr (PROF == P_FV3 && NU) {
            switch (kind) { RSR_BLOCK_F_NU RSR_BLOCK_V3_F default: break; }
        } else if constexpr (PROF == P_FV3 && NM) {
            switch (kind) { RSR_BLOCK_F RSR_BLOCK_V3_NM default: break; }
        } else if constexpr (PROF == P_FV3) {
            switch (kind) { RSR_BLOCK_F RSR_BLOCK_V3_F default: break; }
        } else if constexpr (PROF == P_FV2M2 && NU) {
            switch (kind) { RSR_BLOCK_F_NU RSR_BLOCK_V2 RSR_BLOCK_M2 default: break; }
        } else if constexpr (PROF == P_FV2M2) {
            switch (kind) { RSR_BLOCK_F RSR_BLOCK_V2 RSR_BLOCK_M2 default: break; }
        } else if constexpr (PROF == P_FV3M3) {
            switch (kind) { RSR_BLOCK_F RSR_BLOCK_V3 RSR_BLOCK_M3 default: break; }
        } else {
            switch (kind) { RSR_BLOCK_F RSR_BLOCK_V2 RSR_BLOCK_V3 RSR_BLOCK_M2 RSR_BLOCK_M3 default: break; }
        }
        w = wn;
    }
}

#undef RSR_BLOCK_F
#undef RSR_BLOCK_F_NU
#undef RSR_BLOCK_V3_NM
#undef RSR_BLOCK_V3_F
#undef RSR_BLOCK_V2
#undef RSR_BLOCK_V3
#undef RSR_BLOCK_M2
#undef RSR_BLOCK_M3
#undef RSR_C27
#undef RSR_C9
#undef RSR_C4
#undef RSR_C

__host__ __device__ __forceinline__ uint32_t align4r(uint32_t v) { return (v + 3u) & ~3u; }

constexpr uint32_t kMaxProgsPerWarp = 8;

// Block-cooperative item loop.  All warps of a block run the same programs
// (one work item) on different tiles of the item's chunk, so the SM's
// instruction cache holds one program's case bodies instead of one per warp.
// Per-warp Kahan sums are reduced across warps in a fixed order.
//
// Shared memory: block header (code | constants | meta | cross-warp sums)
// then one region per warp (spill stacks | Kahan state).
// Blocks per SM each instance is compiled for (the register cap follows):
// as many as its accumulators allow without spilling.
// At four points per lane a fourth block (64 registers, a few bytes of
// spill) pays for the F and F+V3 profiles (vector workload: 4.75 ms against
// 5.14 ms at three blocks); F+V2+M2 spills more there and keeps three.  At
// eight points, the F+V3 instances without the leaf-matrix mat-vec handlers
// fit a third block (80 registers, 52 bytes of spill; vector workload 4.29
// ms against 4.50 ms at two blocks); with those handlers they spill twice as
// much and keep two.
template <int PROF, int P, int OMIT>
constexpr int reg_min_blocks() {
    if constexpr (PROF == P_ALL) return P >= 4 ? 1 : 2;
    else if constexpr (PROF == P_FV3M3) return P >= 4 ? 2 : 3;
    else if constexpr (PROF == P_FV2M2) return P >= 8 ? 2 : P >= 4 ? 3 : 4;
    else if constexpr (PROF == P_FV3 && (OMIT & 2) != 0) return P >= 8 ? 3 : 4;
    else return P >= 8 ? 2 : 4;
}

template <int PROF, int P, int OMIT>
__global__ void __launch_bounds__(kRegThreads, reg_min_blocks<PROF, P, OMIT>()) reg_eval_kernel(const LaunchArgs a) {
    extern __shared__ __align__(16) float smem[];
    if (a.run_if && *a.run_if == 0u) return;  // the same for every thread of the launch
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    uint32_t *scode = reinterpret_cast<uint32_t *>(smem);
    float *sconst = smem + align4r(a.smem_code_words);
    uint32_t *meta = reinterpret_cast<uint32_t *>(sconst + align4r(a.smem_const_floats));  // [g][3], [24] item
    double *red = reinterpret_cast<double *>(meta + 32);                                  // [warp][g]
    float *wbase = smem + a.block_hdr_floats + (size_t)warp * a.region_floats;
    float *sacc = wbase + a.acc_off;  // [g][2][32] Kahan state of this warp

    AccIO<P> io;
#pragma unroll
    for (int t = 0; t < N_STACKS; ++t) io.stk[t] = reinterpret_cast<Vf<P> *>(wbase + a.stack_off[t]) + lane;

    for (;;) {
        if (threadIdx.x == 0) meta[24] = atomicAdd(a.item_counter, 1u);
        __syncthreads();
        const uint32_t item_id = meta[24];
        if (item_id >= a.n_items) break;
        const WorkItem it = a.items[item_id];
        const uint32_t G = it.n_progs;
        if (a.active) {
            // an item whose programs have all finished (fits) is skipped whole;
            // the flags are the same for every thread of the block
            bool any = false;
            for (uint32_t g = 0; g < G; ++g) any |= a.active[it.prog_begin + g] != 0;
            if (!any) {
                __syncthreads();  // meta[24] is rewritten by the next item fetch
                continue;
            }
        }
        if (threadIdx.x == 0) {
            uint32_t coff = 0, koff = 0;
            for (uint32_t g = 0; g < G; ++g) {
                const ProgDesc pd = a.progs[it.prog_begin + g];
                meta[3 * g] = coff;
                meta[3 * g + 1] = pd.uop_len;
                meta[3 * g + 2] = koff;
                scode[coff + pd.uop_len] = 0u;  // prefetch pad
                coff += pd.uop_len + 1;
                koff += pd.n_consts;
            }
        }
        __syncthreads();
        for (uint32_t g = 0; g < G; ++g) {
            const ProgDesc pd = a.progs[it.prog_begin + g];
            for (uint32_t i = threadIdx.x; i < pd.uop_len; i += blockDim.x) scode[meta[3 * g] + i] = __ldg(a.code + pd.uop_off + i);
            for (uint32_t i = threadIdx.x; i < pd.n_consts; i += blockDim.x)
                sconst[meta[3 * g + 2] + i] = __ldg(a.consts + pd.const_off + i);
            sacc[(g * 2) * 32 + lane] = 0.0f;
            sacc[(g * 2 + 1) * 32 + lane] = 0.0f;
        }
        __syncthreads();
        const DatasetDesc ds = a.datasets[a.progs[it.prog_begin].dataset];
        io.stride = (uint32_t)ds.stride;
        Acc<PROF, P> acc;
        for (uint32_t tile = it.tile_begin + warp; tile < it.tile_end; tile += nw) {
            const uint64_t p0 = (uint64_t)tile * (32u * P) + (uint64_t)lane * P;
            io.xl = ds.x + p0;
            const Vf<P> y = load_pts<P>(ds.y + p0);
            const bool full = p0 + P <= ds.n_eval;
            for (uint32_t g = 0; g < G; ++g) {
                if (a.active && !a.active[it.prog_begin + g]) continue;
                io.consts = sconst + meta[3 * g + 2];
                run_program<PROF, P, OMIT>(acc, io, scode + meta[3 * g], meta[3 * g + 1]);
                const Vf<P> pred = acc.F[0];
                if (a.mode == MODE_POINTS) {
                    store_pts<P>(a.points_out + (uint64_t)(it.prog_begin + g) * a.points_stride + p0, pred, p0,
                                 ds.n_eval);
                } else {
                    Kahan k;
                    k.s = sacc[(g * 2) * 32 + lane];
                    k.c = sacc[(g * 2 + 1) * 32 + lane];
                    if (full) {
                        // the lane's P squared errors summed pairwise, then one
                        // compensated add per tile
                        float sq[P];
#pragma unroll
                        for (int q = 0; q < P; ++q) {
                            const float d = pred.v[q] - y.v[q];
                            sq[q] = d * d;
                        }
#pragma unroll
                        for (int h = P / 2; h > 0; h /= 2)
#pragma unroll
                            for (int q = 0; q < h; ++q) sq[q] = sq[q] + sq[q + h];
                        k.add(sq[0]);
                    } else {
#pragma unroll
                        for (int q = 0; q < P; ++q) {
                            if (p0 + q < ds.n_eval) {
                                const float d = pred.v[q] - y.v[q];
                                k.add(d * d);
                            }
                        }
                    }
                    sacc[(g * 2) * 32 + lane] = k.s;
                    sacc[(g * 2 + 1) * 32 + lane] = k.c;
                }
            }
        }
        if (a.mode == MODE_MSE) {
            for (uint32_t g = 0; g < G; ++g) {
                Kahan k;
                k.s = sacc[(g * 2) * 32 + lane];
                k.c = sacc[(g * 2 + 1) * 32 + lane];
                const double s = warp_sum(k.value());
                if (lane == 0) red[warp * kMaxProgsPerWarp + g] = s;
            }
            __syncthreads();
            if (threadIdx.x < G) {
                double s = 0.0;
                for (int w = 0; w < nw; ++w) s += red[w * kMaxProgsPerWarp + threadIdx.x];
                a.partials[a.progs[it.prog_begin + threadIdx.x].part_off + it.chunk] = s;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- launchers
// Shared-memory layout (floats).  Block header: code | constants | meta (32
// words) | cross-warp sums (kRegThreads/32 x 8 doubles).  Per warp: stacks
// (per type) | Kahan state.
void reg_layout(uint32_t code_words, uint32_t const_floats, const uint32_t *stack_depth, int P, int G,
                uint32_t *stack_off, uint32_t *acc_off, uint32_t *region_floats, uint32_t *block_hdr_floats) {
    *block_hdr_floats = align4r(code_words) + align4r(const_floats) + 32u + 2u * (kRegThreads / 32) * kMaxProgsPerWarp;
    uint32_t off = 0;
    for (int t = 0; t < N_STACKS; ++t) {
        stack_off[t] = off;
        off += stack_depth[t] * (uint32_t)kStackWidth[t] * 32u * (uint32_t)P;
    }
    *acc_off = off;
    off += 2u * 32u * (uint32_t)G;  // Kahan state of the item's programs
    *region_floats = align4r(off);
}

size_t reg_smem_bytes(uint32_t code_words, uint32_t const_floats, const uint32_t *stack_depth, int P, int G) {
    uint32_t so[N_STACKS], ao, rf, hf;
    reg_layout(code_words, const_floats, stack_depth, P, G, so, &ao, &rf, &hf);
    return ((size_t)hf + (size_t)rf * (kRegThreads / 32)) * 4u;
}

template <int PROF, int P, int OMIT>
static cudaError_t launch_reg_pp(const LaunchArgs &a, uint32_t grid, cudaStream_t st) {
    auto k = reg_eval_kernel<PROF, P, OMIT>;
    const size_t smem = ((size_t)a.block_hdr_floats + (size_t)a.region_floats * (kRegThreads / 32)) * 4u;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemOptin);
    if (e != cudaSuccess) return e;
    k<<<grid, kRegThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// Instantiated points-per-thread values: {2, 4, 8} for the F, F+V3 and
// F+V2+M2 profiles, {2, 4} for the others.
int reg_max_p(int profile) { return profile == P_F || profile == P_FV3 || profile == P_FV2M2 ? 8 : 4; }

// Handler sets a profile has kernels without (the OMIT mask of run_program).
unsigned reg_omittable(int profile) {
    return profile == P_FV3 ? 3u : profile == P_F || profile == P_FV2M2 ? 1u : 0u;
}

template <int PROF, int OMIT>
static cudaError_t launch_reg_p3(const LaunchArgs &a, int P, uint32_t grid, cudaStream_t st) {
    return P >= 8 ? launch_reg_pp<PROF, 8, OMIT>(a, grid, st)
         : P >= 4 ? launch_reg_pp<PROF, 4, OMIT>(a, grid, st) : launch_reg_pp<PROF, 2, OMIT>(a, grid, st);
}

cudaError_t launch_reg(const LaunchArgs &a, int profile, int P, unsigned omit, uint32_t grid, cudaStream_t st) {
    switch (profile) {
        case P_F: return omit & 1u ? launch_reg_p3<P_F, 1>(a, P, grid, st) : launch_reg_p3<P_F, 0>(a, P, grid, st);
        case P_FV3:
            switch (omit & 3u) {
                case 3: return launch_reg_p3<P_FV3, 3>(a, P, grid, st);
                case 2: return launch_reg_p3<P_FV3, 2>(a, P, grid, st);
                case 1: return launch_reg_p3<P_FV3, 1>(a, P, grid, st);
                default: return launch_reg_p3<P_FV3, 0>(a, P, grid, st);
            }
        case P_FV2M2: return omit & 1u ? launch_reg_p3<P_FV2M2, 1>(a, P, grid, st)
                                       : launch_reg_p3<P_FV2M2, 0>(a, P, grid, st);
        case P_FV3M3: return P >= 4 ? launch_reg_pp<P_FV3M3, 4, 0>(a, grid, st)
                                    : launch_reg_pp<P_FV3M3, 2, 0>(a, grid, st);
        default: return P >= 4 ? launch_reg_pp<P_ALL, 4, 0>(a, grid, st) : launch_reg_pp<P_ALL, 2, 0>(a, grid, st);
    }
}

template <int PROF, int P, int OMIT>
static int occ(size_t smem) {
    // the occupancy query counts a block above 48 KB of dynamic shared memory
    // as unlaunchable until the kernel's limit has been raised
    auto k = reg_eval_kernel<PROF, P, OMIT>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemOptin) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kRegThreads, smem) != cudaSuccess) return 0;
    return n;
}

template <int PROF, int OMIT>
static int occ3(int P, size_t smem) {
    return P >= 8 ? occ<PROF, 8, OMIT>(smem) : P >= 4 ? occ<PROF, 4, OMIT>(smem) : occ<PROF, 2, OMIT>(smem);
}

int reg_max_blocks_per_sm(int profile, int P, unsigned omit, size_t smem) {
    switch (profile) {
        case P_F: return omit & 1u ? occ3<P_F, 1>(P, smem) : occ3<P_F, 0>(P, smem);
        case P_FV3:
            switch (omit & 3u) {
                case 3: return occ3<P_FV3, 3>(P, smem);
                case 2: return occ3<P_FV3, 2>(P, smem);
                case 1: return occ3<P_FV3, 1>(P, smem);
                default: return occ3<P_FV3, 0>(P, smem);
            }
        case P_FV2M2: return omit & 1u ? occ3<P_FV2M2, 1>(P, smem) : occ3<P_FV2M2, 0>(P, smem);
        case P_FV3M3: return P >= 4 ? occ<P_FV3M3, 4, 0>(smem) : occ<P_FV3M3, 2, 0>(smem);
        default: return P >= 4 ? occ<P_ALL, 4, 0>(smem) : occ<P_ALL, 2, 0>(smem);
    }
}

}  // namespace rsr
