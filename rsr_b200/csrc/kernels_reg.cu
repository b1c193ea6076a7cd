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

#include "acc_ops.cuh"
#include "kernels.h"
#include "kernels_common.cuh"

namespace rsr {

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
    for (int t = 0; t < N_STACKS; ++t) io.stk[t] = wbase + a.stack_off[t] + lane_point<P>(lane, 0);

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
            const uint64_t t0 = (uint64_t)tile * (32u * P);
            const uint64_t p0 = t0 + lane_point<P>(lane, 0);
            io.xl = ds.x + p0;
            const Vf<P> y = load_lane<P>(ds.y + p0);
            const bool full = t0 + lane_point<P>(lane, P - 1) < ds.n_eval;  // the lane's last value
            for (uint32_t g = 0; g < G; ++g) {
                if (a.active && !a.active[it.prog_begin + g]) continue;
                io.consts = sconst + meta[3 * g + 2];
                run_program<PROF, P, OMIT>(acc, io, scode + meta[3 * g], meta[3 * g + 1]);
                const Vf<P> pred = acc.F[0];
                if (a.mode == MODE_POINTS) {
                    store_lane<P>(a.points_out + (uint64_t)(it.prog_begin + g) * a.points_stride + t0, lane, pred,
                                  t0, ds.n_eval);
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
                            if (t0 + lane_point<P>(lane, q) < ds.n_eval) {
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
    static std::atomic<uint64_t> limit_raised{0};
    cudaError_t e = raise_smem_limit(k, limit_raised);
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

// Loads one instance ahead of its first real launch: an empty launch (run_if
// points at a zero word, so every thread returns at its first check) also
// sizes the context's local memory for the instance's spills.
template <int PROF, int P, int OMIT>
static cudaError_t preload_pp(const uint32_t *zero, cudaStream_t st) {
    auto k = reg_eval_kernel<PROF, P, OMIT>;
    static std::atomic<uint64_t> limit_raised{0};
    cudaError_t e = raise_smem_limit(k, limit_raised);
    if (e != cudaSuccess) return e;
    LaunchArgs none{};
    none.run_if = zero;
    k<<<1, kRegThreads, 0, st>>>(none);
    return cudaGetLastError();
}

template <int PROF, int OMIT>
static cudaError_t preload_p3(const uint32_t *zero, cudaStream_t st) {
    cudaError_t e;
    if ((e = preload_pp<PROF, 2, OMIT>(zero, st)) != cudaSuccess) return e;
    if ((e = preload_pp<PROF, 4, OMIT>(zero, st)) != cudaSuccess) return e;
    return preload_pp<PROF, 8, OMIT>(zero, st);
}

cudaError_t preload_reg(const uint32_t *zero, cudaStream_t st) {
    const cudaError_t r[] = {
        preload_p3<P_F, 0>(zero, st),     preload_p3<P_F, 1>(zero, st),
        preload_p3<P_FV3, 0>(zero, st),   preload_p3<P_FV3, 1>(zero, st),
        preload_p3<P_FV3, 2>(zero, st),   preload_p3<P_FV3, 3>(zero, st),
        preload_p3<P_FV2M2, 0>(zero, st), preload_p3<P_FV2M2, 1>(zero, st),
        preload_pp<P_FV3M3, 2, 0>(zero, st), preload_pp<P_FV3M3, 4, 0>(zero, st),
        preload_pp<P_ALL, 2, 0>(zero, st),   preload_pp<P_ALL, 4, 0>(zero, st)};
    for (cudaError_t e : r)
        if (e != cudaSuccess) return e;
    return cudaSuccess;
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
