// kernels_common.cuh -- pieces shared by the evaluation kernels: launch
// arguments, per-tile data access, compensated accumulation and the warp
// reduction of partial sums.
#pragma once
#include <stdint.h>

#include <atomic>

#include <cuda_runtime.h>

#include "uops.h"
#include "vm_ops.cuh"

namespace rsr {

enum EvalMode : int { MODE_MSE = 0, MODE_POINTS = 1 };

struct LaunchArgs {
    const ProgDesc *progs;
    const DatasetDesc *datasets;
    const WorkItem *items;
    const uint32_t *code;     // code pool
    const float *consts;      // constant pool
    double *partials;         // per (program, chunk) sums; gradient: (1+32) per slot
    float *points_out;        // MODE_POINTS: predictions
    uint64_t points_stride;   // MODE_POINTS: floats between consecutive programs
    uint32_t *item_counter;   // persistent kernels: next work item
    uint32_t *status;         // sticky error flags (bit 0: bad micro-op)
    const uint8_t *active;    // optional per-program mask (launch order): 0 = skip
    const uint32_t *run_if;   // optional: the launch does nothing when *run_if == 0 (device-side
                              // loops whose later rounds may have no work, e.g. line searches)
    uint32_t n_items;
    uint32_t mode;
    uint32_t smem_code_words; // per warp
    uint32_t smem_const_floats;
    uint32_t smem_slots;      // per warp (slot-file kernels; adjoint: value slots)
    uint32_t smem_adj_slots;  // per warp (adjoint: adjoint slots)
    uint32_t progs_per_warp;
    // register kernel: per-warp shared-memory layout (floats)
    uint32_t region_floats;   // per warp
    uint32_t block_hdr_floats;
    uint32_t acc_off;
    uint32_t stack_off[N_STACKS];
    uint32_t tmem_cols;       // register adjoint: tensor-memory columns of a block's tapes
};

// Opt-in dynamic shared-memory limit of one block on sm_100 (227 KB).  Every
// launcher raises its kernel's limit to this value rather than to the launch's
// own size: the limit is per-function state shared by all host threads, and a
// launch from one thread must not see it lowered by another thread.
constexpr int kMaxDynSmemOptin = 227 * 1024;

// Raises kernel k's dynamic shared-memory limit to kMaxDynSmemOptin once per
// device: `done` (a static of the caller's instance) holds one bit per
// device on which it is set, so later launches skip the driver call.
template <typename K>
__host__ inline cudaError_t raise_smem_limit(K k, std::atomic<uint64_t> &done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemOptin);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
    return e;
}

// Kahan-compensated single-precision running sum (one per lane).
struct Kahan {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float v) {
        const float y = v - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Loads P consecutive floats starting at a P-aligned index.
template <int P>
__device__ __forceinline__ Vf<P> load_pts(const float *__restrict__ p) {
    Vf<P> r;
    if constexpr (P == 1) {
        r.v[0] = __ldg(p);
    } else if constexpr (P == 2) {
        float2 a = __ldg(reinterpret_cast<const float2 *>(p));
        r.v[0] = a.x; r.v[1] = a.y;
    } else {
#pragma unroll
        for (int j = 0; j < P / 4; ++j) {
            float4 a = __ldg(reinterpret_cast<const float4 *>(p) + j);
            r.v[4 * j] = a.x; r.v[4 * j + 1] = a.y; r.v[4 * j + 2] = a.z; r.v[4 * j + 3] = a.w;
        }
    }
    return r;
}

template <int P>
__device__ __forceinline__ void store_pts(float *p, const Vf<P> &v, uint64_t first, uint64_t limit) {
#pragma unroll
    for (int k = 0; k < P; ++k)
        if (first + k < limit) p[k] = v.v[k];
}

// ------------------------------------------------ interleaved lane layout
// The register kernels give lane l of a warp the points of a 32*P-point
// tile in runs of at most four: P <= 4, points l*P .. l*P+P-1; P = 8, points
// 4l .. 4l+3 and 128+4l .. 128+4l+3.  Each 16-byte access of the warp then
// covers 512 contiguous bytes -- four L1 wavefronts for a global load, no
// bank conflict for shared memory -- where eight consecutive points a lane
// would take eight (two lanes 32 bytes apart share a 128-byte line or a bank).
// Per-lane values in shared memory use the same layout in blocks of 32*P
// floats: [P/4 runs][32 lanes][4] (P >= 4), [32 lanes][P] below.
template <int P>
constexpr int kLaneRun = P < 4 ? P : 4;

// Offset of value q of `lane` from the start of its tile (or block).
template <int P>
__host__ __device__ __forceinline__ constexpr uint32_t lane_point(int lane, int q) {
    return (uint32_t)((q / kLaneRun<P>) * 32 * kLaneRun<P> + lane * kLaneRun<P> + q % kLaneRun<P>);
}

// Loads a lane's P values; p points at its first (tile start + lane_point(lane, 0)).
template <int P>
__device__ __forceinline__ Vf<P> load_lane(const float *__restrict__ p) {
    if constexpr (P <= 4) {
        return load_pts<P>(p);
    } else {
        Vf<P> r;
#pragma unroll
        for (int j = 0; j < P / 4; ++j) {
            const float4 a = __ldg(reinterpret_cast<const float4 *>(p + j * 128));
            r.v[4 * j] = a.x; r.v[4 * j + 1] = a.y; r.v[4 * j + 2] = a.z; r.v[4 * j + 3] = a.w;
        }
        return r;
    }
}

// Shared-memory image of a lane's P values in a block of 32*P floats; p
// points at the lane's first value (block start + lane_point(lane, 0)).
template <int P>
__device__ __forceinline__ Vf<P> lds_lane(const float *p) {
    if constexpr (P <= 4) {
        return *reinterpret_cast<const Vf<P> *>(p);
    } else {
        Vf<P> r;
#pragma unroll
        for (int j = 0; j < P / 4; ++j) {
            const float4 a = *reinterpret_cast<const float4 *>(p + j * 128);
            r.v[4 * j] = a.x; r.v[4 * j + 1] = a.y; r.v[4 * j + 2] = a.z; r.v[4 * j + 3] = a.w;
        }
        return r;
    }
}

template <int P>
__device__ __forceinline__ void sts_lane(float *p, const Vf<P> &v) {
    if constexpr (P <= 4) {
        *reinterpret_cast<Vf<P> *>(p) = v;
    } else {
#pragma unroll
        for (int j = 0; j < P / 4; ++j)
            *reinterpret_cast<float4 *>(p + j * 128) = make_float4(v.v[4 * j], v.v[4 * j + 1], v.v[4 * j + 2],
                                                                  v.v[4 * j + 3]);
    }
}

// Stores the lane's values whose points lie below `limit`; `tile` is the
// tile's first point, p the output's value of point `tile`.
template <int P>
__device__ __forceinline__ void store_lane(float *p, int lane, const Vf<P> &v, uint64_t tile, uint64_t limit) {
#pragma unroll
    for (int q = 0; q < P; ++q) {
        const uint32_t o = lane_point<P>(lane, q);
        if (tile + o < limit) p[o] = v.v[q];
    }
}

}  // namespace rsr
