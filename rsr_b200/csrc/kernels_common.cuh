// kernels_common.cuh -- pieces shared by the evaluation kernels: launch
// arguments, per-tile data access, compensated accumulation and the warp
// reduction of partial sums.
#pragma once
#include <stdint.h>

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
};

// Opt-in dynamic shared-memory limit of one block on sm_100 (227 KB).  Every
// launcher raises its kernel's limit to this value rather than to the launch's
// own size: the limit is per-function state shared by all host threads, and a
// launch from one thread must not see it lowered by another thread.
constexpr int kMaxDynSmemOptin = 227 * 1024;

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

}  // namespace rsr
