// kernels_plain.cu -- the slot-file interpreter ("plain" kernel) and the
// dataset / finalize kernels.
//
// One program per warp; its slot-form bytecode and constants are staged in
// shared memory, so dispatch is warp-uniform.  Lanes cover data points, P
// consecutive points per lane read with vector loads from the SoA dataset.
// The stack slots of the reference VM (state.rs:12-37) live in shared memory,
// one P-wide value per (slot, lane), and keep the reference's positions, so
// this kernel reproduces eval_simd (evaluator.rs:20-150) for any valid
// program, stale slots and stack_f[0] included.
#include <cuda_runtime.h>
#include <float.h>

#include "kernels_common.cuh"
#include "kernels.h"

namespace rsr {

template <int P>
struct SlotCtx {
    Vf<P> *slots;        // [slot][lane]
    const float *consts; // staged constants
    const float *x;      // dataset features (SoA)
    uint64_t stride;
    uint64_t p0;         // first point of this lane
    int lane;
    __device__ __forceinline__ Vf<P> L(uint32_t s) const { return slots[s * 32 + lane]; }
    __device__ __forceinline__ void S(uint32_t s, const Vf<P> &v) const { slots[s * 32 + lane] = v; }
    __device__ __forceinline__ void Ln(Vf<P> *d, uint32_t s, int n) const {
        for (int i = 0; i < n; ++i) d[i] = L(s + i);
    }
    __device__ __forceinline__ void Sn(uint32_t s, const Vf<P> *v, int n) const {
        for (int i = 0; i < n; ++i) S(s + i, v[i]);
    }
    __device__ __forceinline__ Vf<P> X(uint32_t f) const { return load_pts<P>(x + f * stride + p0); }
};

// One reference instruction in slot form (w0, w1, w2: uops.h).
template <int P>
__device__ __forceinline__ void exec_slot(const SlotCtx<P> &c, uint32_t w0, uint32_t w1, uint32_t w2) {
    const uint32_t op = w0 & 0xFFu, aux = w0 >> 8;
    const uint32_t o = w1 & 0xFFFFu, i0 = w1 >> 16, i1 = w2 & 0xFFFFu, i2 = w2 >> 16;
    Vf<P> A[9], B[9], R[9];
    switch (op) {
        // loads (evaluator.rs:26-142)
        case LOAD_VAR_F: c.S(o, c.X(aux)); break;
        case LOAD_VAR_V2: for (int i = 0; i < 2; ++i) c.S(o + i, c.X(aux + i)); break;
        case LOAD_VAR_V3: for (int i = 0; i < 3; ++i) c.S(o + i, c.X(aux + i)); break;
        case LOAD_VAR_M2: for (int i = 0; i < 4; ++i) c.S(o + i, c.X(aux + i)); break;
        case LOAD_VAR_M3: for (int i = 0; i < 9; ++i) c.S(o + i, c.X(aux + i)); break;
        case LOAD_CONST_F: c.S(o, splat<P>(c.consts[aux])); break;
        case LOAD_CONST_V2: for (int i = 0; i < 2; ++i) c.S(o + i, splat<P>(c.consts[aux + i])); break;
        case LOAD_CONST_V3: for (int i = 0; i < 3; ++i) c.S(o + i, splat<P>(c.consts[aux + i])); break;
        case LOAD_CONST_M2: for (int i = 0; i < 4; ++i) c.S(o + i, splat<P>(c.consts[aux + i])); break;
        case LOAD_CONST_M3: for (int i = 0; i < 9; ++i) c.S(o + i, splat<P>(c.consts[aux + i])); break;
        case SLOT_NOP: break;
        // basic (basic/eval.rs:4-63)
        case ADD_F: c.S(o, c.L(i0) + c.L(i1)); break;
        case SUB_F: c.S(o, c.L(i0) - c.L(i1)); break;
        case MUL_F: c.S(o, c.L(i0) * c.L(i1)); break;
        case DIV_F: c.S(o, c.L(i0) / c.L(i1)); break;
        case SIN_F: c.S(o, vsin(c.L(i0))); break;
        case COS_F: c.S(o, vcos(c.L(i0))); break;
        case EXP_F: c.S(o, vexp(c.L(i0))); break;
        case SQR_F: { Vf<P> a = c.L(i0); c.S(o, a * a); break; }
        case SQRT_F: c.S(o, vsqrt(c.L(i0))); break;
        case LN_F: c.S(o, vlog(c.L(i0))); break;
        // linalg (linalg/eval.rs)
        case MAKE_VEC2: A[0] = c.L(i0); A[1] = c.L(i1); c.Sn(o, A, 2); break;
        case MAKE_VEC3: A[0] = c.L(i0); A[1] = c.L(i1); A[2] = c.L(i2); c.Sn(o, A, 3); break;
        case GET_X_V2: case GET_X_V3: c.S(o, c.L(i0)); break;
        case GET_Y_V2: case GET_Y_V3: c.S(o, c.L(i0 + 1)); break;
        case GET_Z_V3: c.S(o, c.L(i0 + 2)); break;
        case ADD_V2: c.Ln(A, i0, 2); c.Ln(B, i1, 2); for (int i = 0; i < 2; ++i) R[i] = A[i] + B[i]; c.Sn(o, R, 2); break;
        case SUB_V2: c.Ln(A, i0, 2); c.Ln(B, i1, 2); for (int i = 0; i < 2; ++i) R[i] = A[i] - B[i]; c.Sn(o, R, 2); break;
        case SCALE_V2: { Vf<P> s = c.L(i0); c.Ln(A, i1, 2); for (int i = 0; i < 2; ++i) R[i] = A[i] * s; c.Sn(o, R, 2); break; }
        case DOT_V2: c.Ln(A, i0, 2); c.Ln(B, i1, 2); c.S(o, dot2(A, B)); break;
        case NORM_V2: c.Ln(A, i0, 2); c.S(o, norm2(A)); break;
        case ADD_V3: c.Ln(A, i0, 3); c.Ln(B, i1, 3); for (int i = 0; i < 3; ++i) R[i] = A[i] + B[i]; c.Sn(o, R, 3); break;
        case SUB_V3: c.Ln(A, i0, 3); c.Ln(B, i1, 3); for (int i = 0; i < 3; ++i) R[i] = A[i] - B[i]; c.Sn(o, R, 3); break;
        case SCALE_V3: { Vf<P> s = c.L(i0); c.Ln(A, i1, 3); for (int i = 0; i < 3; ++i) R[i] = A[i] * s; c.Sn(o, R, 3); break; }
        case DOT_V3: c.Ln(A, i0, 3); c.Ln(B, i1, 3); c.S(o, dot3(A, B)); break;
        case NORM_V3: c.Ln(A, i0, 3); c.S(o, norm3(A)); break;
        case CROSS_V3: c.Ln(A, i0, 3); c.Ln(B, i1, 3); cross3(A, B, R); c.Sn(o, R, 3); break;
        case MAKE_MAT2: c.Ln(A, i0, 2); c.Ln(A + 2, i1, 2); c.Sn(o, A, 4); break;
        case ADD_M2: c.Ln(A, i0, 4); c.Ln(B, i1, 4); for (int i = 0; i < 4; ++i) R[i] = A[i] + B[i]; c.Sn(o, R, 4); break;
        case SUB_M2: c.Ln(A, i0, 4); c.Ln(B, i1, 4); for (int i = 0; i < 4; ++i) R[i] = A[i] - B[i]; c.Sn(o, R, 4); break;
        case SCALE_M2: { Vf<P> s = c.L(i0); c.Ln(A, i1, 4); for (int i = 0; i < 4; ++i) R[i] = A[i] * s; c.Sn(o, R, 4); break; }
        case MUL_M2: c.Ln(A, i0, 4); c.Ln(B, i1, 4); mul_m2(A, B, R); c.Sn(o, R, 4); break;
        case MUL_M2V2: c.Ln(A, i0, 4); c.Ln(B, i1, 2); mul_m2v2(A, B, R); c.Sn(o, R, 2); break;
        case DET_M2: c.Ln(A, i0, 4); c.S(o, det_m2(A)); break;
        case TRACE_M2: c.Ln(A, i0, 4); c.S(o, trace_m2(A)); break;
        case TRANSPOSE_M2: c.Ln(A, i0, 4); transpose_m2(A, R); c.Sn(o, R, 4); break;
        case INVERSE_M2: c.Ln(A, i0, 4); inverse_m2(A, R); c.Sn(o, R, 4); break;
        case MAKE_MAT3: c.Ln(A, i0, 3); c.Ln(A + 3, i1, 3); c.Ln(A + 6, i2, 3); c.Sn(o, A, 9); break;
        case ADD_M3: c.Ln(A, i0, 9); c.Ln(B, i1, 9); for (int i = 0; i < 9; ++i) R[i] = A[i] + B[i]; c.Sn(o, R, 9); break;
        case SUB_M3: c.Ln(A, i0, 9); c.Ln(B, i1, 9); for (int i = 0; i < 9; ++i) R[i] = A[i] - B[i]; c.Sn(o, R, 9); break;
        case SCALE_M3: { Vf<P> s = c.L(i0); c.Ln(A, i1, 9); for (int i = 0; i < 9; ++i) R[i] = A[i] * s; c.Sn(o, R, 9); break; }
        case MUL_M3: c.Ln(A, i0, 9); c.Ln(B, i1, 9); mul_m3(A, B, R); c.Sn(o, R, 9); break;
        case MUL_M3V3: c.Ln(A, i0, 9); c.Ln(B, i1, 3); mul_m3v3(A, B, R); c.Sn(o, R, 3); break;
        case DET_M3: c.Ln(A, i0, 9); c.S(o, det_m3(A)); break;
        case TRACE_M3: c.Ln(A, i0, 9); c.S(o, trace_m3(A)); break;
        case TRANSPOSE_M3: c.Ln(A, i0, 9); transpose_m3(A, R); c.Sn(o, R, 9); break;
        case INVERSE_M3: c.Ln(A, i0, 9); inverse_m3(A, R); c.Sn(o, R, 9); break;
        default: break;
    }
}

__host__ __device__ __forceinline__ uint32_t align4u(uint32_t v) { return (v + 3u) & ~3u; }

// Stage a program's code and constants into this warp's shared region.
__device__ __forceinline__ void stage_program(uint32_t *scode, float *sconst, const LaunchArgs &a, const ProgDesc &pd,
                                              int lane) {
    for (uint32_t i = lane; i < pd.uop_len; i += 32) scode[i] = __ldg(a.code + pd.uop_off + i);
    for (uint32_t i = lane; i < pd.n_consts; i += 32) sconst[i] = __ldg(a.consts + pd.const_off + i);
    __syncwarp();
}

template <int P>
__global__ void __launch_bounds__(kPlainThreads) plain_eval_kernel(const LaunchArgs a) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t item_id = blockIdx.x * (blockDim.x >> 5) + warp;
    if (item_id >= a.n_items) return;
    if (a.run_if && *a.run_if == 0u) return;
    const uint32_t region = align4u(a.smem_code_words) + align4u(a.smem_const_floats) + a.smem_slots * 32u * P;
    float *base = smem + (size_t)warp * region;
    uint32_t *scode = reinterpret_cast<uint32_t *>(base);
    float *sconst = base + align4u(a.smem_code_words);
    Vf<P> *sslot = reinterpret_cast<Vf<P> *>(sconst + align4u(a.smem_const_floats));
    const WorkItem it = a.items[item_id];
    for (uint32_t g = 0; g < it.n_progs; ++g) {
        const uint32_t pid = it.prog_begin + g;
        if (a.active && !a.active[pid]) continue;
        const ProgDesc pd = a.progs[pid];
        const DatasetDesc ds = a.datasets[pd.dataset];
        stage_program(scode, sconst, a, pd, lane);
        SlotCtx<P> c{sslot, sconst, ds.x, ds.stride, 0, lane};
        Kahan acc;
        for (uint32_t tile = it.tile_begin; tile < it.tile_end; ++tile) {
            c.p0 = (uint64_t)tile * (32u * P) + (uint64_t)lane * P;
            if (pd.flags & PF_NEEDS_ZERO_INIT)
                for (uint32_t s = 0; s < pd.n_slots; ++s) c.S(s, splat<P>(0.0f));
            for (uint32_t pc = 0; pc < pd.uop_len; pc += 3) exec_slot<P>(c, scode[pc], scode[pc + 1], scode[pc + 2]);
            const Vf<P> pred = (pd.flags & PF_RESULT_ZERO) ? splat<P>(0.0f) : c.L(0);
            if (a.mode == MODE_POINTS) {
                store_pts<P>(a.points_out + (uint64_t)pid * a.points_stride + c.p0, pred, c.p0, ds.n_eval);
            } else {
                const Vf<P> y = load_pts<P>(ds.y + c.p0);
#pragma unroll
                for (int k = 0; k < P; ++k) {
                    if (c.p0 + k < ds.n_eval) {
                        const float d = pred.v[k] - y.v[k];
                        acc.add(d * d);
                    }
                }
            }
        }
        if (a.mode == MODE_MSE) {
            const double s = warp_sum(acc.value());
            if (lane == 0) a.partials[pd.part_off + it.chunk] = s;
        }
        __syncwarp();
    }
}

// AoSoA f32x8 batches (dataset.rs:96-154) -> SoA columns x[f*stride + i].
__global__ void aosoa_to_soa_kernel(const float *__restrict__ ff, const float *__restrict__ tb, float *x, float *y,
                                    uint32_t nf, uint64_t nbatch, uint64_t stride) {
    const uint64_t n = nbatch * 8;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i >> 3, l = i & 7;
        for (uint32_t f = 0; f < nf; ++f) x[f * stride + i] = ff[(b * nf + f) * 8 + l];
        y[i] = tb[i];
    }
}

// Per-program reduction of the partial sums in a fixed order, then the
// compute_mse epilogue (evaluator.rs:172-173): divide by num_samples and map
// non-finite results to f32::MAX.  A total above f32::MAX is mapped there
// too, as the reference's f32 accumulator would have overflowed.
__global__ void finalize_mse_kernel(const ProgDesc *progs, const DatasetDesc *datasets, const double *partials,
                                    uint32_t n_progs, float *mse_out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_progs) return;
    const ProgDesc pd = progs[p];
    double s = 0.0;
    for (uint32_t c = 0; c < pd.n_parts; ++c) s += partials[pd.part_off + c];
    const double n = (double)datasets[pd.dataset].num_samples;
    float m = (float)(s / n);
    if (!(s <= (double)FLT_MAX) || !isfinite(m)) m = FLT_MAX;
    mse_out[p] = m;
}

// ------------------------------------------------------------- launchers
template <int P>
static cudaError_t launch_plain_p(const LaunchArgs &a, uint32_t warps_per_block, size_t smem, cudaStream_t st) {
    auto k = plain_eval_kernel<P>;
    static std::atomic<uint64_t> limit_raised{0};
    cudaError_t e = raise_smem_limit(k, limit_raised);
    if (e != cudaSuccess) return e;
    const uint32_t blocks = (a.n_items + warps_per_block - 1) / warps_per_block;
    k<<<blocks, warps_per_block * 32, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_plain(const LaunchArgs &a, int P, uint32_t warps_per_block, size_t smem, cudaStream_t st) {
    switch (P) {
        case 1: return launch_plain_p<1>(a, warps_per_block, smem, st);
        case 2: return launch_plain_p<2>(a, warps_per_block, smem, st);
        default: return launch_plain_p<4>(a, warps_per_block, smem, st);
    }
}

size_t plain_smem_per_warp(uint32_t code_words, uint32_t const_floats, uint32_t slots, int P) {
    return ((size_t)align4u(code_words) + align4u(const_floats) + (size_t)slots * 32u * P) * 4u;
}

// With lazy module loading (the default since CUDA 12.2) a kernel's code is
// loaded, and device memory taken for it and for its local memory, on its
// first launch.  This loads every point-count variant of the slot-file
// kernel and the MSE epilogue ahead of time: each is looked up
// (cudaFuncGetAttributes) and launched once with no work (no items, no
// programs), which returns at once.
cudaError_t preload_plain_mse(cudaStream_t st) {
    cudaFuncAttributes fa;
    cudaError_t e;
    if ((e = cudaFuncGetAttributes(&fa, plain_eval_kernel<1>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, plain_eval_kernel<2>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, plain_eval_kernel<4>)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, finalize_mse_kernel)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(plain_eval_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxDynSmemOptin)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(plain_eval_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxDynSmemOptin)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(plain_eval_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kMaxDynSmemOptin)) != cudaSuccess)
        return e;
    LaunchArgs none{};  // n_items = 0: every warp returns before reading anything
    plain_eval_kernel<1><<<1, 32, 0, st>>>(none);
    plain_eval_kernel<2><<<1, 32, 0, st>>>(none);
    plain_eval_kernel<4><<<1, 32, 0, st>>>(none);
    finalize_mse_kernel<<<1, 32, 0, st>>>(nullptr, nullptr, nullptr, 0u, nullptr);  // n_progs = 0
    return cudaGetLastError();
}

cudaError_t launch_aosoa_to_soa(const float *ff, const float *tb, float *x, float *y, uint32_t nf, uint64_t nbatch,
                                uint64_t stride, int num_sms, cudaStream_t st) {
    const uint64_t n = nbatch * 8;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)num_sms * 16) blocks = (uint64_t)num_sms * 16;
    if (blocks == 0) blocks = 1;
    aosoa_to_soa_kernel<<<(unsigned)blocks, 256, 0, st>>>(ff, tb, x, y, nf, nbatch, stride);
    return cudaGetLastError();
}

// Per-program sums of the partials in the same fixed order, left unscaled
// (stride 1: SSE; stride 33: SSE then the 32 gradient sums), for callers that
// add the sums of several point shards before the epilogue.
__global__ void finalize_sums_kernel(const ProgDesc *progs, const double *partials, uint32_t n_progs,
                                     uint32_t stride, double *out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_progs) return;
    const ProgDesc pd = progs[p];
    for (uint32_t j = 0; j < stride; ++j) {
        double s = 0.0;
        for (uint32_t c = 0; c < pd.n_parts; ++c) s += partials[(size_t)(pd.part_off + c) * stride + j];
        out[(size_t)p * stride + j] = s;
    }
}

cudaError_t launch_finalize_sums(const ProgDesc *progs, const double *partials, uint32_t n, uint32_t stride,
                                 double *out, cudaStream_t st) {
    finalize_sums_kernel<<<(n + 127) / 128, 128, 0, st>>>(progs, partials, n, stride, out);
    return cudaGetLastError();
}

cudaError_t launch_finalize_mse(const ProgDesc *progs, const DatasetDesc *ds, const double *partials, uint32_t n,
                                float *out, cudaStream_t st) {
    finalize_mse_kernel<<<(n + 127) / 128, 128, 0, st>>>(progs, ds, partials, n, out);
    return cudaGetLastError();
}

}  // namespace rsr

namespace rsr {

// FP32 lane-op throughput probe: 8 independent chains of unfused multiply
// and add per thread (the operation mix of the interpreter's arithmetic).
__global__ void fp32_peak_kernel(float *out, int iters, float a, float b) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (float)(threadIdx.x + i) * 1e-3f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = v[i] * a + b;
    }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += v[i];
    if (s == 12345.0f) out[threadIdx.x] = s;  // keeps the chains live
}

cudaError_t measure_fp32_peak(int num_sms, cudaStream_t st, double *lane_ops_per_s) {
    float *out = nullptr;
    cudaError_t e = cudaMalloc(&out, 1024 * sizeof(float));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int iters = 1 << 14, threads = 512, blocks = num_sms * 4;
    fp32_peak_kernel<<<blocks, threads, 0, st>>>(out, 256, 0.999f, 1e-4f);  // warm-up
    cudaEventRecord(e0, st);
    fp32_peak_kernel<<<blocks, threads, 0, st>>>(out, iters, 0.999f, 1e-4f);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    *lane_ops_per_s = (double)blocks * threads * iters * 8 * 2 / (ms * 1e-3);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace rsr
