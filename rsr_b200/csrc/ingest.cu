// ingest.cu -- dataset construction on the device.
//
// rsr_dataset_upload_rows restates Dataset::new (src/engine/data/dataset.rs:
// 37-169) from raw rows: optional z-score normalisation with the reference's
// f32 sequential sums (one thread per column, in row order, so every mean and
// deviation is bit-identical to the reference's), then the normalised values
// in the engine's resident column layout with the reference's zero padding.
// rsr_dataset_subset restates Dataset::subset (dataset.rs:360-447), the
// evenly spaced sample the engine's mini-batch and the API's large-dataset
// path take (src/engine/search/engine.rs:49, src/api.rs:115): point j of the
// subset is point round(j * step) of the source, step = (n - 1) / (m - 1) in
// f64, and zero where that index is past the source's samples.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include <algorithm>
#include <memory>
#include <mutex>

#include "runtime.h"

namespace rsr {
namespace {

// Column c < nf: feature c; column nf: the target.  Sequential f32 sums as
// Iterator::sum over f32 (dataset.rs:65-78, 82-90).
__global__ void norm_stats_kernel(const float *__restrict__ x_rows, const float *__restrict__ y, uint32_t nf,
                                  uint64_t n, float *mean_out, float *std_out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > nf) return;
    const float *col = c < nf ? x_rows + c : y;
    const uint64_t step = c < nf ? nf : 1;
    const float nsf = (float)n;
    float sum = 0.0f;
    for (uint64_t i = 0; i < n; ++i) sum += col[i * step];
    const float mean = sum / nsf;
    float sq = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
        const float d = col[i * step] - mean;
        sq += d * d;  // powi(2)
    }
    const float var = sq / nsf;
    mean_out[c] = mean;
    std_out[c] = var < 1e-9f ? 1.0f : sqrtf(var);
}

// (value - mean) / std into the columns; points past n keep the zero fill
// (get_norm_sample / get_norm_target, dataset.rs:109-125).
__global__ void rows_to_columns_kernel(const float *__restrict__ x_rows, const float *__restrict__ y, uint32_t nf,
                                       uint64_t n, const float *__restrict__ mean, const float *__restrict__ sd,
                                       bool normalize, float *x, float *yo, uint64_t stride) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        for (uint32_t f = 0; f < nf; ++f) {
            const float v = x_rows[i * nf + f];
            x[f * stride + i] = normalize ? (v - mean[f]) / sd[f] : v;
        }
        yo[i] = normalize ? (y[i] - mean[nf]) / sd[nf] : y[i];
    }
}

__global__ void subset_kernel(const float *__restrict__ sx, const float *__restrict__ sy, uint64_t sstride,
                              uint64_t n_src, uint32_t nf, double step, uint64_t m_eval, float *x, float *y,
                              uint64_t stride) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m_eval;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t o = (uint64_t)round((double)j * step);  // f64 product, rounded half away from zero
        const bool in = o < n_src;
        for (uint32_t f = 0; f < nf; ++f) x[f * stride + j] = in ? sx[f * sstride + o] : 0.0f;
        y[j] = in ? sy[o] : 0.0f;
    }
}

}  // namespace
}  // namespace rsr

using namespace rsr;

extern "C" {

int rsr_dataset_upload_rows(rsr_ctx *ctx, const float *x_rows, const float *y, uint32_t num_features,
                            uint64_t num_samples, int normalize, float *stats_out, rsr_dataset *out) {
    if (!ctx || !out || !y || (num_features && !x_rows)) return fail(RSR_EINVAL, "null argument");
    if (num_samples == 0) return fail(RSR_EINVAL, "no samples");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    const uint64_t nb = (num_samples + 7) / 8;
    std::unique_ptr<DatasetRec> rec;
    int rc = alloc_dataset(ctx, num_features, nb, num_samples, &rec);
    if (rc) return rc;
    const size_t xb = (size_t)num_samples * num_features * sizeof(float), yb = (size_t)num_samples * sizeof(float);
    const size_t sb = 2 * (size_t)(num_features + 1) * sizeof(float);
    void *tmp = nullptr;
    cudaError_t e = cudaMalloc(&tmp, xb + yb + sb);
    auto cleanup = [&] {
        if (tmp) cudaFree(tmp);
        cudaFree(rec->x);
        cudaFree(rec->y);
    };
    if (e != cudaSuccess) {
        tmp = nullptr;
        cleanup();
        return cuda_fail(e, "row staging");
    }
    float *dx = (float *)tmp, *dy = (float *)((char *)tmp + xb), *dmean = (float *)((char *)tmp + xb + yb);
    float *dsd = dmean + num_features + 1;
    cudaStream_t st = ctx->stream;
    if (xb) cudaMemcpyAsync(dx, x_rows, xb, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dy, y, yb, cudaMemcpyHostToDevice, st);
    if (normalize) {
        norm_stats_kernel<<<(num_features + 1 + 63) / 64, 64, 0, st>>>(dx, dy, num_features, num_samples, dmean, dsd);
        ctx->launches++;
    }
    rows_to_columns_kernel<<<ctx->num_sms * 4, 256, 0, st>>>(dx, dy, num_features, num_samples, dmean, dsd,
                                                             normalize != 0, rec->x, rec->y, rec->stride);
    ctx->launches++;
    if (normalize && stats_out)
        cudaMemcpyAsync(stats_out, dmean, sb, cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFree(tmp);
    tmp = nullptr;
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "row upload");
    }
    if (!normalize && stats_out)
        for (uint32_t c = 0; c <= num_features; ++c) {
            stats_out[c] = 0.0f;
            stats_out[num_features + 1 + c] = 1.0f;
        }
    *out = register_dataset(ctx, std::move(rec));
    return RSR_OK;
}

int rsr_dataset_subset(rsr_ctx *ctx, rsr_dataset src, uint64_t target_samples, rsr_dataset *out) {
    if (!ctx || !out) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->datasets.find(src);
    if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle");
    const DatasetRec &s = *it->second;
    const uint64_t m = std::min<uint64_t>(target_samples, s.num_samples);
    if (m == 0) return fail(RSR_EINVAL, "empty subset");
    cudaSetDevice(ctx->device);
    const uint64_t nb = (m + 7) / 8;
    std::unique_ptr<DatasetRec> rec;
    int rc = alloc_dataset(ctx, s.num_features, nb, m, &rec);
    if (rc) return rc;
    // the whole dataset when m == num_samples (dataset.rs:362-365): step 1
    const double step = m == s.num_samples ? 1.0 : ((double)s.num_samples - 1.0) / std::max((double)m - 1.0, 1.0);
    const uint64_t n_src = m == s.num_samples ? s.num_batches * 8 : s.num_samples;
    subset_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(s.x, s.y, s.stride, n_src, s.num_features, step,
                                                              nb * 8, rec->x, rec->y, rec->stride);
    ctx->launches++;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(rec->x);
        cudaFree(rec->y);
        return cuda_fail(e, "subset");
    }
    *out = register_dataset(ctx, std::move(rec));
    return RSR_OK;
}

int rsr_dataset_download(rsr_ctx *ctx, rsr_dataset ds, float *feature_flat, float *target_batches) {
    if (!ctx || !target_batches) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->datasets.find(ds);
    if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle");
    const DatasetRec &s = *it->second;
    if (s.num_features && !feature_flat) return fail(RSR_EINVAL, "null argument");
    cudaSetDevice(ctx->device);
    const uint64_t n = s.num_batches * 8;
    std::vector<float> col(n);
    cudaError_t e;
    for (uint32_t f = 0; f < s.num_features; ++f) {
        if ((e = cudaMemcpy(col.data(), s.x + (size_t)f * s.stride, n * sizeof(float), cudaMemcpyDeviceToHost)))
            return cuda_fail(e, "dataset download");
        for (uint64_t i = 0; i < n; ++i) feature_flat[((i >> 3) * s.num_features + f) * 8 + (i & 7)] = col[i];
    }
    if ((e = cudaMemcpy(target_batches, s.y, n * sizeof(float), cudaMemcpyDeviceToHost)))
        return cuda_fail(e, "dataset download");
    return RSR_OK;
}

}  // extern "C"
