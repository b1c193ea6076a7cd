// fit_eval.h -- batched evaluation for the constant-fitting drivers.
//
// A fit keeps one plan resident and, between launches, rewrites only the
// constant pool (each program's parameters) and a per-program active mask:
// programs that have finished their fit are skipped by the kernels.
#pragma once
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "runtime.h"

namespace rsr {
namespace fit {

struct Evaluator {
    Plan plan;
    DevicePlan *dev = nullptr;  // device buffers, owned by a FitWorkspace
    DevBuf *active = nullptr;
    std::vector<uint8_t> mask;  // launch order
    std::vector<float> host_out;
};

inline int prepare(rsr_ctx *ctx, const rsr_population &pop, const uint64_t *dsp, uint64_t ds, bool gradient,
                   cudaStream_t st, std::mutex *plan_mu, Evaluator *ev) {
    int rc;
    if (plan_mu) {
        std::lock_guard<std::mutex> lk(*plan_mu);
        rc = build_plan(ctx, pop, dsp, ds, RSR_KERNEL_AUTO, gradient, MODE_MSE, &ev->plan);
    } else {
        rc = build_plan(ctx, pop, dsp, ds, RSR_KERNEL_AUTO, gradient, MODE_MSE, &ev->plan);
    }
    if (rc) return rc;
    if ((rc = upload_plan(ctx, ev->plan, ev->dev, st))) return rc;
    const size_t n = ev->plan.progs.size();
    cudaError_t e = ev->active->reserve(std::max<size_t>(n, 1));
    if (e != cudaSuccess) return cuda_fail(e, "active mask");
    ev->dev->base.active = (const uint8_t *)ev->active->p;
    ev->mask.assign(n, 1);
    return RSR_OK;
}

// set(i, params) writes caller-order program i's flat parameters into its
// slice of the constant pool; then every wanted program is evaluated and
// mse (and grad, n x 32) are returned in caller order.
template <class Set>
int evaluate(rsr_ctx *ctx, cudaStream_t stream, Evaluator *ev, const std::vector<char> &want, Set set,
             std::vector<float> *mse, std::vector<float> *grad) {
    Plan &P = ev->plan;
    const size_t n = P.progs.size();
    for (size_t li = 0; li < n; ++li) {
        const uint32_t i = P.orig[li];
        if (want[i]) set(i, P.consts.data() + P.progs[li].const_off);
        ev->mask[li] = want[i] ? 1 : 0;
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync((void *)ev->dev->base.consts, P.consts.data(), P.consts.size() * sizeof(float),
                             cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return cuda_fail(e, "constant upload");
    if ((e = cudaMemcpyAsync(ev->active->p, ev->mask.data(), n, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
        return cuda_fail(e, "mask upload");
    int rc = enqueue_plan(ctx, P, ev->dev, stream, nullptr);
    if (rc) return rc;
    const size_t nf = n * (P.gradient ? 33 : 1);
    ev->host_out.resize(nf);
    if ((e = cudaMemcpyAsync(ev->host_out.data(), ev->dev->out.p, nf * sizeof(float), cudaMemcpyDeviceToHost,
                             stream)) != cudaSuccess)
        return cuda_fail(e, "result download");
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(e, "evaluation");
    for (size_t li = 0; li < n; ++li) {
        const uint32_t i = P.orig[li];
        if (!want[i]) continue;
        (*mse)[i] = ev->host_out[li];
        if (grad) memcpy(grad->data() + (size_t)i * 32, ev->host_out.data() + n + li * 32, 32 * sizeof(float));
    }
    return RSR_OK;
}

}  // namespace fit
}  // namespace rsr
