// lbfgs.cu -- batched L-BFGS constant fitting with its state on the device.
//
// Restates run_lbfgs (src/engine/optimize/lbfgs.rs:9-165) for a whole
// population at once.  Every program keeps its own L-BFGS state (memory 6, at
// most 32 parameters, f32 arithmetic in the reference's order) in device
// memory, and the whole iteration runs on the device with no host round trip:
//
//   direction     one thread per program: convergence test (|g| < 1e-5) and
//                 the two-loop recursion (lbfgs.rs:39-106); writes the first
//                 trial point x + p into the MSE plan's constant pool and
//                 marks the program active there.
//   12 rounds of  the MSE evaluation of every program still searching (the
//                 register kernel, which skips inactive programs; a round
//                 nobody searches in costs one empty launch per kernel), then
//                 the Armijo test (c1 = 1e-4, lbfgs.rs:108-125): accept, or
//                 halve the step and write the next trial point.  A search
//                 accepts by its 12th evaluation at the latest (ls_iters > 10),
//                 so 12 rounds always suffice.
//   gradient      the adjoint kernel at the accepted points of the programs
//                 that searched (lbfgs.rs:127),
//   update        the history pair (s, y, rho) when s.y > 1e-10, the move to
//                 the new point (lbfgs.rs:129-151).
//
// One iteration is captured once as a CUDA graph and replayed; the host
// reads a few counters after each replay (one stream synchronisation per
// iteration) to stop when no program is left and to count launches.  The
// programs' MSEs and gradients come from the same plans and kernels as a
// one-program call, so the fit takes exactly the steps of the sequential
// restatement fed with the engine's evaluations.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fit_eval.h"
#include "runtime.h"

namespace rsr {
namespace {

constexpr int kMaxParams = 32;  // lbfgs.rs:6
constexpr int kM = 6;           // lbfgs.rs:7
constexpr int kRounds = 12;     // line-search evaluations per iteration at most (lbfgs.rs:111-125)
// counters[r], r < kRounds: programs searching in round r; counters[kRounds]:
// programs still searching after the last round (always 0);
// counters[kCountGrad]: programs whose gradient is evaluated at the new point.
constexpr int kCountGrad = kRounds + 1;
constexpr int kCounters = kRounds + 2;

// Structure-of-arrays state: element k of program i of an [K][N] array is at
// [k * N + i], so one-thread-per-program kernels read it coalesced.
struct LbfgsDev {
    uint32_t N;
    uint32_t n_grad_plan;        // programs in the gradient plan (its grad block starts there)
    const uint32_t *n;           // [N] min(param_count, 32)
    const uint32_t *grad_li;     // [N] launch index in the gradient plan
    const uint32_t *mse_li;      // [N] launch index in the MSE plan
    const uint32_t *grad_coff;   // [N] constant-pool offset in the gradient plan
    const uint32_t *mse_coff;    // [N] constant-pool offset in the MSE plan
    float *gpool, *mpool;        // the plans' constant pools
    uint8_t *gmask, *mmask;      // the plans' active masks (launch order)
    const float *gout;           // gradient plan results: mse[n] | grad[n][32]
    const float *mout;           // MSE plan results: mse[n]
    float *x, *grad, *p, *next_x;  // [32][N]
    float *s, *y;                  // [kM][32][N]
    float *rho, *alpha;            // [kM][N]
    float *mse, *next_mse, *dir_dot, *step;  // [N]
    int *history, *head, *ls_iters;           // [N]
    uint8_t *done, *searching;                // [N]
    uint32_t *counters;                       // [kCounters]
};

static size_t al256(size_t v) { return (v + 255) & ~(size_t)255; }

__global__ void lbfgs_start_kernel(LbfgsDev d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const uint32_t N = d.N, n = d.n[i], gl = d.grad_li[i];
    d.mse[i] = d.gout[gl];
    for (int k = 0; k < kMaxParams; ++k) d.grad[k * N + i] = d.gout[d.n_grad_plan + (size_t)gl * 32 + k];
    for (uint32_t k = 0; k < n; ++k) d.x[k * N + i] = d.gpool[d.grad_coff[i] + k];
    d.history[i] = 0;
    d.head[i] = 0;
    d.done[i] = n == 0;  // lbfgs.rs:18-21
    d.searching[i] = 0;
}

// Search direction (lbfgs.rs:39-106) and the first trial point.
__global__ void lbfgs_direction_kernel(LbfgsDev d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const uint32_t N = d.N, ml = d.mse_li[i];
    d.searching[i] = 0;
    d.mmask[ml] = 0;
    if (d.done[i]) return;
    const int n = (int)d.n[i];
    float grad_norm_sq = 0.0f;
    for (int k = 0; k < n; ++k) grad_norm_sq += d.grad[k * N + i] * d.grad[k * N + i];
    if (sqrtf(grad_norm_sq) < 1e-5f) {
        d.done[i] = 1;
        return;
    }
    float q[kMaxParams];
    for (int k = 0; k < n; ++k) q[k] = d.grad[k * N + i];
    const int history = d.history[i], head = d.head[i];
    int cur = head;
    for (int h = 0; h < history; ++h) {
        cur = cur == 0 ? kM - 1 : cur - 1;
        const float *sc = d.s + (size_t)cur * kMaxParams * N, *yc = d.y + (size_t)cur * kMaxParams * N;
        float dot = 0.0f;
        for (int j = 0; j < n; ++j) dot += sc[j * N + i] * q[j];
        const float al = d.rho[cur * N + i] * dot;
        d.alpha[cur * N + i] = al;
        for (int j = 0; j < n; ++j) q[j] -= al * yc[j * N + i];
    }
    float gamma = 1.0f;
    if (history > 0) {
        const int last = head == 0 ? kM - 1 : head - 1;
        const float *sl = d.s + (size_t)last * kMaxParams * N, *yl = d.y + (size_t)last * kMaxParams * N;
        float sy = 0.0f, yy = 0.0f;
        for (int j = 0; j < n; ++j) {
            sy += sl[j * N + i] * yl[j * N + i];
            yy += yl[j * N + i] * yl[j * N + i];
        }
        if (yy > 1e-10f) gamma = sy / yy;
    }
    for (int k = 0; k < n; ++k) q[k] *= gamma;
    cur = history < kM ? 0 : head;
    for (int h = 0; h < history; ++h) {
        const float *sc = d.s + (size_t)cur * kMaxParams * N, *yc = d.y + (size_t)cur * kMaxParams * N;
        float dot = 0.0f;
        for (int j = 0; j < n; ++j) dot += yc[j * N + i] * q[j];
        const float beta = d.rho[cur * N + i] * dot;
        const float diff = d.alpha[cur * N + i] - beta;
        for (int j = 0; j < n; ++j) q[j] += sc[j * N + i] * diff;
        cur = (cur + 1) % kM;
    }
    float dd = 0.0f;
    for (int j = 0; j < n; ++j) {
        const float pj = -q[j];
        d.p[j * N + i] = pj;
        dd += pj * d.grad[j * N + i];
    }
    if (dd > -1e-8f) {
        for (int j = 0; j < n; ++j) d.p[j * N + i] = -d.grad[j * N + i];
        dd = -grad_norm_sq;
        d.history[i] = 0;
    }
    d.dir_dot[i] = dd;
    const float step = 1.0f;
    d.step[i] = step;
    d.ls_iters[i] = 0;
    d.searching[i] = 1;
    float *pool = d.mpool + d.mse_coff[i];
    for (int j = 0; j < n; ++j) {
        const float nx = d.x[j * N + i] + step * d.p[j * N + i];
        d.next_x[j * N + i] = nx;
        pool[j] = nx;
    }
    d.mmask[ml] = 1;
    atomicAdd(&d.counters[0], 1u);
}

// Armijo test of round r's evaluations (lbfgs.rs:108-125).
__global__ void lbfgs_line_search_kernel(LbfgsDev d, int r) {
    if (d.counters[r] == 0u) return;  // nobody searched in this round
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N || !d.searching[i]) return;
    const uint32_t N = d.N, ml = d.mse_li[i];
    const float m = d.mout[ml];
    const float c1 = 1e-4f;
    const float step = d.step[i];
    if (m <= d.mse[i] + c1 * step * d.dir_dot[i] || d.ls_iters[i] > 10) {
        d.next_mse[i] = m;
        d.searching[i] = 0;
        d.mmask[ml] = 0;
        return;
    }
    const float ns = step * 0.5f;
    d.step[i] = ns;
    d.ls_iters[i] += 1;
    const int n = (int)d.n[i];
    float *pool = d.mpool + d.mse_coff[i];
    for (int j = 0; j < n; ++j) {
        const float nx = d.x[j * N + i] + ns * d.p[j * N + i];
        d.next_x[j * N + i] = nx;
        pool[j] = nx;
    }
    atomicAdd(&d.counters[r + 1], 1u);
}

// The accepted points into the gradient plan (lbfgs.rs:127).
__global__ void lbfgs_gradient_points_kernel(LbfgsDev d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N) return;
    const uint32_t N = d.N, gl = d.grad_li[i];
    if (d.done[i]) {
        d.gmask[gl] = 0;
        return;
    }
    const int n = (int)d.n[i];
    float *pool = d.gpool + d.grad_coff[i];
    for (int j = 0; j < n; ++j) pool[j] = d.next_x[j * N + i];
    d.gmask[gl] = 1;
    atomicAdd(&d.counters[kCountGrad], 1u);
}

// History update and move (lbfgs.rs:129-151).
__global__ void lbfgs_update_kernel(LbfgsDev d) {
    if (d.counters[kCountGrad] == 0u) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.N || d.done[i]) return;
    const uint32_t N = d.N;
    const int n = (int)d.n[i];
    const float *ng = d.gout + d.n_grad_plan + (size_t)d.grad_li[i] * 32;
    float sy = 0.0f;
    for (int j = 0; j < n; ++j) {
        const float sn = d.next_x[j * N + i] - d.x[j * N + i];
        const float yn = ng[j] - d.grad[j * N + i];
        sy += sn * yn;
    }
    if (sy > 1e-10f) {
        const int h = d.head[i];
        float *sh = d.s + (size_t)h * kMaxParams * N, *yh = d.y + (size_t)h * kMaxParams * N;
        for (int j = 0; j < n; ++j) {
            sh[j * N + i] = d.next_x[j * N + i] - d.x[j * N + i];
            yh[j * N + i] = ng[j] - d.grad[j * N + i];
        }
        d.rho[h * N + i] = 1.0f / sy;
        d.head[i] = (h + 1) % kM;
        if (d.history[i] < kM) d.history[i] += 1;
    }
    for (int j = 0; j < n; ++j) d.x[j * N + i] = d.next_x[j * N + i];
    d.mse[i] = d.next_mse[i];
    for (int k = 0; k < kMaxParams; ++k) d.grad[k * N + i] = ng[k];
}

// Device state of N programs: the LbfgsDev pointers into one buffer.
size_t state_bytes(uint32_t N, LbfgsDev *d, char *base) {
    size_t o = 0;
    auto take = [&](size_t bytes) {
        char *p = base ? base + o : nullptr;
        o += al256(bytes);
        return p;
    };
    const size_t f = sizeof(float), u = sizeof(uint32_t);
    d->n = (const uint32_t *)take(N * u);
    d->grad_li = (const uint32_t *)take(N * u);
    d->mse_li = (const uint32_t *)take(N * u);
    d->grad_coff = (const uint32_t *)take(N * u);
    d->mse_coff = (const uint32_t *)take(N * u);
    d->x = (float *)take((size_t)kMaxParams * N * f);
    d->grad = (float *)take((size_t)kMaxParams * N * f);
    d->p = (float *)take((size_t)kMaxParams * N * f);
    d->next_x = (float *)take((size_t)kMaxParams * N * f);
    d->s = (float *)take((size_t)kM * kMaxParams * N * f);
    d->y = (float *)take((size_t)kM * kMaxParams * N * f);
    d->rho = (float *)take((size_t)kM * N * f);
    d->alpha = (float *)take((size_t)kM * N * f);
    d->mse = (float *)take(N * f);
    d->next_mse = (float *)take(N * f);
    d->dir_dot = (float *)take(N * f);
    d->step = (float *)take(N * f);
    d->history = (int *)take(N * sizeof(int));
    d->head = (int *)take(N * sizeof(int));
    d->ls_iters = (int *)take(N * sizeof(int));
    d->done = (uint8_t *)take(N);
    d->searching = (uint8_t *)take(N);
    d->counters = (uint32_t *)take(kCounters * u);
    return o;
}

// One L-BFGS iteration on stream st (capturable).
int enqueue_iteration(rsr_ctx *ctx, fit::Evaluator &gev, fit::Evaluator &mev, const LbfgsDev &d, cudaStream_t st) {
    const uint32_t blocks = (d.N + 127) / 128;
    cudaError_t e;
    if ((e = cudaMemsetAsync(d.counters, 0, kCounters * sizeof(uint32_t), st)) != cudaSuccess)
        return cuda_fail(e, "L-BFGS counters");
    lbfgs_direction_kernel<<<blocks, 128, 0, st>>>(d);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "L-BFGS direction");
    ctx->launches++;
    int rc;
    for (int r = 0; r < kRounds; ++r) {
        mev.dev->base.run_if = d.counters + r;
        if ((rc = enqueue_plan(ctx, mev.plan, mev.dev, st, nullptr))) return rc;
        lbfgs_line_search_kernel<<<blocks, 128, 0, st>>>(d, r);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "L-BFGS line search");
        ctx->launches++;
    }
    lbfgs_gradient_points_kernel<<<blocks, 128, 0, st>>>(d);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "L-BFGS gradient points");
    ctx->launches++;
    gev.dev->base.run_if = d.counters + kCountGrad;
    if ((rc = enqueue_plan(ctx, gev.plan, gev.dev, st, nullptr))) return rc;
    lbfgs_update_kernel<<<blocks, 128, 0, st>>>(d);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "L-BFGS update");
    ctx->launches++;
    return RSR_OK;
}

}  // namespace

int fit_population(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds,
                   uint32_t max_iterations, cudaStream_t stream, std::mutex *plan_mu,
                   const std::atomic<bool> *cancel, FitWorkspace *ws, float *params_out, float *mse_out,
                   rsr_fit_stats *stats) {
    NvtxRange nvtx_range("rsr: L-BFGS fit");
    const uint32_t N = pop->n_programs;
    rsr_fit_stats local{};
    if (N == 0) {
        if (stats) *stats = local;
        return RSR_OK;
    }
    FitWorkspace own;
    if (!ws) ws = &own;
    fit::Evaluator gev, mev;
    gev.dev = &ws->grad;
    gev.active = &ws->grad_active;
    mev.dev = &ws->mse;
    mev.active = &ws->mse_active;
    int rc = fit::prepare(ctx, *pop, dsp, ds, true, stream, plan_mu, &gev);
    if (!rc) rc = fit::prepare(ctx, *pop, dsp, ds, false, stream, plan_mu, &mev);
    if (rc) return rc;

    // device state, and the per-program maps into the two plans
    LbfgsDev d{};
    const size_t bytes = state_bytes(N, &d, nullptr);
    cudaError_t e;
    if ((e = ws->lbfgs_state.reserve(bytes)) != cudaSuccess) return cuda_fail(e, "L-BFGS state");
    state_bytes(N, &d, (char *)ws->lbfgs_state.p);
    d.N = N;
    d.n_grad_plan = (uint32_t)gev.plan.progs.size();
    d.gpool = const_cast<float *>(gev.dev->base.consts);
    d.mpool = const_cast<float *>(mev.dev->base.consts);
    d.gmask = (uint8_t *)gev.active->p;
    d.mmask = (uint8_t *)mev.active->p;
    d.gout = gev.dev->mse;
    d.mout = mev.dev->mse;
    std::vector<uint32_t> maps((size_t)5 * N);
    for (uint32_t i = 0; i < N; ++i)
        maps[i] = (uint32_t)std::min<uint64_t>(pop->param_off[i + 1] - pop->param_off[i], kMaxParams);
    for (size_t li = 0; li < gev.plan.progs.size(); ++li) {
        const uint32_t i = gev.plan.orig[li];
        maps[N + i] = (uint32_t)li;
        maps[3 * (size_t)N + i] = gev.plan.progs[li].const_off;
    }
    for (size_t li = 0; li < mev.plan.progs.size(); ++li) {
        const uint32_t i = mev.plan.orig[li];
        maps[2 * (size_t)N + i] = (uint32_t)li;
        maps[4 * (size_t)N + i] = mev.plan.progs[li].const_off;
    }
    const uint32_t *dst[5] = {d.n, d.grad_li, d.mse_li, d.grad_coff, d.mse_coff};
    for (int m = 0; m < 5; ++m)
        if ((e = cudaMemcpyAsync((void *)dst[m], maps.data() + (size_t)m * N, N * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, stream)) != cudaSuccess)
            return cuda_fail(e, "L-BFGS maps");
    if ((e = ws->lbfgs_counts.reserve(kCounters * sizeof(uint32_t))) != cudaSuccess)
        return cuda_fail(e, "cudaHostAlloc");
    uint32_t *counts = (uint32_t *)ws->lbfgs_counts.p;

    // initial evaluation at the starting constants (lbfgs.rs:32-33); programs
    // without parameters only get their MSE (lbfgs.rs:18-21)
    if ((e = cudaMemsetAsync(gev.active->p, 1, gev.plan.progs.size(), stream)) != cudaSuccess)
        return cuda_fail(e, "mask");
    gev.dev->base.run_if = nullptr;
    if ((rc = enqueue_plan(ctx, gev.plan, gev.dev, stream, nullptr))) return rc;
    local.gradient_evaluations++;
    lbfgs_start_kernel<<<(N + 127) / 128, 128, 0, stream>>>(d);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "L-BFGS start");
    ctx->launches++;

    // one iteration as a CUDA graph, replayed
    cudaGraphExec_t exec = nullptr;
    if (ctx->opts.use_graphs && max_iterations > 0) {
        cudaGraph_t g = nullptr;
        if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return cuda_fail(e, "L-BFGS graph capture");
        const uint64_t before = ctx->launches.load();
        rc = enqueue_iteration(ctx, gev, mev, d, stream);
        e = cudaStreamEndCapture(stream, &g);
        ctx->launches = before;  // counted at replay
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "L-BFGS graph capture");
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "L-BFGS graph instantiate");
    }
    uint64_t replays = 0;
    for (uint32_t iter = 0; iter < max_iterations; ++iter) {
        if (cancel && cancel->load()) {
            rc = fail(RSR_ECANCELED, "fit cancelled");
            break;
        }
        if (exec) {
            if ((e = cudaGraphLaunch(exec, stream)) != cudaSuccess) {
                rc = cuda_fail(e, "L-BFGS graph launch");
                break;
            }
            replays++;
        } else if ((rc = enqueue_iteration(ctx, gev, mev, d, stream))) {
            break;
        }
        if ((e = cudaMemcpyAsync(counts, d.counters, kCounters * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                 stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            rc = cuda_fail(e, "L-BFGS iteration");
            break;
        }
        if (counts[0] == 0) break;  // every program has converged or has no parameters
        local.iterations++;
        for (int r = 0; r < kRounds; ++r) local.mse_evaluations += counts[r] ? 1u : 0u;
        if (counts[kCountGrad]) local.gradient_evaluations++;
    }
    if (exec) {
        // launches of the replays: per iteration the direction, line-search,
        // gradient-point and update kernels plus the two plans' launches
        uint64_t per_plan_g = 1, per_plan_m = 1;
        for (const Group &g : gev.plan.groups) per_plan_g += g.n_items ? 1 : 0;
        for (const Group &g : mev.plan.groups) per_plan_m += g.n_items ? 1 : 0;
        ctx->launches += replays * (3 + kRounds + kRounds * per_plan_m + per_plan_g);
        cudaGraphExecDestroy(exec);
    }
    gev.dev->base.run_if = nullptr;
    mev.dev->base.run_if = nullptr;
    if (rc) {
        cudaStreamSynchronize(stream);
        return rc;
    }

    // results (lbfgs.rs:154-155): parameters beyond the first 32 unchanged
    std::vector<float> x((size_t)kMaxParams * N), m(N);
    if ((e = cudaMemcpyAsync(x.data(), d.x, x.size() * sizeof(float), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(m.data(), d.mse, N * sizeof(float), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
        return cuda_fail(e, "L-BFGS results");
    for (uint32_t i = 0; i < N; ++i) {
        const uint64_t p0 = pop->param_off[i];
        const uint32_t np = (uint32_t)(pop->param_off[i + 1] - p0), n = std::min<uint32_t>(np, kMaxParams);
        for (uint32_t k = 0; k < np; ++k) params_out[p0 + k] = k < n ? x[(size_t)k * N + i] : pop->params[p0 + k];
        mse_out[i] = m[i];
    }
    if (stats) *stats = local;
    return RSR_OK;
}

}  // namespace rsr

using namespace rsr;

extern "C" int rsr_fit_lbfgs(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp,
                             uint32_t max_iterations, float *params_out, float *mse_out, rsr_fit_stats *stats) {
    if (!ctx || !pop || !params_out || !mse_out) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return fit_population(ctx, pop, dsp, ds, max_iterations, ctx->stream, nullptr, nullptr, nullptr, params_out,
                          mse_out, stats);
}
