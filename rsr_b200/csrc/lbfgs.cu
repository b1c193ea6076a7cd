// lbfgs.cu -- batched L-BFGS constant fitting on the engine's gradient.
//
// Restates run_lbfgs (src/engine/optimize/lbfgs.rs:9-165) for a whole
// population at once: every program keeps its own L-BFGS state (memory 6,
// at most 32 parameters, f32 arithmetic in the reference's order), and the
// evaluations the reference makes one program at a time -- one
// compute_mse_with_gradient per iteration, up to 12 compute_mse calls in the
// backtracking line search -- are issued for all programs still active in
// one launch each: the adjoint kernel for gradients, the register kernel for
// line-search MSEs.  Programs and datasets stay resident; only the constant
// pool (and a per-program active mask) is copied per evaluation.
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

struct State {
    int n = 0;                      // min(param_count, 32)
    uint32_t np = 0;                // param_count
    float x[kMaxParams] = {0};
    float s[kM][kMaxParams] = {{0}}, y[kM][kMaxParams] = {{0}};
    float rho[kM] = {0}, alpha[kM] = {0};
    float grad[kMaxParams] = {0};
    float p[kMaxParams] = {0}, next_x[kMaxParams] = {0};
    float mse = 0.0f, dir_dot = 0.0f, step = 1.0f, next_mse = 0.0f;
    int history = 0, head = 0, ls_iters = 0;
    bool done = false;
};

using fit::Evaluator;
using fit::prepare;

// The L-BFGS evaluation: the first n parameters of every program from x (or
// from next_x during the line search).
int evaluate(rsr_ctx *ctx, cudaStream_t stream, Evaluator *ev, const std::vector<State> &st,
             const std::vector<char> &want, bool use_next_x, std::vector<float> *mse, std::vector<float> *grad) {
    return fit::evaluate(
        ctx, stream, ev, want,
        [&](uint32_t i, float *params) {
            const State &s = st[i];
            for (int k = 0; k < s.n; ++k) params[k] = use_next_x ? s.next_x[k] : s.x[k];
        },
        mse, grad);
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
    Evaluator gev, mev;
    gev.dev = &ws->grad;
    gev.active = &ws->grad_active;
    mev.dev = &ws->mse;
    mev.active = &ws->mse_active;
    int rc = prepare(ctx, *pop, dsp, ds, true, stream, plan_mu, &gev);
    if (!rc) rc = prepare(ctx, *pop, dsp, ds, false, stream, plan_mu, &mev);
    if (rc) return rc;

    std::vector<State> st(N);
    for (uint32_t i = 0; i < N; ++i) {
        const uint64_t p0 = pop->param_off[i], p1 = pop->param_off[i + 1];
        st[i].np = (uint32_t)(p1 - p0);
        st[i].n = (int)std::min<uint32_t>(st[i].np, kMaxParams);
        for (int k = 0; k < st[i].n; ++k) st[i].x[k] = pop->params[p0 + k];
        st[i].done = st[i].n == 0;  // lbfgs.rs:18-21
    }
    std::vector<float> mse(N, 0.0f), grad((size_t)N * 32, 0.0f);
    std::vector<char> want(N, 1);
    // initial gradient (lbfgs.rs:32-33); programs without parameters only get
    // their MSE (their constants are not touched, lbfgs.rs:18-21)
    if ((rc = evaluate(ctx, stream, &gev, st, want, false, &mse, &grad))) return rc;
    local.gradient_evaluations++;
    for (uint32_t i = 0; i < N; ++i) {
        st[i].mse = mse[i];
        memcpy(st[i].grad, grad.data() + (size_t)i * 32, sizeof(float) * 32);
    }

    for (uint32_t iter = 0; iter < max_iterations; ++iter) {
        if (cancel && cancel->load()) return fail(RSR_ECANCELED, "fit cancelled");
        bool any = false;
        // direction (lbfgs.rs:39-106)
        for (uint32_t i = 0; i < N; ++i) {
            State &s = st[i];
            if (s.done) continue;
            const int n = s.n;
            float grad_norm_sq = 0.0f;
            for (int k = 0; k < n; ++k) grad_norm_sq += s.grad[k] * s.grad[k];
            if (sqrtf(grad_norm_sq) < 1e-5f) { s.done = true; continue; }
            float q[kMaxParams];
            for (int k = 0; k < n; ++k) q[k] = s.grad[k];
            int cur = s.head;
            for (int h = 0; h < s.history; ++h) {
                cur = cur == 0 ? kM - 1 : cur - 1;
                float dot = 0.0f;
                for (int j = 0; j < n; ++j) dot += s.s[cur][j] * q[j];
                s.alpha[cur] = s.rho[cur] * dot;
                for (int j = 0; j < n; ++j) q[j] -= s.alpha[cur] * s.y[cur][j];
            }
            float gamma = 1.0f;
            if (s.history > 0) {
                const int last = s.head == 0 ? kM - 1 : s.head - 1;
                float sy = 0.0f, yy = 0.0f;
                for (int j = 0; j < n; ++j) { sy += s.s[last][j] * s.y[last][j]; yy += s.y[last][j] * s.y[last][j]; }
                if (yy > 1e-10f) gamma = sy / yy;
            }
            for (int k = 0; k < n; ++k) q[k] *= gamma;
            cur = s.history < kM ? 0 : s.head;
            for (int h = 0; h < s.history; ++h) {
                float dot = 0.0f;
                for (int j = 0; j < n; ++j) dot += s.y[cur][j] * q[j];
                const float beta = s.rho[cur] * dot;
                for (int j = 0; j < n; ++j) q[j] += s.s[cur][j] * (s.alpha[cur] - beta);
                cur = (cur + 1) % kM;
            }
            float dd = 0.0f;
            for (int j = 0; j < n; ++j) { s.p[j] = -q[j]; dd += s.p[j] * s.grad[j]; }
            if (dd > -1e-8f) {
                for (int j = 0; j < n; ++j) s.p[j] = -s.grad[j];
                dd = -grad_norm_sq;
                s.history = 0;
            }
            s.dir_dot = dd;
            s.step = 1.0f;
            s.ls_iters = 0;
            any = true;
        }
        if (!any) break;
        local.iterations++;
        // backtracking line search (lbfgs.rs:108-125), all searching programs per launch
        std::vector<char> searching(N, 0);
        for (uint32_t i = 0; i < N; ++i) searching[i] = !st[i].done;
        for (;;) {
            bool left = false;
            for (uint32_t i = 0; i < N; ++i)
                if (searching[i]) {
                    State &s = st[i];
                    for (int j = 0; j < s.n; ++j) s.next_x[j] = s.x[j] + s.step * s.p[j];
                    left = true;
                }
            if (!left) break;
            if ((rc = evaluate(ctx, stream, &mev, st, searching, true, &mse, nullptr))) return rc;
            local.mse_evaluations++;
            for (uint32_t i = 0; i < N; ++i) {
                if (!searching[i]) continue;
                State &s = st[i];
                const float m = mse[i];
                const float c1 = 1e-4f;
                if (m <= s.mse + c1 * s.step * s.dir_dot || s.ls_iters > 10) {
                    s.next_mse = m;
                    searching[i] = 0;
                } else {
                    s.step *= 0.5f;
                    s.ls_iters++;
                }
            }
        }
        // gradient at the new point (lbfgs.rs:127)
        for (uint32_t i = 0; i < N; ++i) want[i] = !st[i].done;
        if ((rc = evaluate(ctx, stream, &gev, st, want, true, &mse, &grad))) return rc;
        local.gradient_evaluations++;
        // history update (lbfgs.rs:129-151)
        for (uint32_t i = 0; i < N; ++i) {
            State &s = st[i];
            if (s.done) continue;
            const float *ng = grad.data() + (size_t)i * 32;
            float sn[kMaxParams], yn[kMaxParams], sy = 0.0f;
            for (int j = 0; j < s.n; ++j) {
                sn[j] = s.next_x[j] - s.x[j];
                yn[j] = ng[j] - s.grad[j];
                sy += sn[j] * yn[j];
            }
            if (sy > 1e-10f) {
                memcpy(s.s[s.head], sn, sizeof(float) * s.n);
                memcpy(s.y[s.head], yn, sizeof(float) * s.n);
                s.rho[s.head] = 1.0f / sy;
                s.head = (s.head + 1) % kM;
                if (s.history < kM) s.history++;
            }
            memcpy(s.x, s.next_x, sizeof(float) * s.n);
            s.mse = s.next_mse;
            memcpy(s.grad, ng, sizeof(float) * 32);
        }
    }
    // results (lbfgs.rs:154-155): parameters beyond the first 32 unchanged
    for (uint32_t i = 0; i < N; ++i) {
        const uint64_t p0 = pop->param_off[i];
        for (uint32_t k = 0; k < st[i].np; ++k)
            params_out[p0 + k] = (int)k < st[i].n ? st[i].x[k] : pop->params[p0 + k];
        mse_out[i] = st[i].mse;
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
