// nelder_mead.cu -- batched Nelder-Mead constant fitting.
//
// Restates run_nelder_mead (src/engine/optimize/nelder_mead.rs:9-165), the
// derivative-free fit the reference uses for programs with non-differentiable
// operators, for a whole population at once: every program keeps its own
// simplex over its Float constants (at most 32), with the reference's
// coefficients (reflection 1, expansion 2, contraction 0.5, shrink 0.5), its
// L1-regularised objective (mse + 0.01 * sum |c|) and its stopping rule, in
// f32 in the reference's order.  Each phase of an iteration evaluates at most
// one candidate per program, so the programs' reflections share one launch,
// their expansions and contractions a second, and the vertices of shrinking
// simplices one launch per vertex index.
//
// One deliberate difference: the simplex is ordered with a stable sort where
// the reference uses sort_unstable_by, so vertices of equal fitness keep
// their order here; the reference leaves that order unspecified.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fit_eval.h"
#include "runtime.h"

namespace rsr {
namespace {

constexpr int kMaxNm = 32;
constexpr float kL1 = 0.01f;  // L1_REG_LAMBDA, nelder_mead.rs:7
constexpr float kAlpha = 1.0f, kGamma = 2.0f, kRho = 0.5f, kSigma = 0.5f;

struct Vertex {
    float fit = 0.0f, mse = 0.0f;
    float x[kMaxNm] = {0};
};

enum Phase { PH_DONE, PH_REFLECT, PH_SECOND, PH_SHRINK };

struct NmState {
    int n = 0;                   // Float constants optimised
    uint32_t opt[kMaxNm] = {0};  // their offsets in the program's flat parameters
    Vertex s[kMaxNm + 1];
    float centroid[kMaxNm] = {0}, refl[kMaxNm] = {0}, cand[kMaxNm] = {0};
    float rfit = 0.0f, rmse = 0.0f, limit = 0.0f;
    bool expanding = false;
    Phase phase = PH_DONE;
    const float *eval_x = nullptr;  // the point the next launch evaluates
};

// nelder_mead.rs:41-50: the objective of a point
float objective(const NmState &s, const float *x, float mse) {
    float l1 = 0.0f;
    for (int j = 0; j < s.n; ++j) l1 += fabsf(x[j]);
    return mse + kL1 * l1;
}

// sort_unstable_by(partial_cmp) on fit, stable here; NaN fits sort last
void sort_simplex(NmState &s) {
    std::stable_sort(s.s, s.s + s.n + 1, [](const Vertex &a, const Vertex &b) {
        if (std::isnan(a.fit)) return false;
        if (std::isnan(b.fit)) return true;
        return a.fit < b.fit;
    });
}

}  // namespace

int fit_nelder_mead(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds,
                    uint32_t max_iterations, cudaStream_t stream, std::mutex *plan_mu,
                    const std::atomic<bool> *cancel, float *params_out, float *mse_out, rsr_fit_stats *stats) {
    NvtxRange nvtx_range("rsr: Nelder-Mead fit");
    const uint32_t N = pop->n_programs;
    rsr_fit_stats local{};
    if (N == 0) {
        if (stats) *stats = local;
        return RSR_OK;
    }
    FitWorkspace ws;
    fit::Evaluator ev;
    ev.dev = &ws.mse;
    ev.active = &ws.mse_active;
    int rc = fit::prepare(ctx, *pop, dsp, ds, false, stream, plan_mu, &ev);
    if (rc) return rc;

    // Float constants of each program and their flat offsets (nelder_mead.rs:22-31)
    std::vector<NmState> st(N);
    for (uint32_t i = 0; i < N; ++i) {
        NmState &s = st[i];
        uint32_t flat = 0;
        const uint64_t k0 = pop->kind_off[i], k1 = pop->kind_off[i + 1];
        for (uint64_t c = k0; c < k1; ++c) {
            const uint8_t kind = pop->const_kinds[c];
            if (kind == 0 && s.n < kMaxNm) {  // Scalar::Float
                s.opt[s.n] = flat;
                s.s[0].x[s.n] = pop->params[pop->param_off[i] + flat];
                ++s.n;
            }
            flat += (uint32_t)kind_width(kind);
        }
    }
    std::vector<char> want(N, 0);
    std::vector<float> mse(N, 0.0f);
    auto run = [&](const std::vector<char> &w) {
        int r = fit::evaluate(
            ctx, stream, &ev, w,
            [&](uint32_t i, float *params) {
                const NmState &s = st[i];
                for (int j = 0; j < s.n; ++j) params[s.opt[j]] = s.eval_x[j];
            },
            &mse, nullptr);
        if (!r) local.mse_evaluations++;
        return r;
    };

    // starting point, every program (also those without Float constants, for mse_out)
    for (uint32_t i = 0; i < N; ++i) {
        st[i].eval_x = st[i].s[0].x;
        want[i] = 1;
    }
    if ((rc = run(want))) return rc;
    int max_n = 0;
    for (uint32_t i = 0; i < N; ++i) {
        NmState &s = st[i];
        s.s[0].mse = mse[i];
        s.s[0].fit = objective(s, s.s[0].x, mse[i]);
        max_n = std::max(max_n, s.n);
        s.phase = s.n > 0 ? PH_REFLECT : PH_DONE;
    }
    // initial simplex: vertex k+1 moves constant k by 10% (or 0.01 near zero), nelder_mead.rs:55-61
    for (int k = 0; k < max_n; ++k) {
        for (uint32_t i = 0; i < N; ++i) {
            NmState &s = st[i];
            want[i] = s.n > k;
            if (!want[i]) continue;
            Vertex &v = s.s[k + 1];
            memcpy(v.x, s.s[0].x, sizeof(v.x));
            const float val = v.x[k];
            v.x[k] += fabsf(val) < 1e-4f ? 0.01f : val * 0.10f;
            s.eval_x = v.x;
        }
        if ((rc = run(want))) return rc;
        for (uint32_t i = 0; i < N; ++i)
            if (want[i]) {
                NmState &s = st[i];
                s.s[k + 1].mse = mse[i];
                s.s[k + 1].fit = objective(s, s.s[k + 1].x, mse[i]);
            }
    }

    for (uint32_t iter = 0; iter < max_iterations; ++iter) {
        if (cancel && cancel->load()) return fail(RSR_ECANCELED, "fit cancelled");
        // sort, stop test, centroid, reflection (nelder_mead.rs:69-97)
        bool any = false;
        for (uint32_t i = 0; i < N; ++i) {
            NmState &s = st[i];
            want[i] = 0;
            if (s.phase == PH_DONE) continue;
            sort_simplex(s);
            const int n = s.n;
            const float best_fit = s.s[0].fit, best_mse = s.s[0].mse, worst_fit = s.s[n].fit;
            if (fabsf(worst_fit - best_fit) < 1e-7f || best_mse < 1e-8f) {
                s.phase = PH_DONE;
                continue;
            }
            for (int j = 0; j < n; ++j) s.centroid[j] = 0.0f;
            for (int v = 0; v < n; ++v)
                for (int j = 0; j < n; ++j) s.centroid[j] += s.s[v].x[j];
            for (int j = 0; j < n; ++j) s.centroid[j] /= (float)n;
            for (int j = 0; j < n; ++j) s.refl[j] = s.centroid[j] + kAlpha * (s.centroid[j] - s.s[n].x[j]);
            s.eval_x = s.refl;
            want[i] = 1;
            any = true;
        }
        if (!any) break;
        local.iterations++;
        if ((rc = run(want))) return rc;
        // accept the reflection, or prepare an expansion or a contraction (nelder_mead.rs:98-138)
        any = false;
        for (uint32_t i = 0; i < N; ++i) {
            if (!want[i]) continue;
            NmState &s = st[i];
            const int n = s.n;
            s.rmse = mse[i];
            s.rfit = objective(s, s.refl, mse[i]);
            const float best_fit = s.s[0].fit, worst_fit = s.s[n].fit, second_worst = s.s[n - 1].fit;
            want[i] = 0;
            if (s.rfit >= best_fit && s.rfit < second_worst) {
                s.s[n].fit = s.rfit;
                s.s[n].mse = s.rmse;
                memcpy(s.s[n].x, s.refl, sizeof(float) * kMaxNm);
                continue;
            }
            if (s.rfit < best_fit) {
                for (int j = 0; j < n; ++j) s.cand[j] = s.centroid[j] + kGamma * (s.refl[j] - s.centroid[j]);
                s.expanding = true;
            } else {
                if (s.rfit < worst_fit) {
                    for (int j = 0; j < n; ++j) s.cand[j] = s.centroid[j] + kRho * (s.refl[j] - s.centroid[j]);
                    s.limit = s.rfit;
                } else {
                    for (int j = 0; j < n; ++j) s.cand[j] = s.centroid[j] + kRho * (s.s[n].x[j] - s.centroid[j]);
                    s.limit = worst_fit;
                }
                s.expanding = false;
            }
            s.eval_x = s.cand;
            want[i] = 1;
            any = true;
        }
        if (!any) continue;
        if ((rc = run(want))) return rc;
        // settle expansions and contractions; failed contractions shrink (nelder_mead.rs:104-150)
        int shrink_n = 0;
        std::vector<char> shrinking(N, 0);
        for (uint32_t i = 0; i < N; ++i) {
            if (!want[i]) continue;
            NmState &s = st[i];
            const int n = s.n;
            const float cfit = objective(s, s.cand, mse[i]);
            if (s.expanding) {
                if (cfit < s.rfit) {
                    s.s[n].fit = cfit;
                    s.s[n].mse = mse[i];
                    memcpy(s.s[n].x, s.cand, sizeof(float) * kMaxNm);
                } else {
                    s.s[n].fit = s.rfit;
                    s.s[n].mse = s.rmse;
                    memcpy(s.s[n].x, s.refl, sizeof(float) * kMaxNm);
                }
            } else if (cfit < s.limit) {
                s.s[n].fit = cfit;
                s.s[n].mse = mse[i];
                memcpy(s.s[n].x, s.cand, sizeof(float) * kMaxNm);
            } else {
                const float *best = s.s[0].x;
                for (int v = 1; v <= n; ++v)
                    for (int j = 0; j < n; ++j) s.s[v].x[j] = best[j] + kSigma * (s.s[v].x[j] - best[j]);
                shrinking[i] = 1;
                shrink_n = std::max(shrink_n, n);
            }
        }
        for (int v = 1; v <= shrink_n; ++v) {
            for (uint32_t i = 0; i < N; ++i) {
                want[i] = shrinking[i] && st[i].n >= v;
                if (want[i]) st[i].eval_x = st[i].s[v].x;
            }
            if ((rc = run(want))) return rc;
            for (uint32_t i = 0; i < N; ++i)
                if (want[i]) {
                    NmState &s = st[i];
                    s.s[v].mse = mse[i];
                    s.s[v].fit = objective(s, s.s[v].x, mse[i]);
                }
        }
    }
    // results (nelder_mead.rs:152-157): the best vertex's constants, its MSE
    for (uint32_t i = 0; i < N; ++i) {
        NmState &s = st[i];
        const uint64_t p0 = pop->param_off[i], p1 = pop->param_off[i + 1];
        for (uint64_t k = p0; k < p1; ++k) params_out[k] = pop->params[k];
        if (s.n > 0) {
            sort_simplex(s);
            for (int j = 0; j < s.n; ++j) params_out[p0 + s.opt[j]] = s.s[0].x[j];
        }
        mse_out[i] = s.s[0].mse;
    }
    if (stats) *stats = local;
    return RSR_OK;
}

}  // namespace rsr

using namespace rsr;

extern "C" int rsr_fit_nelder_mead(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds,
                                   const rsr_dataset *dsp, uint32_t max_iterations, float *params_out,
                                   float *mse_out, rsr_fit_stats *stats) {
    if (!ctx || !pop || !params_out || !mse_out) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return fit_nelder_mead(ctx, pop, dsp, ds, max_iterations, ctx->stream, nullptr, nullptr, params_out, mse_out,
                           stats);
}
