// cma_es.cu -- batched CMA-ES constant fitting.
//
// Restates run_cma_es (src/engine/optimize/cmaes.rs:19-192), the fit the
// reference uses for non-differentiable programs with vector or matrix
// constants, for a whole population at once.  Each program keeps its own
// search state (mean, diagonal covariance, evolution path, step size) in f32
// with the reference's constants: 16 candidates per generation, the best 8
// recombined with log weights, c_c and c_cov from the effective selection
// mass, sigma shrunk by exp(-0.01) per generation, fitness = mse + 0.01 * L1.
// The population is encoded once with every program replicated 16 times, so
// one launch scores the 16 candidates of every program of a generation; only
// the constant pool is rewritten between launches.
//
// The reference's search vector is the flat parameters followed by a second
// copy of them (flatten_params fills the first param_count entries, then the
// loop over the constants appends them again, cmaes.rs:27-75): the second
// copy only enters the L1 term and the dimension count, and the program reads
// the first param_count entries.  That layout is kept here.
//
// Random numbers: the reference draws from rand::rng() (an unseeded
// thread-local generator).  Here each program has its own splitmix64 stream
// seeded from (seed, program index), so results do not depend on how the
// population is batched; normals follow the reference's Box-Muller form
// (cmaes.rs:13-17) in f32.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fit_eval.h"
#include "runtime.h"

namespace rsr {
namespace {

constexpr int kMaxCm = 32;  // MAX_PARAMS, cmaes.rs:8
constexpr int kLambda = 16, kMu = kLambda / 2;
constexpr float kL1 = 0.01f;  // L1_REG_LAMBDA, cmaes.rs:11
constexpr float kPi = 3.14159265358979f;
constexpr float kSigmaDecay = 0x1.fae7dp-1f;  // exp(-0.01) rounded to f32 (cmaes.rs:176)

struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }  // [0, 1), 24 bits
    // rand_normal (cmaes.rs:13-17)
    float normal() {
        const float u1 = std::max(uniform(), 1e-8f);
        const float u2 = uniform();
        return sqrtf(-2.0f * logf(u1)) * cosf(2.0f * kPi * u2);
    }
};

struct CmState {
    int n = 0;       // search dimensions (flat parameters and their copy, at most 32)
    int pc = 0;      // the program's flat parameters
    bool done = true;
    float sigma = 0.5f, c_c = 0.0f, c_cov = 0.0f;
    float mean[kMaxCm] = {0}, c_diag[kMaxCm], p_c[kMaxCm] = {0};
    float pop[kLambda][kMaxCm], step[kLambda][kMaxCm];
    float best_point[kMaxCm] = {0};
    float best_mse = 0.0f, best_fit = 0.0f;
    SplitMix rng{0};
};

}  // namespace

int fit_cma_es(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds, uint32_t max_iterations,
               uint64_t seed, cudaStream_t stream, std::mutex *plan_mu, const std::atomic<bool> *cancel,
               float *params_out, float *mse_out, rsr_fit_stats *stats) {
    NvtxRange nvtx_range("rsr: CMA-ES fit");
    const uint32_t N = pop->n_programs;
    rsr_fit_stats local{};
    if (N == 0) {
        if (stats) *stats = local;
        return RSR_OK;
    }
    // the population with every program replicated kLambda times (replica r
    // of program i at index i * kLambda + r)
    std::vector<uint32_t> code;
    std::vector<uint8_t> kinds;
    std::vector<float> params;
    std::vector<uint64_t> code_off{0}, kind_off{0}, param_off{0}, rdsp;
    for (uint32_t i = 0; i < N; ++i)
        for (int r = 0; r < kLambda; ++r) {
            code.insert(code.end(), pop->code + pop->code_off[i], pop->code + pop->code_off[i + 1]);
            kinds.insert(kinds.end(), pop->const_kinds + pop->kind_off[i], pop->const_kinds + pop->kind_off[i + 1]);
            params.insert(params.end(), pop->params + pop->param_off[i], pop->params + pop->param_off[i + 1]);
            code_off.push_back(code.size());
            kind_off.push_back(kinds.size());
            param_off.push_back(params.size());
            if (dsp) rdsp.push_back(dsp[i]);
        }
    const rsr_population rep{N * (uint32_t)kLambda, code.data(), code_off.data(), kinds.data(), kind_off.data(),
                             params.data(), param_off.data()};
    FitWorkspace ws;
    fit::Evaluator ev;
    ev.dev = &ws.mse;
    ev.active = &ws.mse_active;
    int rc = fit::prepare(ctx, rep, dsp ? rdsp.data() : nullptr, ds, false, stream, plan_mu, &ev);
    if (rc) return rc;

    // weights and effective selection mass (cmaes.rs:80-94); the two
    // logarithms are the f32-rounded natural logs
    float w[kMu], sum_w = 0.0f, mu_eff = 0.0f;
    for (int i = 0; i < kMu; ++i) {
        w[i] = std::max((float)log((double)((float)kMu + 0.5f)) - (float)log((double)(i + 1)), 0.0f);
        sum_w += w[i];
    }
    for (int i = 0; i < kMu; ++i) {
        w[i] /= sum_w;
        mu_eff += w[i] * w[i];
    }
    mu_eff = 1.0f / mu_eff;

    std::vector<CmState> st(N);
    std::vector<char> want(rep.n_programs, 0);
    std::vector<float> mse(rep.n_programs, 0.0f);
    // the point that replica r of program i is scored at next
    auto run = [&](auto point_of) {
        int r2 = fit::evaluate(
            ctx, stream, &ev, want,
            [&](uint32_t k, float *prm) {
                const CmState &s = st[k / kLambda];
                const float *x = point_of(s, k % kLambda);
                for (int j = 0; j < s.pc; ++j) prm[j] = x[j];
            },
            &mse, nullptr);
        if (!r2) local.mse_evaluations++;
        return r2;
    };

    // search vectors and the starting score (cmaes.rs:25-112)
    for (uint32_t i = 0; i < N; ++i) {
        CmState &s = st[i];
        const uint32_t pc = (uint32_t)(pop->param_off[i + 1] - pop->param_off[i]);
        s.pc = (int)std::min<uint32_t>(pc, kMaxCm);
        int n = s.pc;
        for (int j = 0; j < s.pc; ++j) s.mean[j] = pop->params[pop->param_off[i] + j];
        for (int j = 0; j < s.pc && n < kMaxCm; ++j) s.mean[n++] = pop->params[pop->param_off[i] + j];
        s.n = s.pc == 0 ? 0 : n;
        s.done = s.n == 0;
        s.rng.s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1));
        for (int j = 0; j < kMaxCm; ++j) s.c_diag[j] = 1.0f;
        const float fn = (float)s.n;
        s.c_c = (4.0f + mu_eff / fn) / (fn + 4.0f + 2.0f * mu_eff / fn);
        const float a = fn + 1.414f, b = fn + 2.0f;
        s.c_cov = (1.0f / mu_eff) * (2.0f / (a * a)) + (1.0f - 1.0f / mu_eff) * ((2.0f * mu_eff - 1.0f) / (b * b + mu_eff));
        want[(size_t)i * kLambda] = 1;  // every program, for mse_out of those without parameters
    }
    if ((rc = run([](const CmState &s, int) { return s.mean; }))) return rc;
    for (uint32_t i = 0; i < N; ++i) {
        CmState &s = st[i];
        float l1 = 0.0f;
        for (int j = 0; j < s.n; ++j) l1 += fabsf(s.mean[j]);
        s.best_mse = mse[(size_t)i * kLambda];
        s.best_fit = s.best_mse + kL1 * l1;
        memcpy(s.best_point, s.mean, sizeof(s.mean));
    }

    std::vector<std::pair<float, int>> order(kLambda);
    for (uint32_t it = 0; it < max_iterations; ++it) {
        if (cancel && cancel->load()) return fail(RSR_ECANCELED, "fit cancelled");
        // sample (cmaes.rs:119-135)
        bool any = false;
        for (uint32_t i = 0; i < N; ++i) {
            CmState &s = st[i];
            for (int r = 0; r < kLambda; ++r) want[(size_t)i * kLambda + r] = !s.done;
            if (s.done) continue;
            any = true;
            for (int r = 0; r < kLambda; ++r)
                for (int j = 0; j < s.n; ++j) {
                    const float z = s.rng.normal() * sqrtf(s.c_diag[j]);
                    s.step[r][j] = z;
                    s.pop[r][j] = s.mean[j] + s.sigma * z;
                }
        }
        if (!any) break;
        local.iterations++;
        if ((rc = run([](const CmState &s, int r) { return s.pop[r]; }))) return rc;
        // select, recombine, adapt (cmaes.rs:137-178)
        for (uint32_t i = 0; i < N; ++i) {
            CmState &s = st[i];
            if (s.done) continue;
            const int n = s.n;
            float fmse[kLambda];
            for (int r = 0; r < kLambda; ++r) {
                float l1 = 0.0f;
                for (int j = 0; j < n; ++j) l1 += fabsf(s.pop[r][j]);
                fmse[r] = mse[(size_t)i * kLambda + r];
                order[r] = {fmse[r] + kL1 * l1, r};
            }
            // sort_unstable_by(partial_cmp) on fitness, stable here; NaN last
            std::stable_sort(order.begin(), order.end(), [](const auto &x, const auto &y) {
                if (std::isnan(x.first)) return false;
                if (std::isnan(y.first)) return true;
                return x.first < y.first;
            });
            if (order[0].first < s.best_fit) {
                s.best_fit = order[0].first;
                s.best_mse = fmse[order[0].second];
                memcpy(s.best_point, s.pop[order[0].second], sizeof(s.best_point));
            }
            if (s.best_mse < 1e-8f) {
                s.done = true;
                continue;
            }
            float step_mean[kMaxCm] = {0}, old_mean[kMaxCm];
            memcpy(old_mean, s.mean, sizeof(old_mean));
            for (int k = 0; k < kMu; ++k) {
                const int r = order[k].second;
                for (int j = 0; j < n; ++j) {
                    step_mean[j] += w[k] * s.step[r][j];
                    s.mean[j] += w[k] * (s.pop[r][j] - old_mean[j]);
                }
            }
            const float path = sqrtf(s.c_c * (2.0f - s.c_c) * mu_eff);
            for (int j = 0; j < n; ++j) {
                s.p_c[j] = (1.0f - s.c_c) * s.p_c[j] + path * step_mean[j];
                float cov = 0.0f;
                for (int k = 0; k < kMu; ++k) {
                    const int r = order[k].second;
                    cov += w[k] * (s.step[r][j] * s.step[r][j]);
                }
                float c = (1.0f - s.c_cov) * s.c_diag[j] + (s.c_cov / mu_eff) * (s.p_c[j] * s.p_c[j]) +
                          s.c_cov * (1.0f - 1.0f / mu_eff) * cov;
                s.c_diag[j] = std::min(std::max(c, 1e-6f), 1e6f);
            }
            s.sigma *= kSigmaDecay;
        }
    }
    // results (cmaes.rs:180-191): the best point's first param_count entries
    for (uint32_t i = 0; i < N; ++i) {
        const CmState &s = st[i];
        const uint64_t p0 = pop->param_off[i], p1 = pop->param_off[i + 1];
        for (uint64_t k = p0; k < p1; ++k) params_out[k] = pop->params[k];
        for (int j = 0; j < s.pc; ++j) params_out[p0 + j] = s.best_point[j];
        mse_out[i] = s.best_mse;
    }
    if (stats) *stats = local;
    return RSR_OK;
}

}  // namespace rsr

using namespace rsr;

extern "C" int rsr_fit_cma_es(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp,
                              uint32_t max_iterations, uint64_t seed, float *params_out, float *mse_out,
                              rsr_fit_stats *stats) {
    if (!ctx || !pop || !params_out || !mse_out) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return fit_cma_es(ctx, pop, dsp, ds, max_iterations, seed, ctx->stream, nullptr, nullptr, params_out, mse_out,
                      stats);
}
