// serving.cu -- the device-resident request loop (rsr_server).
//
// Island threads submit evaluation and constant-fit jobs from any thread
// (rsr_submit copies the population, so the caller's arrays may go away);
// `slots` worker threads, each with its own CUDA stream and cached device
// buffers, take jobs from one FIFO queue, so several jobs are on the device
// at once and their kernels overlap.  Continuous batching: a worker that
// frees up takes the oldest waiting job and, for evaluation jobs, every job
// of the same kind queued directly behind it (up to max_batch_programs
// programs and the memory budget), encodes them as one population and runs
// one launch; results are scattered back per job.  Memory admission: each
// job carries an estimate of its device footprint; a job above the budget is
// refused at submit, and a batch waits until the in-flight footprints leave
// room for it.
//
// Results do not depend on the mix: a program's MSE and gradient come from
// the same kernels whether it runs alone or merged; the register kernel's
// points-per-thread follows the largest dataset in a launch, which changes
// the order of the f32 partial sums only (within the engine's 1e-6 MSE
// tolerance).  Fit jobs run one per slot, exactly as rsr_fit_lbfgs.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

namespace rsr {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Job {
    uint64_t ticket = 0;
    uint32_t kind = RSR_JOB_MSE, fit_iterations = 0;
    std::vector<uint32_t> code;
    std::vector<uint64_t> code_off;
    std::vector<uint8_t> kinds;
    std::vector<uint64_t> kind_off;
    std::vector<float> params;
    std::vector<uint64_t> param_off;
    std::vector<uint64_t> dsp;      // dataset per program
    std::vector<uint64_t> handles;  // distinct datasets, referenced while the job lives
    float *mse_out = nullptr, *grad_out = nullptr, *params_out = nullptr;
    uint64_t seed = 0;  // RSR_JOB_FIT_AUTO: CMA-ES streams
    uint64_t est_bytes = 0, program_points = 0;
    std::atomic<bool> cancel{false};
    uint32_t state = RSR_JOB_QUEUED;
    int status = RSR_OK;
    std::string msg;
    uint32_t batch_jobs = 0;
    Clock::time_point t_submit, t_start, t_done;

    uint32_t n() const { return (uint32_t)(code_off.size() - 1); }
    rsr_population pop() const {
        rsr_population p{};
        p.n_programs = n();
        p.code = code.data();
        p.code_off = code_off.data();
        p.const_kinds = kinds.data();
        p.kind_off = kind_off.data();
        p.params = params.data();
        p.param_off = param_off.data();
        return p;
    }
};
using JobPtr = std::shared_ptr<Job>;

struct Slot {
    // a batch runs as up to two chunks of programs, each with its own plan
    // buffers and stream: the second is planned while the first runs
    cudaStream_t st = nullptr, st2 = nullptr;
    EncodeScratch enc;  // the slot plans with its own encoding storage and threads
    DevicePlan dev, dev2;
    FitWorkspace fit;
    HostBuf host;       // pinned results of a batch
    size_t cached() const {
        return dev.pool.cap + dev.partials.cap + dev.out.cap + dev2.pool.cap + dev2.partials.cap + dev2.out.cap +
               fit.grad.pool.cap + fit.grad.partials.cap + fit.grad.out.cap + fit.mse.pool.cap +
               fit.mse.partials.cap + fit.mse.out.cap;
    }
    void trim() {
        dev.pool.release(); dev.partials.release(); dev.out.release(); dev.counters.release();
        dev2.pool.release(); dev2.partials.release(); dev2.out.release(); dev2.counters.release();
        for (DevicePlan *d : {&fit.grad, &fit.mse}) {
            d->pool.release(); d->partials.release(); d->out.release(); d->counters.release();
        }
        fit.grad_active.release();
        fit.mse_active.release();
    }
};

// The optimiser optimize_individual_constants (src/engine/optimize/mod.rs:
// 24-58) picks for a program: L-BFGS when every opcode is differentiable
// (all but the inverses), else CMA-ES when a constant is a vector or matrix,
// else Nelder-Mead.
enum FitMethod { FIT_LBFGS = 0, FIT_CMAES = 1, FIT_NM = 2 };

int fit_method(const Job &j, uint32_t i) {
    for (uint64_t k = j.code_off[i]; k < j.code_off[i + 1]; ++k) {
        const uint32_t op = j.code[k] & 0xFFu;
        if (op == INVERSE_M2 || op == INVERSE_M3) {
            for (uint64_t c = j.kind_off[i]; c < j.kind_off[i + 1]; ++c)
                if (j.kinds[c] >= 3) return FIT_CMAES;  // Vec2, Vec3, Mat2, Mat3
            return FIT_NM;
        }
    }
    return FIT_LBFGS;
}

// Device bytes one job's launch(es) hold: plan pool, partial sums, outputs.
uint64_t estimate_bytes(const Job &j, const std::vector<uint64_t> &n_eval_per_prog) {
    const bool grad = j.kind != RSR_JOB_MSE;
    uint64_t b = 4096;
    for (uint32_t i = 0; i < j.n(); ++i) {
        const uint64_t len = j.code_off[i + 1] - j.code_off[i];
        const uint64_t np = j.param_off[i + 1] - j.param_off[i];
        const uint64_t parts = std::max<uint64_t>(1, (n_eval_per_prog[i] + 4095) / 4096);
        uint64_t per = 64 + 16 * (len + 1) + 4 * (np + 1) + 24 * parts + 8 * parts * (grad ? 33 : 1) + 4 * 33;
        if (j.kind == RSR_JOB_FIT || j.kind == RSR_JOB_FIT_AUTO)
            per += 64 + 16 * (len + 1) + 4 * (np + 1) + 24 * parts + 8 * parts + 8;
        // CMA-ES plans 16 copies of the program
        if (j.kind == RSR_JOB_FIT_AUTO && fit_method(j, i) == FIT_CMAES) per *= 16;
        b += per;
    }
    return b;
}

}  // namespace
}  // namespace rsr

using namespace rsr;

struct rsr_server {
    rsr_ctx *ctx = nullptr;
    rsr_server_options opts{};
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_mem;
    std::deque<JobPtr> queue;
    std::unordered_map<uint64_t, JobPtr> jobs;
    uint64_t next_ticket = 1;
    bool stopping = false;
    uint64_t mem_inflight = 0, mem_peak = 0;
    std::vector<std::unique_ptr<Slot>> slots;
    std::vector<std::thread> workers;
    // statistics since the last reset
    uint64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, refused = 0, launches = 0;
    std::vector<double> lat;
    double pp = 0.0;
    bool have_t0 = false;
    Clock::time_point t0, t_last;
};

namespace rsr {
namespace {

void unref_datasets(rsr_ctx *ctx, const std::vector<JobPtr> &batch) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    for (const JobPtr &j : batch)
        for (uint64_t h : j->handles) {
            auto it = ctx->datasets.find(h);
            if (it != ctx->datasets.end()) it->second->refs--;
        }
}

std::string thread_error() {
    const char *m = rsr_last_error();
    return m ? std::string(m) : std::string();
}

// One launch over the merged population of `batch` (all MSE or all
// MSE+gradient); writes every job's outputs.  Returns the launch status.
int run_eval(rsr_server *S, Slot &slot, const std::vector<JobPtr> &batch) {
    NvtxRange nvtx_range("rsr: serving batch");
    rsr_ctx *ctx = S->ctx;
    const bool gradient = batch[0]->kind == RSR_JOB_MSE_GRAD;
    std::vector<uint32_t> code;
    std::vector<uint64_t> code_off{0}, kind_off{0}, param_off{0}, dsp;
    std::vector<uint8_t> kinds;
    std::vector<float> params;
    std::vector<uint32_t> first;  // first merged index of each job
    for (const JobPtr &j : batch) {
        first.push_back((uint32_t)dsp.size());
        for (uint32_t i = 0; i < j->n(); ++i) {
            code.insert(code.end(), j->code.begin() + j->code_off[i], j->code.begin() + j->code_off[i + 1]);
            kinds.insert(kinds.end(), j->kinds.begin() + j->kind_off[i], j->kinds.begin() + j->kind_off[i + 1]);
            params.insert(params.end(), j->params.begin() + j->param_off[i], j->params.begin() + j->param_off[i + 1]);
            code_off.push_back(code.size());
            kind_off.push_back(kinds.size());
            param_off.push_back(params.size());
            dsp.push_back(j->dsp[i]);
        }
    }
    const uint32_t n = (uint32_t)dsp.size();
    if (n == 0) return RSR_OK;
    // Batches of 512 programs or more run as two chunks (a third, then the
    // rest): the second chunk is encoded while the first one's kernels run,
    // and its launches fill the SMs the first one's tail frees.
    const uint32_t split = n >= 512 ? n / 3 : n;
    const uint32_t starts[3] = {0, split, n};
    const int n_chunks = split < n ? 2 : 1;
    const size_t stride = gradient ? 33 : 1;
    cudaError_t e;
    if ((e = slot.host.reserve((size_t)n * stride * sizeof(float))) != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
    float *res = (float *)slot.host.p;
    Plan plans[2];
    int rc = RSR_OK;
    int launched = 0;
    for (int k = 0; k < n_chunks && !rc; ++k) {
        const uint32_t s0 = starts[k], cnt = starts[k + 1] - s0;
        rsr_population pop{cnt, code.data(), code_off.data() + s0, kinds.data(), kind_off.data() + s0,
                           params.data(), param_off.data() + s0};
        DevicePlan &dev = k ? slot.dev2 : slot.dev;
        cudaStream_t st = k ? slot.st2 : slot.st;
        // ctx->mu only around the dataset and tuning tables: slots encode in parallel
        rc = build_plan(ctx, pop, dsp.data() + s0, 0, RSR_KERNEL_AUTO, gradient, MODE_MSE, &plans[k], &slot.enc,
                        &ctx->mu);
        if (!rc) rc = upload_plan(ctx, plans[k], &dev, st);
        if (!rc) rc = enqueue_plan(ctx, plans[k], &dev, st, nullptr);
        if (!rc && (e = cudaMemcpyAsync(res + (size_t)s0 * stride, dev.out.p, (size_t)cnt * stride * sizeof(float),
                                        cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            rc = cuda_fail(e, "result download");
        if (!rc) launched = k + 1;
    }
    // wait for whatever was launched, error or not, before buffers are reused
    for (int k = 0; k < n_chunks; ++k) {
        const cudaError_t se = cudaStreamSynchronize(k ? slot.st2 : slot.st);
        if (!rc && se != cudaSuccess) rc = cuda_fail(se, "evaluation");
    }
    if (rc) return rc;
    // scatter: merged index -> (job, local index)
    for (int k = 0; k < launched; ++k) {
        const uint32_t s0 = starts[k], cnt = starts[k + 1] - s0;
        const float *r = res + (size_t)s0 * stride;
        for (uint32_t li = 0; li < cnt; ++li) {
            const uint32_t m = s0 + plans[k].orig[li];
            const size_t b = std::upper_bound(first.begin(), first.end(), m) - first.begin() - 1;
            Job &j = *batch[b];
            const uint32_t q = m - first[b];
            j.mse_out[q] = r[li];
            if (gradient) memcpy(j.grad_out + (size_t)q * 32, r + cnt + (size_t)li * 32, 32 * sizeof(float));
        }
    }
    return RSR_OK;
}

// An RSR_JOB_FIT_AUTO job: the programs split by the optimiser the reference
// would pick for them (fit_method), each group fitted by its batched driver
// on this slot's stream, results scattered back in the job's order.
int fit_auto(rsr_server *S, Slot &slot, Job &j) {
    NvtxRange nvtx_range("rsr: serving fit (auto)");
    const uint32_t n = j.n();
    struct Sub {
        std::vector<uint32_t> idx, code;
        std::vector<uint8_t> kinds;
        std::vector<float> params, out_params, out_mse;
        std::vector<uint64_t> code_off{0}, kind_off{0}, param_off{0}, dsp;
    } sub[3];
    for (uint32_t i = 0; i < n; ++i) {
        Sub &g = sub[fit_method(j, i)];
        g.idx.push_back(i);
        g.code.insert(g.code.end(), j.code.begin() + j.code_off[i], j.code.begin() + j.code_off[i + 1]);
        g.kinds.insert(g.kinds.end(), j.kinds.begin() + j.kind_off[i], j.kinds.begin() + j.kind_off[i + 1]);
        g.params.insert(g.params.end(), j.params.begin() + j.param_off[i], j.params.begin() + j.param_off[i + 1]);
        g.code_off.push_back(g.code.size());
        g.kind_off.push_back(g.kinds.size());
        g.param_off.push_back(g.params.size());
        g.dsp.push_back(j.dsp[i]);
    }
    for (int m = 0; m < 3; ++m) {
        Sub &g = sub[m];
        if (g.idx.empty()) continue;
        const rsr_population pop{(uint32_t)g.idx.size(), g.code.data(), g.code_off.data(), g.kinds.data(),
                                 g.kind_off.data(), g.params.data(), g.param_off.data()};
        g.out_params.assign(std::max<size_t>(g.params.size(), 1), 0.0f);
        g.out_mse.assign(g.idx.size(), 0.0f);
        int rc;
        if (m == FIT_LBFGS)  // optimize/mod.rs:50-52: 15 iterations whatever the budget
            rc = fit_population(S->ctx, &pop, g.dsp.data(), 0, 15, slot.st, &S->ctx->mu, &j.cancel, &slot.fit,
                                g.out_params.data(), g.out_mse.data(), nullptr);
        else if (m == FIT_CMAES)  // optimize/mod.rs:53-55
            rc = fit_cma_es(S->ctx, &pop, g.dsp.data(), 0, std::max(j.fit_iterations / 16, 2u), j.seed, slot.st,
                            &S->ctx->mu, &j.cancel, g.out_params.data(), g.out_mse.data(), nullptr);
        else  // optimize/mod.rs:56-57
            rc = fit_nelder_mead(S->ctx, &pop, g.dsp.data(), 0, j.fit_iterations, slot.st, &S->ctx->mu, &j.cancel,
                                 g.out_params.data(), g.out_mse.data(), nullptr);
        if (rc) return rc;
        for (size_t k = 0; k < g.idx.size(); ++k) {
            const uint32_t i = g.idx[k];
            j.mse_out[i] = g.out_mse[k];
            std::copy(g.out_params.begin() + g.param_off[k], g.out_params.begin() + g.param_off[k + 1],
                      j.params_out + j.param_off[i]);
        }
    }
    return RSR_OK;
}

void finish(rsr_server *S, const std::vector<JobPtr> &batch, const std::vector<int> &status,
            const std::vector<std::string> &msgs, uint64_t need) {
    const auto now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (size_t i = 0; i < batch.size(); ++i) {
            Job &j = *batch[i];
            j.status = status[i];
            j.msg = msgs[i];
            j.t_done = now;
            j.state = RSR_JOB_DONE;
            if (j.status == RSR_OK) {
                S->completed++;
                S->lat.push_back(ms_between(j.t_submit, j.t_done));
                S->pp += (double)j.program_points;
            } else if (j.status == RSR_ECANCELED) {
                S->cancelled++;
            } else {
                S->failed++;
            }
        }
        S->t_last = now;
        S->mem_inflight -= need;
    }
    S->cv_done.notify_all();
    S->cv_mem.notify_all();
    unref_datasets(S->ctx, batch);
}

void worker_main(rsr_server *S, Slot *slot) {
    cudaSetDevice(S->ctx->device);
    for (;;) {
        std::vector<JobPtr> batch;
        uint64_t need = 0;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stopping || !S->queue.empty(); });
            if (S->queue.empty()) return;  // stopping
            JobPtr head = S->queue.front();
            S->queue.pop_front();
            batch.push_back(head);
            need = head->est_bytes;
            if (head->kind != RSR_JOB_FIT && head->kind != RSR_JOB_FIT_AUTO) {
                uint64_t progs = head->n();
                while (!S->queue.empty()) {
                    const JobPtr &j = S->queue.front();
                    if (j->kind != head->kind || progs + j->n() > S->opts.max_batch_programs ||
                        need + j->est_bytes > S->budget)
                        break;
                    progs += j->n();
                    need += j->est_bytes;
                    batch.push_back(j);
                    S->queue.pop_front();
                }
            }
            // memory admission: wait for the in-flight footprint to leave room
            S->cv_mem.wait(lk, [&] { return S->mem_inflight + need <= S->budget || S->mem_inflight == 0; });
            S->mem_inflight += need;
            S->mem_peak = std::max(S->mem_peak, S->mem_inflight);
            const auto now = Clock::now();
            for (const JobPtr &j : batch) {
                j->state = RSR_JOB_RUNNING;
                j->t_start = now;
                j->batch_jobs = (uint32_t)batch.size();
            }
            S->launches++;
        }
        std::vector<int> status(batch.size(), RSR_OK);
        std::vector<std::string> msgs(batch.size());
        if (batch[0]->kind == RSR_JOB_FIT_AUTO) {
            Job &j = *batch[0];
            if (j.cancel.load()) {
                status[0] = RSR_ECANCELED;
                msgs[0] = "cancelled";
            } else {
                status[0] = fit_auto(S, *slot, j);
                if (status[0]) msgs[0] = thread_error();
            }
        } else if (batch[0]->kind == RSR_JOB_FIT) {
            Job &j = *batch[0];
            if (j.cancel.load()) {
                status[0] = RSR_ECANCELED;
                msgs[0] = "cancelled";
            } else {
                rsr_population pop = j.pop();
                int rc = fit_population(S->ctx, &pop, j.dsp.data(), 0, j.fit_iterations, slot->st, &S->ctx->mu,
                                        &j.cancel, &slot->fit, j.params_out, j.mse_out, nullptr);
                status[0] = rc;
                if (rc) msgs[0] = thread_error();
            }
        } else {
            int rc = run_eval(S, *slot, batch);
            if (rc && batch.size() > 1) {
                // isolate the failing job(s): run each job of the batch alone
                for (size_t i = 0; i < batch.size(); ++i) {
                    std::vector<JobPtr> one{batch[i]};
                    status[i] = run_eval(S, *slot, one);
                    if (status[i]) msgs[i] = thread_error();
                }
            } else if (rc) {
                status[0] = rc;
                msgs[0] = thread_error();
            }
        }
        // keep at most an even share of the budget cached on this slot
        if (slot->cached() > S->budget / std::max<uint32_t>(1, S->opts.slots)) {
            cudaStreamSynchronize(slot->st);
            slot->trim();
        }
        finish(S, batch, status, msgs, need);
    }
}

}  // namespace
}  // namespace rsr

extern "C" {

void rsr_server_options_default(rsr_server_options *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(*o);
    o->slots = 4;
    o->max_batch_programs = 16384;
    o->max_queue = 65536;
    o->mem_budget_bytes = 0;
}

int rsr_server_create(rsr_ctx *ctx, const rsr_server_options *opts, rsr_server **out) {
    if (!ctx || !out) return fail(RSR_EINVAL, "null argument");
    auto S = std::make_unique<rsr_server>();
    S->ctx = ctx;
    rsr_server_options_default(&S->opts);
    if (opts) memcpy(&S->opts, opts, std::min<size_t>(sizeof(rsr_server_options), opts->struct_size ? opts->struct_size : sizeof(rsr_server_options)));
    S->opts.struct_size = sizeof(rsr_server_options);
    if (S->opts.slots == 0 || S->opts.slots > 64) return fail(RSR_EINVAL, "slots must be 1..64");
    if (S->opts.max_batch_programs == 0) S->opts.max_batch_programs = 16384;
    if (S->opts.max_queue == 0) S->opts.max_queue = 65536;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        const uint64_t free_budget =
            ctx->opts.mem_budget_bytes > ctx->mem_in_use ? ctx->opts.mem_budget_bytes - ctx->mem_in_use : 0;
        S->budget = S->opts.mem_budget_bytes ? S->opts.mem_budget_bytes : free_budget / 2;
        // every kernel a job may use is loaded now rather than on the job's time
        if (const int rc = preload_eval_kernels(ctx)) return rc;
    }
    if (S->budget == 0) return fail(RSR_ENOMEM, "no device memory left for serving");
    cudaSetDevice(ctx->device);
    for (uint32_t i = 0; i < S->opts.slots; ++i) {
        auto sl = std::make_unique<Slot>();
        cudaError_t e = cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking);
        if (e == cudaSuccess) {
            e = cudaStreamCreateWithFlags(&sl->st2, cudaStreamNonBlocking);
            if (e != cudaSuccess) cudaStreamDestroy(sl->st);
        }
        if (e != cudaSuccess) {
            for (auto &s : S->slots) {
                cudaStreamDestroy(s->st);
                cudaStreamDestroy(s->st2);
            }
            return cuda_fail(e, "cudaStreamCreate");
        }
        S->slots.push_back(std::move(sl));
    }
    rsr_server *raw = S.release();
    for (auto &sl : raw->slots) raw->workers.emplace_back(worker_main, raw, sl.get());
    *out = raw;
    return RSR_OK;
}

int rsr_server_destroy(rsr_server *S) {
    if (!S) return RSR_OK;
    std::vector<JobPtr> dropped;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
        for (JobPtr &j : S->queue) {
            j->state = RSR_JOB_DONE;
            j->status = RSR_ECANCELED;
            j->msg = "server shut down";
            S->cancelled++;
            dropped.push_back(j);
        }
        S->queue.clear();
    }
    S->cv_work.notify_all();
    S->cv_done.notify_all();
    for (auto &t : S->workers) t.join();
    if (!dropped.empty()) unref_datasets(S->ctx, dropped);
    cudaSetDevice(S->ctx->device);
    for (auto &sl : S->slots) {
        cudaStreamSynchronize(sl->st);
        cudaStreamSynchronize(sl->st2);
        sl->trim();
        sl->dev.staging.release();
        sl->dev2.staging.release();
        sl->fit.grad.staging.release();
        sl->fit.mse.staging.release();
        sl->host.release();
        cudaStreamDestroy(sl->st);
        cudaStreamDestroy(sl->st2);
    }
    delete S;
    return RSR_OK;
}

int rsr_submit(rsr_server *S, const rsr_job *job, uint64_t *ticket) {
    if (!S || !job || !ticket || !job->pop) return fail(RSR_EINVAL, "null argument");
    const rsr_population &p = *job->pop;
    if (job->kind > RSR_JOB_FIT_AUTO) return fail(RSR_EINVAL, "unknown job kind");
    if (p.n_programs && (!p.code_off || !p.kind_off || !p.param_off)) return fail(RSR_EINVAL, "null population array");
    if (p.n_programs && !job->mse_out) return fail(RSR_EINVAL, "mse_out is null");
    if (job->kind == RSR_JOB_MSE_GRAD && p.n_programs && !job->grad_out) return fail(RSR_EINVAL, "grad_out is null");
    if ((job->kind == RSR_JOB_FIT || job->kind == RSR_JOB_FIT_AUTO) && p.n_programs && !job->params_out)
        return fail(RSR_EINVAL, "params_out is null");
    auto j = std::make_shared<Job>();
    j->kind = job->kind;
    j->fit_iterations = job->fit_iterations;
    const uint32_t n = p.n_programs;
    j->code_off.resize(n + 1);
    j->kind_off.resize(n + 1);
    j->param_off.resize(n + 1);
    j->code_off[0] = j->kind_off[0] = j->param_off[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (p.code_off[i + 1] < p.code_off[i] || p.kind_off[i + 1] < p.kind_off[i] || p.param_off[i + 1] < p.param_off[i])
            return fail(RSR_EINVAL, "population offsets decrease at " + std::to_string(i));
        j->code_off[i + 1] = j->code_off[i] + (p.code_off[i + 1] - p.code_off[i]);
        j->kind_off[i + 1] = j->kind_off[i] + (p.kind_off[i + 1] - p.kind_off[i]);
        j->param_off[i + 1] = j->param_off[i] + (p.param_off[i + 1] - p.param_off[i]);
    }
    if (n) {
        j->code.assign(p.code + p.code_off[0], p.code + p.code_off[n]);
        j->kinds.assign(p.const_kinds + p.kind_off[0], p.const_kinds + p.kind_off[n]);
        j->params.assign(p.params + p.param_off[0], p.params + p.param_off[n]);
    }
    j->dsp.resize(n);
    for (uint32_t i = 0; i < n; ++i) j->dsp[i] = job->ds_per_program ? job->ds_per_program[i] : job->ds;
    j->mse_out = job->mse_out;
    j->grad_out = job->grad_out;
    j->params_out = job->params_out;
    j->seed = job->seed;
    // datasets: resolve, size the job, and hold a reference until it is done
    std::vector<uint64_t> n_eval(n, 0);
    {
        std::lock_guard<std::mutex> lk(S->ctx->mu);
        std::unordered_map<uint64_t, uint64_t> seen;
        for (uint32_t i = 0; i < n; ++i) {
            auto f = seen.find(j->dsp[i]);
            if (f == seen.end()) {
                auto it = S->ctx->datasets.find(j->dsp[i]);
                if (it == S->ctx->datasets.end())
                    return fail(RSR_ENOTFOUND, "unknown dataset handle " + std::to_string(j->dsp[i]));
                f = seen.emplace(j->dsp[i], it->second->num_batches * 8).first;
            }
            n_eval[i] = f->second;
            j->program_points += S->ctx->datasets.find(j->dsp[i])->second->num_samples;
        }
        j->est_bytes = estimate_bytes(*j, n_eval);
        if (j->est_bytes > S->budget) {
            std::lock_guard<std::mutex> lk2(S->mu);
            S->refused++;
            return fail(RSR_ENOMEM, "job needs about " + std::to_string(j->est_bytes >> 20) +
                                        " MiB of device memory, above the serving budget");
        }
        for (auto &kv : seen) {
            S->ctx->datasets.find(kv.first)->second->refs++;
            j->handles.push_back(kv.first);
        }
    }
    int refused = RSR_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping || S->queue.size() >= S->opts.max_queue) {
            S->refused++;
            refused = S->stopping ? RSR_ECANCELED : RSR_EBUSY;
        } else {
            j->ticket = S->next_ticket++;
            j->t_submit = Clock::now();
            if (!S->have_t0) {
                S->t0 = j->t_submit;
                S->have_t0 = true;
            }
            S->submitted++;
            S->jobs.emplace(j->ticket, j);
            S->queue.push_back(j);
            *ticket = j->ticket;
        }
    }
    if (refused) {
        unref_datasets(S->ctx, {j});
        return fail(refused, refused == RSR_ECANCELED ? "server shut down" : "queue full");
    }
    S->cv_work.notify_one();
    return RSR_OK;
}

int rsr_poll(rsr_server *S, uint64_t ticket, uint32_t *state) {
    if (!S || !state) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return fail(RSR_ENOTFOUND, "unknown ticket");
    *state = it->second->state;
    return RSR_OK;
}

int rsr_wait(rsr_server *S, uint64_t ticket, uint64_t timeout_us, rsr_job_info *info) {
    if (!S) return fail(RSR_EINVAL, "null argument");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return fail(RSR_ENOTFOUND, "unknown ticket");
    JobPtr j = it->second;
    auto done = [&] { return j->state == RSR_JOB_DONE; };
    if (timeout_us == 0) S->cv_done.wait(lk, done);
    else if (!S->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), done))
        return fail(RSR_ETIMEDOUT, "job still running");
    if (info) {
        info->status = j->status;
        info->batch_jobs = j->batch_jobs;
        info->queue_ms = j->batch_jobs ? ms_between(j->t_submit, j->t_start) : ms_between(j->t_submit, j->t_done);
        info->latency_ms = ms_between(j->t_submit, j->t_done);
    }
    S->jobs.erase(ticket);
    if (j->status != RSR_OK) return fail(j->status, j->msg);
    return RSR_OK;
}

int rsr_cancel(rsr_server *S, uint64_t ticket) {
    if (!S) return fail(RSR_EINVAL, "null argument");
    JobPtr dropped;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->jobs.find(ticket);
        if (it == S->jobs.end()) return fail(RSR_ENOTFOUND, "unknown ticket");
        JobPtr j = it->second;
        j->cancel.store(true);
        if (j->state == RSR_JOB_QUEUED) {
            auto q = std::find(S->queue.begin(), S->queue.end(), j);
            if (q != S->queue.end()) S->queue.erase(q);
            j->state = RSR_JOB_DONE;
            j->status = RSR_ECANCELED;
            j->msg = "cancelled";
            j->t_done = Clock::now();
            S->cancelled++;
            dropped = j;
        }
    }
    S->cv_done.notify_all();
    if (dropped) unref_datasets(S->ctx, {dropped});
    return RSR_OK;
}

int rsr_server_stats(rsr_server *S, rsr_serving_stats *st, int reset) {
    if (!S || !st) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->failed = S->failed;
    st->cancelled = S->cancelled;
    st->refused = S->refused;
    st->launches = S->launches;
    st->peak_mem_bytes = S->mem_peak;
    if (!S->lat.empty()) {
        std::vector<double> v = S->lat;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) {
            const double r = q * (double)(v.size() - 1);
            const size_t lo = (size_t)std::floor(r), hi = std::min(v.size() - 1, lo + 1);
            return v[lo] + (v[hi] - v[lo]) * (r - (double)lo);
        };
        st->p50_ms = pct(0.50);
        st->p95_ms = pct(0.95);
        st->p99_ms = pct(0.99);
        st->max_ms = v.back();
        double s = 0.0;
        for (double x : v) s += x;
        st->mean_ms = s / (double)v.size();
    }
    if (S->have_t0) {
        st->wall_s = std::max(0.0, ms_between(S->t0, S->t_last) / 1000.0);
        st->program_points_per_sec = st->wall_s > 0 ? S->pp / st->wall_s : 0.0;
    }
    if (reset) {
        S->submitted = S->completed = S->failed = S->cancelled = S->refused = S->launches = 0;
        S->lat.clear();
        S->pp = 0.0;
        S->have_t0 = false;
        S->mem_peak = S->mem_inflight;
    }
    return RSR_OK;
}

}  // extern "C"
