// runtime.h -- host-side engine state behind the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <functional>
#include <thread>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/rsr_gpu.h"
#include "encoder.h"
#include "kernels.h"
#include "uops.h"

namespace rsr {

// A fixed set of host threads for data-parallel host work (program
// encoding): run(n, f) calls f(0..n-1) across the threads and returns when
// all calls are done.  One caller at a time (build_plan runs under the
// context's lock).
class TaskPool {
  public:
    explicit TaskPool(unsigned threads);
    ~TaskPool();
    unsigned size() const { return (unsigned)threads_.size() + 1; }
    void run(uint32_t n, const std::function<void(uint32_t)> &f);

  private:
    void work();
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(uint32_t)> *task_ = nullptr;
    uint32_t n_ = 0;
    std::atomic<uint32_t> next_{0};
    size_t finished_ = 0;
    uint64_t epoch_ = 0;
    bool stop_ = false;
};

// NVTX range for profiler timelines (a no-op unless a profiler is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

// Grow-only device allocation.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t bytes);
    void release();
    ~DevBuf() { release(); }
};

// Pinned host staging buffer.
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t bytes);
    void release();
    ~HostBuf() { release(); }
};

struct DatasetRec {
    float *x = nullptr;   // features, SoA, stride points per feature
    float *y = nullptr;
    uint32_t num_features = 0;
    uint64_t num_batches = 0, num_samples = 0, stride = 0;
    size_t bytes = 0;
    std::atomic<int> refs{0};  // prepared batches and in-flight jobs holding it
    DatasetDesc desc() const {
        DatasetDesc d{};
        d.x = x; d.y = y; d.stride = stride; d.n_eval = num_batches * 8; d.num_samples = num_samples;
        d.num_features = num_features;
        return d;
    }
};

// Tuned launch shape for one (kernel profile, dataset size class).
struct TuneChoice {
    int P = 0;
    int G = 0;
};

// One kernel launch inside a plan.
struct Group {
    int kind = 0;        // 0 plain, 1 register, 2 slot-file adjoint, 3 register adjoint
    int profile = -1;
    unsigned omit = 0;      // register kernel: handler sets its programs do not need (launch_reg)
    bool no_unary = false;  // adjoint kernel: no unary Float op in the launch's programs
    int P = 4;
    int G = 1;
    uint32_t item_begin = 0, n_items = 0;  // into the plan's item array
    uint32_t code_words = 0, const_floats = 0, slots = 0;  // per-warp staging maxima
    uint32_t adj_slots = 0;                                  // adjoint kernel: adjoint slots
    uint32_t parts = 1;   // register adjoint: about this many parts (kPartPoints points) an item, at most one more
    uint32_t stack_depth[N_STACKS] = {0, 0, 0, 0, 0};       // register kernel: spill slots per type
    // launch shape of the last enqueue (filled in by enqueue_plan)
    mutable uint32_t grid = 0;
    mutable size_t smem = 0;
    mutable uint32_t warps_per_block = 0;
    mutable uint32_t tmem_cols = 0;     // register adjoint: tensor-memory columns of a warp's tape
    uint64_t flops = 0;           // algorithmic FP32 lane-ops of one run
    uint64_t program_points = 0;
    uint64_t item_work = 0;       // code length x tiles of the group's longest item
};

// A population encoded and laid out for the device: what one launch of the
// engine needs besides the datasets.
struct Plan {
    std::vector<ProgDesc> progs;            // launch order
    std::vector<uint32_t> orig;             // launch index -> caller index
    std::vector<DatasetDesc> datasets;      // launch dataset table
    std::vector<uint64_t> ds_handles;
    std::vector<WorkItem> items;
    std::vector<uint32_t> code;
    std::vector<float> consts;
    std::vector<Group> groups;
    uint32_t n_partials = 0;                // doubles (gradient: 33 per slot)
    bool gradient = false;
    bool raw_sums = false;                  // MODE_MSE: unscaled f64 sums instead of the epilogue
    int mode = MODE_MSE;
    uint64_t points_stride = 0;
    uint64_t flops = 0;                     // algorithmic lane-ops of one run
    uint64_t program_points = 0;
    uint32_t n_plain = 0, n_reg = 0;

    // Empty, with the vectors' capacity kept for the next build.
    void reset() {
        Plan keep = std::move(*this);
        *this = Plan();
        progs = std::move(keep.progs); progs.clear();
        orig = std::move(keep.orig); orig.clear();
        datasets = std::move(keep.datasets); datasets.clear();
        ds_handles = std::move(keep.ds_handles); ds_handles.clear();
        items = std::move(keep.items); items.clear();
        code = std::move(keep.code); code.clear();
        consts = std::move(keep.consts); consts.clear();
        groups = std::move(keep.groups); groups.clear();
    }
};

// Device copy of a plan plus the buffers one run writes.
struct DevicePlan {
    DevBuf pool;        // progs | datasets | items | code | consts
    DevBuf partials;
    DevBuf out;         // mse (n floats) [+ grad (n*32 floats)]
    DevBuf counters;    // one item counter per group
    DevBuf status;
    HostBuf staging;    // pinned image of the pool, uploaded with one copy
    cudaEvent_t staged = nullptr;  // recorded after the staging buffer's copy
    // Every launch of a plan but the first goes to one of two side streams,
    // forked from and joined back into the caller's stream, so that a
    // launch's blocks take the SMs that the previous launch's last blocks free.
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    LaunchArgs base{};
    float *mse = nullptr, *grad = nullptr;
    DevicePlan() = default;
    DevicePlan(const DevicePlan &) = delete;
    DevicePlan &operator=(const DevicePlan &) = delete;
    ~DevicePlan() {
        if (staged) cudaEventDestroy(staged);
        if (fork) cudaEventDestroy(fork);
        for (int i = 0; i < 2; ++i) {
            if (join[i]) cudaEventDestroy(join[i]);
            if (side[i]) cudaStreamDestroy(side[i]);
        }
    }
};

}  // namespace rsr

struct rsr_ctx {
    int device = 0;
    int num_sms = 0;
    size_t smem_per_sm = 0;    // shared memory of an SM (bytes)
    size_t smem_reserved = 0;  // shared memory the system reserves per block
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // odd chunks of a chunked one-shot call
    rsr_options opts{};
    std::mutex mu;
    std::map<uint64_t, std::unique_ptr<rsr::DatasetRec>> datasets;
    uint64_t next_handle = 1;
    uint64_t mem_in_use = 0;
    std::map<std::pair<int, int>, rsr::TuneChoice> tune;  // (profile, log2 points) -> choice
    rsr::TuneChoice force;     // set while the autotuner measures a candidate
    rsr::DevicePlan scratch;   // for one-shot calls
    rsr::DevicePlan pipe[2];   // one-shot calls split into chunks, alternating
    rsr::HostBuf results;      // pinned results of a chunked one-shot call
    std::unique_ptr<rsr::TaskPool> encoders;  // host threads for program encoding
    // Kept between calls so that encoding and planning a population of a
    // size seen before allocates nothing new: one encoding per program of
    // the largest population so far, and the plans of one-shot calls.
    std::vector<rsr::EncodedProgram> enc_cache;
    std::vector<int> enc_rc;
    std::vector<std::string> enc_msg;
    std::vector<rsr::Plan> call_plans;
    void *l2buf = nullptr;
    size_t l2bytes = 0;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    std::atomic<uint64_t> launches{0};
    std::atomic<uint64_t> last_h2d{0}, last_d2h{0};   // bytes copied by the last evaluation call
    bool kernels_loaded = false;  // preload_eval_kernels has run
};

struct rsr_batch {
    rsr::Plan plan;
    rsr::DevicePlan dev;
    cudaGraphExec_t graph = nullptr;
    bool graph_ready = false;
    float eval_ms = 0.0f, total_ms = 0.0f;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    std::vector<cudaEvent_t> gev;          // per-group kernel events (runs without graphs)
    std::vector<float> group_ms;
    uint64_t pool_bytes = 0;
};

namespace rsr {
// Encoding storage and threads of one planner: a caller that plans with its
// own (a serving slot) needs the context's lock only for the dataset and
// tuning tables, not for the encoding.
struct EncodeScratch {
    std::vector<EncodedProgram> enc;
    std::vector<int> rc;
    std::vector<std::string> msg;
    std::unique_ptr<TaskPool> pool;
    unsigned threads = 16;  // capped by the host's hardware threads
};
// Planning and execution (runtime.cu), shared with the serving loop.
// scratch == nullptr: the context's own encoding storage and threads (the
// caller holds ctx->mu).  With scratch, table_mu (ctx->mu) is taken only
// around the reads of the context's dataset and tuning tables.
int build_plan(rsr_ctx *ctx, const rsr_population &pop, const uint64_t *ds_per_prog, uint64_t ds_all, int kernel,
               bool gradient, int mode, Plan *plan, EncodeScratch *scratch = nullptr, std::mutex *table_mu = nullptr);
int upload_plan(rsr_ctx *ctx, const Plan &plan, DevicePlan *dev, cudaStream_t st);
// Loads every evaluation kernel instance once per context (caller holds
// ctx->mu), so that no later call pays for a kernel's first launch.
int preload_eval_kernels(rsr_ctx *ctx);
// A zero-filled resident dataset of the given shape (columns padded to the
// stride), and its registration in the context's table (caller holds ctx->mu).
int alloc_dataset(rsr_ctx *ctx, uint32_t nf, uint64_t nbatch, uint64_t nsamples, std::unique_ptr<DatasetRec> *out);
rsr_dataset register_dataset(rsr_ctx *ctx, std::unique_ptr<DatasetRec> rec);
// Batched L-BFGS (lbfgs.cu) on stream st.  plan_mu, when given, is held while
// plans are built (they read the context's dataset and tuning tables);
// cancel, when set, stops the fit between iterations with RSR_ECANCELED.
// ws, when given, supplies (and keeps) the device buffers of the fit.
struct FitWorkspace {
    DevicePlan grad, mse;
    DevBuf grad_active, mse_active;
    DevBuf lbfgs_state;   // device-resident L-BFGS state of every program (lbfgs.cu)
    HostBuf lbfgs_counts; // pinned copy of the per-iteration counters
};
int fit_population(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds,
                   uint32_t max_iterations, cudaStream_t stream, std::mutex *plan_mu,
                   const std::atomic<bool> *cancel, FitWorkspace *ws, float *params_out, float *mse_out,
                   rsr_fit_stats *stats);
// Batched Nelder-Mead and CMA-ES (nelder_mead.cu, cma_es.cu); plan_mu and
// cancel as for fit_population.
int fit_nelder_mead(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds,
                    uint32_t max_iterations, cudaStream_t stream, std::mutex *plan_mu,
                    const std::atomic<bool> *cancel, float *params_out, float *mse_out, rsr_fit_stats *stats);
int fit_cma_es(rsr_ctx *ctx, const rsr_population *pop, const uint64_t *dsp, uint64_t ds, uint32_t max_iterations,
               uint64_t seed, cudaStream_t stream, std::mutex *plan_mu, const std::atomic<bool> *cancel,
               float *params_out, float *mse_out, rsr_fit_stats *stats);
// group_events: optional, 2 per group (before/after its kernel); not used
// while capturing a graph.
int enqueue_plan(rsr_ctx *ctx, const Plan &plan, DevicePlan *dev, cudaStream_t st, cudaEvent_t ev_mid,
                 cudaEvent_t *group_events = nullptr);
// The no-allocation entry point's fixed-array slot encoder (noalloc.cu), for
// diagnostics; words must hold noalloc_max_words() words.
int noalloc_slot_form(const rsr_program &p, uint32_t num_features, uint32_t *words, uint32_t *n_words,
                      uint32_t *n_slots, uint32_t *flags, const char **err);
uint32_t noalloc_max_words();
}  // namespace rsr
