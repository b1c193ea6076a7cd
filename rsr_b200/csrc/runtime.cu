// runtime.cu -- contexts, resident datasets, launch planning and the C ABI
// entry points of include/rsr_gpu.h.
#include <cuda_runtime.h>
#include <float.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <thread>
#include <unordered_map>
#include <numeric>

#include "runtime.h"

namespace rsr {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }
int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    return fail(e == cudaErrorMemoryAllocation ? RSR_ENOMEM : RSR_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

// Growth is geometric below 64 MB (at least 1.5x the old capacity): a buffer
// reused by calls of slowly growing size is reallocated a few times, not at
// every call, and each cudaFree of the old buffer synchronises the device.
static size_t grow_to(size_t bytes, size_t cap, size_t floor) {
    size_t want = std::max(bytes, floor);
    if (cap && want < ((size_t)64 << 20)) want = std::max(want, std::min(cap + cap / 2, (size_t)64 << 20));
    return want;
}

cudaError_t DevBuf::reserve(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = grow_to(bytes, cap, 256);
    release();
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

cudaError_t HostBuf::reserve(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = grow_to(bytes, cap, (size_t)1 << 20);
    release();
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        return e;
    }
    cap = want;
    return cudaSuccess;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

TaskPool::TaskPool(unsigned threads) {
    for (unsigned i = 1; i < threads; ++i) threads_.emplace_back([this] { work(); });
}

TaskPool::~TaskPool() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : threads_) t.join();
}

void TaskPool::work() {
    uint64_t seen = 0;
    for (;;) {
        const std::function<void(uint32_t)> *f;
        uint32_t n;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || epoch_ != seen; });
            if (stop_) return;
            seen = epoch_;
            f = task_;
            n = n_;
        }
        for (uint32_t i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) (*f)(i);
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (++finished_ == threads_.size()) done_cv_.notify_all();
        }
    }
}

void TaskPool::run(uint32_t n, const std::function<void(uint32_t)> &f) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        task_ = &f;
        n_ = n;
        next_.store(0);
        finished_ = 0;
        ++epoch_;
    }
    cv_.notify_all();
    for (uint32_t i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) f(i);
    // every worker takes part in every run and has left it before the next
    // one starts, so none can pick up this run's task or counter late
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return finished_ == threads_.size(); });
}

// register path = profile + 8 * (spill-depth class + 3 * omitted-handler mask)
static constexpr int kRegPathStride = 8;
// Tape shared memory per warp that the adjoint's points per lane aim for.
// More points per lane amortise the dispatch over more work at the cost of
// fewer resident tapes per SM.  Gradient of 256 programs x 1M points (matrix
// workload): 28.8 ms at 40 KB against 33.2 ms at 27 KB and 43 ms at 14 KB.
// Uneven workload (2048 programs, 16 datasets), whose longest tapes need
// more than 40 KB at 4 points per lane: 49.7 ms at 80 KB against 52.6 ms at
// 40 KB and 81.6 ms at 20 KB; the vector and matrix workloads' tapes fit
// 40 KB at 4 points and do not change.
static constexpr size_t kGradTapeBudget = 80 * 1024;
// Register adjoint: shared memory the warps' stacks (which the adjoint
// stacks reuse) and gradient sums may take in a block (one block per SM,
// the rest of the 227 KB for code, constants and sums), and the first path
// number of its launches in a gradient plan.
static constexpr size_t kAdjRegionBudget = 200 * 1024;
static constexpr int kAdjPathBase = 0;
// Points per work-item chunk (all P).  8192 measured slower on every kernel
// (vector register 4.32 ms against 4.30, matrix register 4.84 against 4.69,
// vector adjoint 6.68 against 5.90): coarser items balance worse.
static constexpr uint64_t kChunkPoints = kPartPoints;
// Work items of the register adjoint cover several parts: its block is the
// SM's only one, and between items the SM waits for the next item's code
// and for the item's cross-warp sums.  A launch takes the most parts an
// item (about 4, 2 or 1) that still leave it kAdjItemsPerSm items an SM, so
// that a small batch keeps short items and its launch does not end on a few
// long ones, and whose cross-warp sums fit the block's shared memory.  A
// dataset's parts are spread evenly over floor(parts / k) items of at most
// k + 1 parts (25 parts: one item of 5 and five of 4), so that no item is a
// few tiles on an otherwise idle block.  The kernel sums every part on its
// own, so the sums do not depend on the items.
static constexpr uint64_t kAdjItemsPerSm = 8;

// Items a dataset of n_parts parts is cut into, at about k parts an item
// and at most k + 1 (k = 1: one part an item).
static uint64_t adj_items(uint64_t n_parts, uint32_t k) {
    if (k <= 1) return n_parts;
    return std::max<uint64_t>({1, n_parts / k, (n_parts + k) / (k + 1)});
}
// Points per lane of a register-adjoint path (its launch's P).
static int adj_path_p(int pth) { return 2 << (((pth - kAdjPathBase) / N_PROFILES) % 3); }
static constexpr uint64_t kStrideAlign = 1024;   // dataset column padding
static constexpr int kGradSlotDoubles = 33;      // sse + 32 gradient sums

static uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }
static int log2_bucket(uint64_t n) {
    int b = 0;
    while ((1ull << (b + 1)) <= n) ++b;
    return b;
}

// Default launch shape of the register kernel per profile: points per
// thread and programs per warp.  F+V3 on 64k points or more takes the shape
// the autotuner picks for the 100k-point vector workload (8 points per lane,
// 4 programs per item: 4.28 ms against 4.56 ms at 4 and 2).
static TuneChoice default_choice(int profile, uint64_t n_eval) {
    switch (profile) {
        case P_F: return {8, 4};
        case P_FV3: return n_eval >= 65536 ? TuneChoice{8, 4} : TuneChoice{4, 2};
        default: return {4, 4};
    }
}

static TuneChoice choice_for(rsr_ctx *ctx, int profile, uint64_t n_eval) {
    TuneChoice c = default_choice(profile, n_eval);
    auto it = ctx->tune.find({profile, log2_bucket(n_eval)});
    if (it != ctx->tune.end()) c = it->second;
    if (ctx->opts.points_per_thread > 0) c.P = ctx->opts.points_per_thread;
    if (ctx->opts.programs_per_warp > 0) c.G = ctx->opts.programs_per_warp;
    if (ctx->force.P > 0) c = ctx->force;
    // variants that exist (kernels_reg.cu): P in {2, 4, 8} up to reg_max_p
    const int maxP = reg_max_p(profile);
    if (c.P > maxP) c.P = maxP;
    if (c.P != 2 && c.P != 4 && c.P != 8) c.P = c.P < 2 ? 2 : 4;
    c.G = std::max(1, std::min(c.G, 8));
    return c;
}

int build_plan(rsr_ctx *ctx, const rsr_population &pop, const uint64_t *ds_per_prog, uint64_t ds_all, int kernel,
               bool gradient, int mode, Plan *plan, EncodeScratch *scratch, std::mutex *table_mu) {
    NvtxRange nvtx_range("rsr: encode + plan");
    Plan &P = *plan;
    P.reset();
    P.gradient = gradient;
    P.mode = mode;
    const uint32_t n = pop.n_programs;
    if (n == 0) return RSR_OK;
    if (!pop.code_off || !pop.kind_off || !pop.param_off) return fail(RSR_EINVAL, "population offsets are null");
    // The first gradient plan of a context loads every kernel instance (the
    // caller holds ctx->mu here), ~40 ms: a 20-iteration fit of the matrix
    // workload whose adjoint instances were first launched from its
    // captured iteration took 0.95 s, 0.22 s once they had been launched.
    if (gradient && !scratch && !ctx->kernels_loaded) {
        const int rc = preload_eval_kernels(ctx);
        if (rc) return rc;
    }
    // datasets
    std::map<uint64_t, uint32_t> ds_index;
    std::vector<uint32_t> prog_ds(n);
    std::unique_lock<std::mutex> table_lock;
    if (table_mu) table_lock = std::unique_lock<std::mutex>(*table_mu);
    for (uint32_t i = 0; i < n; ++i) {
        uint64_t h = ds_per_prog ? ds_per_prog[i] : ds_all;
        auto f = ds_index.find(h);
        if (f == ds_index.end()) {
            auto it = ctx->datasets.find(h);
            if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle " + std::to_string(h));
            uint32_t idx = (uint32_t)P.datasets.size();
            P.datasets.push_back(it->second->desc());
            P.ds_handles.push_back(h);
            f = ds_index.emplace(h, idx).first;
        }
        prog_ds[i] = f->second;
    }
    if (table_lock.owns_lock()) table_lock.unlock();
    // encode: each program only in the form its kernel needs, in parallel
    // for large populations
    for (uint32_t i = 0; i < n; ++i)
        if (pop.code_off[i + 1] < pop.code_off[i] || pop.kind_off[i + 1] < pop.kind_off[i] ||
            pop.param_off[i + 1] < pop.param_off[i])
            return fail(RSR_EINVAL, "population offsets decrease at " + std::to_string(i));
    const bool fuse = (ctx->opts.flags & RSR_OPT_NO_LOAD_FUSION) == 0;
    const unsigned forms = gradient ? (FORM_TAPE | FORM_ADJ) : kernel == RSR_KERNEL_PLAIN ? FORM_SLOT : FORM_ACC;
    std::vector<EncodedProgram> &enc = scratch ? scratch->enc : ctx->enc_cache;
    std::vector<int> &erc = scratch ? scratch->rc : ctx->enc_rc;
    std::vector<std::string> &emsg = scratch ? scratch->msg : ctx->enc_msg;
    if (enc.size() < n) {
        enc.resize(n);
        erc.resize(n);
        emsg.resize(n);
    }
    auto encode_one = [&](uint32_t i, unsigned f) {
        const uint64_t c0 = pop.code_off[i], k0 = pop.kind_off[i], p0 = pop.param_off[i];
        erc[i] = encode_program(pop.code + c0, (uint32_t)(pop.code_off[i + 1] - c0), pop.const_kinds + k0,
                                (uint32_t)(pop.kind_off[i + 1] - k0), pop.params + p0,
                                (uint32_t)(pop.param_off[i + 1] - p0), P.datasets[prog_ds[i]].num_features, &enc[i],
                                &emsg[i], fuse, f);
    };
    if (n >= 64) {  // a program takes ~2 us to encode; a pool run costs ~10 us
        std::unique_ptr<TaskPool> &pool = scratch ? scratch->pool : ctx->encoders;
        if (!pool)
            pool = std::make_unique<TaskPool>(std::max(
                1u, std::min(scratch ? scratch->threads : 16u, std::thread::hardware_concurrency())));
        // programs in blocks of 16 per task
        const uint32_t nb = (n + 15) / 16;
        pool->run(nb, [&](uint32_t b) {
            for (uint32_t i = b * 16; i < std::min(n, b * 16 + 16); ++i) encode_one(i, forms);
        });
    } else {
        for (uint32_t i = 0; i < n; ++i) encode_one(i, forms);
    }
    for (uint32_t i = 0; i < n; ++i)
        if (erc[i] != RSR_OK) return fail(erc[i], "program " + std::to_string(i) + ": " + emsg[i]);
    // path per program: <= -2 slot-file adjoint, -1 plain, >= 0 register
    // profile (MSE plans) or register adjoint (gradient plans)
    std::vector<int> path(n);
    std::vector<uint8_t> adj_omit(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        if (gradient && enc[i].adj_profile >= 0 && adj_supported(enc[i].adj_profile) &&
            !(ctx->opts.flags & RSR_OPT_SLOT_ADJOINT)) {
            // register adjoint: the most points per lane (8, 4, 2) whose tape
            // fits a warp's share of the SM's tensor memory (512 columns / (warps
            // / 4), P columns a slot) and whose stacks and sums fit the block's
            // shared memory; launches by points per lane and profile
            const EncodedProgram &E = enc[i];
            uint32_t depth[N_STACKS];
            for (int t = 0; t < N_STACKS; ++t) depth[t] = (uint32_t)E.adj_depth[t];
            const uint32_t np = (uint32_t)E.consts.size();
            int pc = adj_max_p(E.adj_profile) >= 8 ? 2 : 1;  // points per lane 2 << pc
            for (; pc >= 0; --pc) {
                const int P = 2 << pc, nw = adj_block_warps(E.adj_profile, P);
                const uint32_t cols = 512u / (uint32_t)(nw / 4);
                if (E.adj_tape * (uint32_t)P <= cols &&
                    (size_t)adj_warp_floats(depth, P, np) * 4u * (size_t)nw <= kAdjRegionBudget)
                    break;
            }
            if (pc >= 0) {
                const int bucket = 0;
                // the handler sets the program does not use (forward entries:
                // two words each after the header words); a launch leaves out
                // those none of its programs uses
                const uint32_t mv = (uint32_t)(K_V3 + kv_mulm(kBinOps[SV3], 3));
                unsigned omit = adj_omittable(E.adj_profile);
                const uint32_t n_fwd = E.adj_code.empty() ? 0u : E.adj_code[0];
                for (uint32_t q = 0; q < n_fwd; ++q) {
                    const uint32_t kind = E.adj_code[kAdjHeaderWords + 2 * q] & 0xFFu;
                    if (kind >= (uint32_t)K_F_UN && kind < (uint32_t)K_F_END) omit &= ~1u;
                    if (kind >= mv + 1 && kind <= mv + 3) omit &= ~2u;
                }
                adj_omit[i] = (uint8_t)omit;
                path[i] = kAdjPathBase + ((bucket * 3 + pc) * N_PROFILES + E.adj_profile);
                continue;
            }
        }
        if (gradient) {
            // adjoint launches by tape size, so that a block's shared memory
            // follows its own programs' tapes: steps of 16 slots up to 256,
            // then <= 512 and more (a launch sizes every warp's tape for its
            // largest program, and a finer step packs more tapes per SM)
            const uint32_t nt = enc[i].n_tape_val + enc[i].n_tape_adj;
            const int bucket = nt <= 256 ? (int)((nt + 15) / 16) : nt <= 512 ? 17 : 18;
            // Points per lane: the most (4, 2, 1) whose tape fits
            // kGradTapeBudget, decided from the program alone, so that its
            // sums do not depend on the other programs of the call.
            int lp = 2;
            while (lp > 0 && grad_smem_per_warp((uint32_t)enc[i].tape_code.size() + 1, (uint32_t)enc[i].consts.size(),
                                                enc[i].n_tape_val, enc[i].n_tape_adj, 1 << lp) > kGradTapeBudget)
                --lp;
            // programs without a unary Float op run on a kernel built without
            // those handlers (F and F+V3 profiles)
            bool nu = grad_has_no_unary(enc[i].tape_profile);
            const std::vector<uint32_t> &tc = enc[i].tape_code;
            for (size_t w = 2; w + 5 <= tc.size(); w += 5) {
                const uint32_t op = tc[w] & 0xFFu;
                if (op >= (uint32_t)SIN_F && op <= (uint32_t)LN_F) nu = false;
            }
            // one launch per (tape-size bucket, points per lane, no-unary
            // flag, kernel profile)
            path[i] = -2 - (((bucket * 3 + lp) * 2 + (nu ? 1 : 0)) * N_PROFILES + enc[i].tape_profile);
        }
        else if (kernel == RSR_KERNEL_PLAIN || enc[i].profile < 0) path[i] = -1;
        else {
            // the register kernel's spill stacks for 2 points per lane must fit
            // one block next to the program's own code and constants
            uint32_t depth[N_STACKS];
            for (int t = 0; t < N_STACKS; ++t) depth[t] = (uint32_t)enc[i].depth_fast[t];
            const uint32_t cw = (uint32_t)enc[i].reg_code.size() + 1, cf = (uint32_t)enc[i].consts.size();
            if (reg_smem_bytes(cw, cf, depth, 2, 1) > kRegSmemBudget / 2) {
                path[i] = -1;
            } else {
                // launches by spill depth, so that shallow programs (most of
                // a random population) run with small spill stacks and leave
                // the SM's unified L1 to their feature loads
                uint32_t dmax = 0;
                for (int t = 0; t < N_STACKS; ++t) dmax = std::max(dmax, depth[t]);
                const int cls = dmax <= 1 ? 0 : dmax <= 2 ? 1 : 2;
                // and apart by the handler sets the program does not use
                // (unary Float ops; mat-vec with a leaf or spilled matrix),
                // whose kernels are built without them: smaller kernels,
                // fewer instruction-cache misses
                const uint32_t mv = (uint32_t)(K_V3 + kv_mulm(kBinOps[SV3], 3));
                unsigned omit = reg_omittable(enc[i].profile);
                for (uint32_t w : enc[i].reg_code) {
                    const uint32_t kind = w & 0xFFu;
                    if (kind >= (uint32_t)K_F_UN && kind < (uint32_t)K_F_END) omit &= ~1u;
                    if (kind >= mv + 1 && kind <= mv + 3) omit &= ~2u;
                }
                path[i] = enc[i].profile + kRegPathStride * (cls + 3 * (int)omit);
            }
        }
        // programs the register kernel cannot take run on the slot-file kernel
        if (path[i] == -1 && !(forms & FORM_SLOT)) {
            encode_one(i, FORM_SLOT);
            if (erc[i] != RSR_OK) return fail(erc[i], "program " + std::to_string(i) + ": " + emsg[i]);
        }
    }
    // group programs by (path, dataset), each group sorted by descending code length
    // (one 64-bit key per program: path, dataset, then longer code first and
    // the caller's order among equals, as a stable sort by those would give)
    std::vector<uint32_t> order(n);
    {
        std::vector<std::pair<uint64_t, uint32_t>> keyed(n);
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t len = enc[i].reg_code.size() + enc[i].slot_code.size();
            const uint64_t key = ((uint64_t)(uint32_t)(path[i] + (1 << 20)) << 42) | ((uint64_t)prog_ds[i] << 22) |
                                 ((1ull << 22) - 1 - std::min<uint64_t>(len, (1ull << 22) - 1));
            keyed[i] = {key, i};
        }
        std::sort(keyed.begin(), keyed.end());
        for (uint32_t i = 0; i < n; ++i) order[i] = keyed[i].second;
    }
    P.progs.resize(n);
    P.orig = order;
    {
        size_t cw = 0, cf = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const EncodedProgram &E = enc[i];
            cw += path[i] <= -2 ? E.tape_code.size() : path[i] == -1 ? E.slot_code.size()
                : gradient ? E.adj_code.size() : E.reg_code.size();
            cf += E.consts.size();
        }
        P.code.reserve(cw);
        P.consts.reserve(cf);
    }
    uint32_t part = 0;
    for (uint32_t li = 0; li < n; ++li) {
        const uint32_t i = order[li];
        const EncodedProgram &E = enc[i];
        const std::vector<uint32_t> &code = path[i] <= -2 ? E.tape_code : path[i] == -1 ? E.slot_code
                                            : gradient ? E.adj_code : E.reg_code;
        ProgDesc d{};
        d.uop_off = (uint32_t)P.code.size();
        d.uop_len = (uint32_t)code.size();
        d.const_off = (uint32_t)P.consts.size();
        d.n_consts = (uint32_t)E.consts.size();
        const bool reg_adj = gradient && path[i] >= 0;
        d.n_slots = reg_adj ? E.adj_tape : E.n_slots;
        d.flags = (E.result_zero ? PF_RESULT_ZERO : 0u) | (E.needs_zero_init ? PF_NEEDS_ZERO_INIT : 0u) |
                  (E.differentiable ? PF_DIFFERENTIABLE : 0u);
        d.dataset = prog_ds[i];
        const uint64_t n_eval = P.datasets[d.dataset].n_eval;
        d.n_parts = (uint32_t)std::max<uint64_t>(1, (n_eval + kChunkPoints - 1) / kChunkPoints);
        d.part_off = part;
        if (reg_adj) {
            uint32_t depth[N_STACKS];
            for (int t = 0; t < N_STACKS; ++t) depth[t] = (uint32_t)E.adj_depth[t];
            d.n_tape = adj_pack_depth(depth);
        } else {
            d.n_tape = E.n_tape_val | (E.n_tape_adj << 16);
        }
        part += d.n_parts;
        P.code.insert(P.code.end(), code.begin(), code.end());
        P.consts.insert(P.consts.end(), E.consts.begin(), E.consts.end());
        P.progs[li] = d;
        P.flops += (uint64_t)(gradient ? E.adj_flops_per_point : E.flops_per_point) * n_eval;
        P.program_points += n_eval;
    }
    P.n_partials = part * (gradient ? kGradSlotDoubles : 1);
    // work items, one group per (path) run; an item has at most as many
    // chunks as its first program has partial sums
    P.items.reserve(part);
    static thread_local std::vector<std::pair<uint64_t, WorkItem>> items, full, tail;
    uint32_t li = 0;
    while (li < n) {
        const int pth = path[order[li]];
        uint32_t end = li;
        while (end < n && path[order[end]] == pth) ++end;
        Group g;
        g.kind = pth <= -2 ? 2 : pth == -1 ? 0 : gradient ? 3 : 1;
        g.profile = g.kind == 3 ? (pth - kAdjPathBase) % N_PROFILES
                  : pth >= 0 ? pth % kRegPathStride : pth <= -2 ? (-2 - pth) % N_PROFILES : -1;
        g.omit = g.kind == 1 ? (unsigned)(pth / kRegPathStride / 3) : 0u;
        if (g.kind == 3) {
            g.omit = 3u;
            for (uint32_t j = li; j < end; ++j) g.omit &= adj_omit[order[j]];
        }
        g.item_begin = (uint32_t)P.items.size();
        if (g.kind == 3) {
            g.G = 1;
            g.P = adj_path_p(pth);
        } else if (g.kind == 1) {
            // P and G are per profile and dataset size; one launch uses one P,
            // the largest dataset's choice.
            uint64_t max_eval = 0;
            for (uint32_t j = li; j < end; ++j) max_eval = std::max(max_eval, P.datasets[P.progs[j].dataset].n_eval);
            if (table_mu) table_lock = std::unique_lock<std::mutex>(*table_mu);
            TuneChoice c = choice_for(ctx, g.profile, max_eval);
            if (table_lock.owns_lock()) table_lock.unlock();
            g.P = c.P;
            g.G = c.G;
            P.n_reg += end - li;
        } else if (g.kind == 0) {
            g.G = 1;
            P.n_plain += end - li;
        } else {
            g.G = 1;
            g.no_unary = ((-2 - pth) / N_PROFILES) % 2 != 0;
            g.P = 1 << (((-2 - pth) / (2 * N_PROFILES)) % 3);
        }
        // tile size and per-warp staging requirements
        uint32_t j = li;
        items.clear();
        while (j < end) {
            uint32_t k = j + 1;
            const uint32_t ds = P.progs[j].dataset;
            while (k < end && k - j < (uint32_t)g.G && P.progs[k].dataset == ds) ++k;
            uint32_t cw = 0, cf = 0, sl = 0, len_sum = 0;
            for (uint32_t q = j; q < k; ++q) {
                cw += P.progs[q].uop_len + 1;
                cf += P.progs[q].n_consts;
                sl = std::max(sl, g.kind == 2 ? P.progs[q].n_tape & 0xFFFFu : P.progs[q].n_slots);
                if (g.kind == 2) g.adj_slots = std::max(g.adj_slots, P.progs[q].n_tape >> 16);
                len_sum += P.progs[q].uop_len;
                if (g.kind == 1)
                    for (int t = 0; t < N_STACKS; ++t)
                        g.stack_depth[t] = std::max(g.stack_depth[t], (uint32_t)enc[order[q]].depth_fast[t]);
                if (g.kind == 3) {  // slots: the largest warp region (floats)
                    uint32_t depth[N_STACKS];
                    for (int t = 0; t < N_STACKS; ++t) depth[t] = (uint32_t)enc[order[q]].adj_depth[t];
                    sl = std::max(sl, adj_warp_floats(depth, g.P, (uint32_t)enc[order[q]].consts.size()));
                }
            }
            g.code_words = std::max(g.code_words, cw);
            g.const_floats = std::max(g.const_floats, cf);
            g.slots = std::max(g.slots, sl);
            items.emplace_back(len_sum, WorkItem{j, k - j, 0, 0, 0, 0});
            j = k;
        }
        // register kernel: the tuned points per thread, halved while a block
        // would not fit
        if (g.kind == 1)
            while (g.P > 2 && reg_smem_bytes(g.code_words, g.const_floats, g.stack_depth, g.P, g.G) > kRegSmemBudget)
                g.P >>= 1;
        // points per thread of the slot-file kernel: largest that fits the smem budget
        if (g.kind == 0) {
            int Pp = 4;
            while (Pp > 1 && plain_smem_per_warp(g.code_words, g.const_floats, g.slots, Pp) > 110 * 1024) Pp >>= 1;
            g.P = Pp;
        }
        // register adjoint: parts per work item
        if (g.kind == 3) {
            const int nw = adj_block_warps(g.profile, g.P);
            uint32_t k = kAdjMaxParts - 1;
            for (; k > 1; k >>= 1) {
                uint64_t n_items = 0;
                for (uint32_t q = li; q < end; ++q) n_items += adj_items(P.progs[q].n_parts, k);
                if (n_items >= kAdjItemsPerSm * (uint64_t)ctx->num_sms &&
                    adj_smem_bytes(g.code_words, g.const_floats, g.slots, nw, k + 1) <= (size_t)kMaxDynSmemOptin)
                    break;
            }
            g.parts = k;
        }
        // Expand each item into chunks of kChunkPoints (g.parts of them for
        // the register adjoint) and order them longest first (persistent
        // kernels pull items in this order; any order gives the same sums).
        // A chunk's work is its programs' code length times its tiles: every
        // chunk but an item's last has the same tile count whatever the
        // dataset, so the items sorted by code length give the full chunks in
        // order, and the short last chunks are merged in.
        const uint64_t tile_pts = 32ull * g.P;
        const uint64_t part_tiles = kChunkPoints / tile_pts;
        const uint64_t tpc = g.parts * part_tiles;
        std::stable_sort(items.begin(), items.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
        full.clear();
        tail.clear();
        for (auto &pr : items) {
            const WorkItem &w = pr.second;
            const uint64_t n_eval = P.datasets[P.progs[w.prog_begin].dataset].n_eval;
            const uint64_t n_tiles = (n_eval + tile_pts - 1) / tile_pts;
            if (g.kind == 3) {  // parts spread evenly over the items
                const uint64_t n_parts = P.progs[w.prog_begin].n_parts, m = n_tiles ? adj_items(n_parts, g.parts) : 0;
                for (uint64_t c = 0; c < m; ++c) {
                    WorkItem it = w;
                    const uint64_t p0 = c * n_parts / m, p1 = (c + 1) * n_parts / m;
                    it.tile_begin = (uint32_t)(p0 * part_tiles);
                    it.tile_end = (uint32_t)std::min(n_tiles, p1 * part_tiles);
                    it.chunk = (uint32_t)p0;  // the item's first part
                    const uint64_t tiles = it.tile_end - it.tile_begin;
                    (tiles == tpc ? full : tail).emplace_back(pr.first * tiles, it);
                }
                continue;
            }
            for (uint64_t c = 0, t = 0; t < n_tiles; ++c, t += tpc) {
                WorkItem it = w;
                it.tile_begin = (uint32_t)t;
                it.tile_end = (uint32_t)std::min(n_tiles, t + tpc);
                it.chunk = (uint32_t)c;
                const uint64_t tiles = it.tile_end - it.tile_begin;
                (tiles == tpc ? full : tail).emplace_back(pr.first * tiles, it);
            }
        }
        std::stable_sort(tail.begin(), tail.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
        g.item_work = std::max(full.empty() ? 0 : full[0].first, tail.empty() ? 0 : tail[0].first);
        size_t a = 0, b = 0;
        while (a < full.size() || b < tail.size())
            P.items.push_back(b == tail.size() || (a < full.size() && full[a].first >= tail[b].first) ? full[a++].second
                                                                                                   : tail[b++].second);
        g.n_items = (uint32_t)P.items.size() - g.item_begin;
        for (uint32_t q = li; q < end; ++q) {
            const EncodedProgram &E = enc[order[q]];
            const uint64_t ne = P.datasets[P.progs[q].dataset].n_eval;
            g.flops += (uint64_t)(gradient ? E.adj_flops_per_point : E.flops_per_point) * ne;
            g.program_points += ne;
        }
        P.groups.push_back(g);
        li = end;
    }
    // Launches run side by side (enqueue_plan): the one whose longest item
    // takes longest goes first, so that it does not become the plan's tail.
    std::stable_sort(P.groups.begin(), P.groups.end(),
                     [](const Group &a, const Group &b) { return a.item_work > b.item_work; });
    return RSR_OK;
}

int upload_plan(rsr_ctx *ctx, const Plan &plan, DevicePlan *dev, cudaStream_t st) {
    NvtxRange nvtx_range("rsr: upload");
    const size_t n = plan.progs.size();
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t o_progs = 0;
    const size_t o_ds = o_progs + al(n * sizeof(ProgDesc));
    const size_t o_items = o_ds + al(plan.datasets.size() * sizeof(DatasetDesc));
    const size_t o_code = o_items + al(plan.items.size() * sizeof(WorkItem));
    const size_t o_consts = o_code + al((plan.code.size() + 1) * sizeof(uint32_t));
    const size_t total = o_consts + al((plan.consts.size() + 1) * sizeof(float));
    cudaError_t e;
    if ((e = dev->pool.reserve(total)) != cudaSuccess) return cuda_fail(e, "plan pool");
    if ((e = dev->partials.reserve(std::max<size_t>(plan.n_partials, 1) * sizeof(double))) != cudaSuccess)
        return cuda_fail(e, "partials");
    size_t out_floats = plan.mode == MODE_POINTS ? n * plan.points_stride : n * (plan.gradient ? 33 : 1);
    if (plan.raw_sums) out_floats *= 2;  // doubles
    if ((e = dev->out.reserve(std::max<size_t>(out_floats, 1) * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, "outputs");
    if ((e = dev->counters.reserve(std::max<size_t>(plan.groups.size(), 1) * sizeof(uint32_t) + 64)) != cudaSuccess)
        return cuda_fail(e, "counters");
    // the staging buffer may still feed this plan's previous copy
    if (dev->staged) {
        if ((e = cudaEventSynchronize(dev->staged)) != cudaSuccess) return cuda_fail(e, "staging wait");
    } else if ((e = cudaEventCreateWithFlags(&dev->staged, cudaEventDisableTiming)) != cudaSuccess) {
        return cuda_fail(e, "cudaEventCreate");
    }
    if (!dev->fork) {
        if ((e = cudaEventCreateWithFlags(&dev->fork, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_fail(e, "cudaEventCreate");
        for (int i = 0; i < 2; ++i) {
            if ((e = cudaEventCreateWithFlags(&dev->join[i], cudaEventDisableTiming)) != cudaSuccess)
                return cuda_fail(e, "cudaEventCreate");
            if ((e = cudaStreamCreateWithFlags(&dev->side[i], cudaStreamNonBlocking)) != cudaSuccess)
                return cuda_fail(e, "cudaStreamCreate");
        }
    }
    if ((e = dev->staging.reserve(total)) != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
    char *h = (char *)dev->staging.p;
    memcpy(h + o_progs, plan.progs.data(), n * sizeof(ProgDesc));
    memcpy(h + o_ds, plan.datasets.data(), plan.datasets.size() * sizeof(DatasetDesc));
    memcpy(h + o_items, plan.items.data(), plan.items.size() * sizeof(WorkItem));
    memcpy(h + o_code, plan.code.data(), plan.code.size() * sizeof(uint32_t));
    memcpy(h + o_consts, plan.consts.data(), plan.consts.size() * sizeof(float));
    if ((e = cudaMemcpyAsync(dev->pool.p, h, total, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "plan upload");
    if ((e = cudaEventRecord(dev->staged, st)) != cudaSuccess) return cuda_fail(e, "staging event");
    ctx->last_h2d = total;
    char *d = (char *)dev->pool.p;
    LaunchArgs &a = dev->base;
    a = LaunchArgs{};
    a.progs = (const ProgDesc *)(d + o_progs);
    a.datasets = (const DatasetDesc *)(d + o_ds);
    a.items = (const WorkItem *)(d + o_items);
    a.code = (const uint32_t *)(d + o_code);
    a.consts = (const float *)(d + o_consts);
    a.partials = (double *)dev->partials.p;
    a.mode = (uint32_t)plan.mode;
    a.points_stride = plan.points_stride;
    a.points_out = plan.mode == MODE_POINTS ? (float *)dev->out.p : nullptr;
    dev->mse = (float *)dev->out.p;
    dev->grad = plan.gradient ? (float *)dev->out.p + n : nullptr;
    return RSR_OK;
}

// Blocks per SM of a register or register-adjoint instance at a shared-memory
// size, from the occupancy API once per (device, instance, size): the query
// costs the host more than the launch it sizes.
static int blocks_per_sm(int device, int kind, int profile, int P, unsigned omit, size_t smem) {
    static std::mutex mu;
    static std::unordered_map<uint64_t, int> cache;
    const uint64_t key = ((uint64_t)(device & 255) << 56) | ((uint64_t)(kind & 3) << 54) |
                         ((uint64_t)(profile & 7) << 51) | ((uint64_t)(P & 15) << 47) | ((uint64_t)(omit & 3) << 45) |
                         (uint64_t)(smem & ((1ull << 45) - 1));
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    (void)kind;
    const int n = reg_max_blocks_per_sm(profile, P, omit, smem);
    if (n > 0) {
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = n;
    }
    return n;
}

int preload_eval_kernels(rsr_ctx *ctx) {
    if (ctx->kernels_loaded) return RSR_OK;
    cudaSetDevice(ctx->device);
    uint32_t *zero = nullptr;
    cudaError_t e = cudaMalloc(&zero, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    cudaStream_t st = ctx->stream;
    if ((e = cudaMemsetAsync(zero, 0, sizeof(uint32_t), st)) == cudaSuccess &&
        (e = preload_plain_mse(st)) == cudaSuccess && (e = preload_reg(zero, st)) == cudaSuccess &&
        (e = preload_adj(zero, st)) == cudaSuccess && (e = preload_grad(zero, st)) == cudaSuccess)
        e = cudaStreamSynchronize(st);
    else
        cudaStreamSynchronize(st);  // the launches made so far finish before the word is freed
    cudaFree(zero);
    if (e != cudaSuccess) return cuda_fail(e, "kernel preload");
    ctx->kernels_loaded = true;
    return RSR_OK;
}

// Makes st wait for the launches a plan put on its side streams.
static cudaError_t join_side_streams(DevicePlan *dev, cudaStream_t st, unsigned forked) {
    cudaError_t first = cudaSuccess;
    for (int sd = 0; sd < 2; ++sd)
        if (forked & (1u << sd)) {
            cudaError_t e = cudaEventRecord(dev->join[sd], dev->side[sd]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, dev->join[sd], 0);
            if (first == cudaSuccess) first = e;
        }
    return first;
}

int enqueue_plan(rsr_ctx *ctx, const Plan &plan, DevicePlan *dev, cudaStream_t st, cudaEvent_t ev_mid,
                 cudaEvent_t *group_events) {
    NvtxRange nvtx_range("rsr: launch");
    const uint32_t n = (uint32_t)plan.progs.size();
    if (n == 0) {
        if (ev_mid) cudaEventRecord(ev_mid, st);
        return RSR_OK;
    }
    cudaError_t e;
    uint32_t *counters = (uint32_t *)dev->counters.p;
    if ((e = cudaMemsetAsync(counters, 0, plan.groups.size() * sizeof(uint32_t), st)) != cudaSuccess)
        return cuda_fail(e, "counter reset");
    // Launch j > 0 goes to side stream (j - 1) % 2 unless per-launch timing is
    // asked for (events around each launch then time it alone).  Launches
    // share nothing but the partials, which each item writes at its own index.
    const bool concurrent = !group_events && dev->side[0];
    unsigned forked = 0;
    int j = -1;
    for (size_t gi = 0; gi < plan.groups.size(); ++gi) {
        const Group &g = plan.groups[gi];
        if (g.n_items == 0) continue;
        cudaStream_t gs = st;
        if (concurrent && ++j > 0) {
            const int sd = (j - 1) & 1;
            if (!(forked & (1u << sd))) {
                if (!forked && (e = cudaEventRecord(dev->fork, st)) != cudaSuccess) return cuda_fail(e, "fork");
                if ((e = cudaStreamWaitEvent(dev->side[sd], dev->fork, 0)) != cudaSuccess) return cuda_fail(e, "fork");
                forked |= 1u << sd;
            }
            gs = dev->side[sd];
        }
        LaunchArgs a = dev->base;
        a.items = dev->base.items + g.item_begin;
        a.n_items = g.n_items;
        a.item_counter = counters + gi;
        a.smem_code_words = g.code_words;
        a.smem_const_floats = g.const_floats;
        a.smem_slots = g.slots;
        a.progs_per_warp = g.G;
        if (group_events) cudaEventRecord(group_events[2 * gi], gs);
        if (g.kind == 0) {
            const size_t per = plain_smem_per_warp(g.code_words, g.const_floats, g.slots, g.P);
            uint32_t wpb = (uint32_t)std::max<size_t>(1, std::min<size_t>(kPlainThreads / 32, (200 * 1024) / per));
            g.grid = (g.n_items + wpb - 1) / wpb;
            g.smem = per * wpb;
            g.warps_per_block = wpb;
            e = launch_plain(a, g.P, wpb, per * wpb, gs);
        } else if (g.kind == 1) {
            reg_layout(g.code_words, g.const_floats, g.stack_depth, g.P, g.G, a.stack_off, &a.acc_off, &a.region_floats,
                       &a.block_hdr_floats);
            const size_t smem = ((size_t)a.block_hdr_floats + (size_t)a.region_floats * (kRegThreads / 32)) * 4u;
            int bps = std::max(1, blocks_per_sm(ctx->device, 1, g.profile, g.P, g.omit, smem));
            uint32_t grid = (uint32_t)std::min<uint64_t>((uint64_t)bps * ctx->num_sms, g.n_items);
            g.grid = std::max(1u, grid);
            g.smem = smem;
            g.warps_per_block = kRegThreads / 32;
            e = launch_reg(a, g.profile, g.P, g.omit, g.grid, gs);
        } else if (g.kind == 3) {
            const int nw = adj_block_warps(g.profile, g.P);
            adj_layout(g.code_words, g.const_floats, g.slots, nw, g.parts + (g.parts > 1), &a);
            g.tmem_cols = a.tmem_cols;
            // One block per SM: it allocates all of the SM's tensor memory,
            // and its shared memory is padded past half the SM's so that no
            // second such block, of this launch or one beside it, shares the
            // SM and waits for the columns.
            const size_t half = ctx->smem_per_sm / 2 + 16;
            const size_t pad = half > ctx->smem_reserved ? half - ctx->smem_reserved : 0;
            const size_t smem =
                std::max(adj_smem_bytes(g.code_words, g.const_floats, g.slots, nw, g.parts + (g.parts > 1)), pad);
            if (nw < 4 || smem > (size_t)kMaxDynSmemOptin) {
                e = cudaErrorInvalidValue;
                join_side_streams(dev, st, forked);
                return fail(RSR_EINVAL, "register adjoint launch needs " + std::to_string(smem) +
                                            " bytes of shared memory per block");
            }
            g.grid = std::max(1u, (uint32_t)std::min<uint64_t>((uint64_t)ctx->num_sms, g.n_items));
            g.smem = smem;
            g.warps_per_block = (uint32_t)nw;
            e = launch_adj(a, g.profile, g.P, g.omit, g.grid, smem, gs);
        } else {
            const size_t per = grad_smem_per_warp(g.code_words, g.const_floats, g.slots, g.adj_slots, g.P);
            a.smem_adj_slots = g.adj_slots;
            // one warp per block: blocks as small as a tape, so an SM packs as
            // many tapes as its shared memory holds
            const uint32_t wpb = 1;
            a.progs_per_warp = (uint32_t)g.P;  // adjoint kernel reads P from here
            g.grid = (g.n_items + wpb - 1) / wpb;
            g.smem = per * wpb;
            g.warps_per_block = wpb;
            e = launch_grad(a, g.profile, g.no_unary, wpb, per * wpb, gs);
        }
        if (e != cudaSuccess) {
            // launches already on the side streams must finish before the
            // caller's stream (and the next use of this plan's buffers) moves on
            join_side_streams(dev, st, forked);
            return cuda_fail(e, "kernel launch");
        }
        if (group_events) cudaEventRecord(group_events[2 * gi + 1], gs);
        ctx->launches++;
    }
    if ((e = join_side_streams(dev, st, forked)) != cudaSuccess) return cuda_fail(e, "join");
    if (ev_mid) cudaEventRecord(ev_mid, st);
    if (plan.mode == MODE_MSE && plan.raw_sums) {
        e = launch_finalize_sums(dev->base.progs, dev->base.partials, n, plan.gradient ? 33u : 1u,
                                 (double *)dev->out.p, st);
        if (e != cudaSuccess) return cuda_fail(e, "finalize launch");
        ctx->launches++;
    } else if (plan.mode == MODE_MSE) {
        if (plan.gradient)
            e = launch_finalize_grad(dev->base.progs, dev->base.datasets, dev->base.partials, n, dev->mse, dev->grad, st);
        else
            e = launch_finalize_mse(dev->base.progs, dev->base.datasets, dev->base.partials, n, dev->mse, st);
        if (e != cudaSuccess) return cuda_fail(e, "finalize launch");
        ctx->launches++;
    }
    return RSR_OK;
}

// Copy results back in caller order.
static int fetch_results(rsr_ctx *ctx, const Plan &plan, DevicePlan &dev, cudaStream_t st, float *mse_out,
                         float *grad_out, float *points_out) {
    NvtxRange nvtx_range("rsr: download");
    const size_t n = plan.progs.size();
    if (n == 0) return RSR_OK;
    cudaError_t e;
    if (plan.mode == MODE_POINTS) {
        const size_t per = plan.points_stride;
        std::vector<float> tmp(n * per);
        if ((e = cudaMemcpyAsync(tmp.data(), dev.out.p, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, st)))
            return cuda_fail(e, "points download");
        if ((e = cudaStreamSynchronize(st))) return cuda_fail(e, "evaluation");
        ctx->last_d2h = tmp.size() * sizeof(float);
        for (size_t li = 0; li < n; ++li) memcpy(points_out + (size_t)plan.orig[li] * per, tmp.data() + li * per, per * sizeof(float));
        return RSR_OK;
    }
    const size_t nf = n * (plan.gradient ? 33 : 1);
    std::vector<float> tmp(nf);
    if ((e = cudaMemcpyAsync(tmp.data(), dev.out.p, nf * sizeof(float), cudaMemcpyDeviceToHost, st)))
        return cuda_fail(e, "result download");
    if ((e = cudaStreamSynchronize(st))) return cuda_fail(e, "evaluation");
    ctx->last_d2h = nf * sizeof(float);
    for (size_t li = 0; li < n; ++li) {
        if (mse_out) mse_out[plan.orig[li]] = tmp[li];
        if (grad_out && plan.gradient) memcpy(grad_out + (size_t)plan.orig[li] * 32, tmp.data() + n + li * 32, 32 * sizeof(float));
    }
    (void)ctx;
    return RSR_OK;
}

static rsr_population single_pop(const rsr_program *p, uint64_t offs[6]) {
    offs[0] = 0; offs[1] = p->len; offs[2] = 0; offs[3] = p->n_consts; offs[4] = 0; offs[5] = p->n_params;
    rsr_population pop{};
    pop.n_programs = 1;
    pop.code = p->code;
    pop.code_off = offs;
    pop.const_kinds = p->const_kinds;
    pop.kind_off = offs + 2;
    pop.params = p->params;
    pop.param_off = offs + 4;
    return pop;
}

// A large MSE (or MSE + gradient) call in chunks of programs: the host
// encodes chunk k+1 while the device runs chunk k.  Chunks alternate between
// two device plans, each with its own stream, so chunk k+1's first launch
// fills the SMs that chunk k's last blocks leave; a plan's buffers are
// rewritten by a later chunk on the same stream, after the device is done
// with them.
static int run_chunked(rsr_ctx *ctx, const rsr_population &pop, const uint64_t *dsp, uint64_t ds, int kernel,
                       bool gradient, float *mse, float *grad, const std::vector<uint32_t> &start) {
    const uint32_t n_chunks = (uint32_t)start.size() - 1;
    NvtxRange nvtx_range("rsr: chunked call");
    const uint32_t n = pop.n_programs, stride = gradient ? 33u : 1u;
    cudaError_t e;
    if ((e = ctx->results.reserve((size_t)n * stride * sizeof(float))) != cudaSuccess)
        return cuda_fail(e, "cudaHostAlloc");
    float *res = (float *)ctx->results.p;
    if (ctx->call_plans.size() < n_chunks) ctx->call_plans.resize(n_chunks);
    std::vector<Plan> &plans = ctx->call_plans;
    auto sync_both = [&] {
        cudaStreamSynchronize(ctx->stream2);
        cudaStreamSynchronize(ctx->stream);
    };
    uint64_t h2d = 0;
    for (uint32_t k = 0; k < n_chunks; ++k) {
        const uint32_t s0 = start[k], cnt = start[k + 1] - s0;
        rsr_population sub = pop;
        sub.n_programs = cnt;
        sub.code_off = pop.code_off + s0;
        sub.kind_off = pop.kind_off + s0;
        sub.param_off = pop.param_off + s0;
        int rc = build_plan(ctx, sub, dsp ? dsp + s0 : nullptr, ds, kernel, gradient, MODE_MSE, &plans[k]);
        if (rc) {
            // report the program by its index in the caller's population
            std::string m = rsr_last_error();
            const size_t at = m.rfind("program ", 0) == 0 ? 8 : std::string::npos;
            if (at != std::string::npos) {
                size_t end = m.find(':', at);
                m = "program " + std::to_string(s0 + std::stoul(m.substr(at, end - at))) + m.substr(end);
            }
            sync_both();
            return fail(rc, m);
        }
        DevicePlan *dev = &ctx->pipe[k & 1];
        cudaStream_t st = (k & 1) ? ctx->stream2 : ctx->stream;
        if ((rc = upload_plan(ctx, plans[k], dev, st))) { sync_both(); return rc; }
        h2d += ctx->last_h2d;
        if ((rc = enqueue_plan(ctx, plans[k], dev, st, nullptr))) { sync_both(); return rc; }
        if ((e = cudaMemcpyAsync(res + (size_t)s0 * stride, dev->out.p, (size_t)cnt * stride * sizeof(float),
                                 cudaMemcpyDeviceToHost, st)) != cudaSuccess) {
            sync_both();
            return cuda_fail(e, "result download");
        }
    }
    if ((e = cudaStreamSynchronize(ctx->stream2)) != cudaSuccess) return cuda_fail(e, "evaluation");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(e, "evaluation");
    for (uint32_t k = 0; k < n_chunks; ++k) {
        const uint32_t s0 = start[k], cnt = start[k + 1] - s0;
        const float *r = res + (size_t)s0 * stride;
        for (uint32_t li = 0; li < cnt; ++li) {
            const uint32_t i = s0 + plans[k].orig[li];
            if (mse) mse[i] = r[li];
            if (gradient && grad) memcpy(grad + (size_t)i * 32, r + cnt + (size_t)li * 32, 32 * sizeof(float));
        }
    }
    ctx->last_h2d = h2d;
    ctx->last_d2h = (uint64_t)n * stride * sizeof(float);
    return RSR_OK;
}

// Chunks of a chunked call double in size from kFirstChunk programs up to
// kMaxChunk, and the last one takes the rest (up to one and a half chunks):
// the device starts on a small first chunk soon, and since the host plans a
// program several times faster than the device runs it, each later chunk is
// planned while the device still runs the chunks before it.
static constexpr uint32_t kFirstChunk = 256, kMaxChunk = 8192;

static std::vector<uint32_t> chunk_starts(uint32_t n) {
    std::vector<uint32_t> start{0};
    uint32_t size = kFirstChunk;
    while (n - start.back() > size + size / 2) {
        start.push_back(start.back() + size);
        if (size < kMaxChunk) size *= 2;
    }
    start.push_back(n);
    return start;
}

static int run_oneshot(rsr_ctx *ctx, const rsr_population &pop, const uint64_t *dsp, uint64_t ds, int kernel,
                       bool gradient, int mode, float *mse, float *grad, float *points) {
    if (mode == MODE_MSE && pop.n_programs >= 4 * kFirstChunk)
        return run_chunked(ctx, pop, dsp, ds, kernel, gradient, mse, grad, chunk_starts(pop.n_programs));
    if (ctx->call_plans.empty()) ctx->call_plans.resize(1);
    Plan &plan = ctx->call_plans[0];
    int rc = build_plan(ctx, pop, dsp, ds, kernel, gradient, mode, &plan);
    if (rc) return rc;
    if (mode == MODE_POINTS) {
        plan.points_stride = plan.datasets.empty() ? 0 : plan.datasets[0].n_eval;
    }
    if ((rc = upload_plan(ctx, plan, &ctx->scratch, ctx->stream))) return rc;
    if ((rc = enqueue_plan(ctx, plan, &ctx->scratch, ctx->stream, nullptr))) return rc;
    return fetch_results(ctx, plan, ctx->scratch, ctx->stream, mse, grad, points);
}

int alloc_dataset(rsr_ctx *ctx, uint32_t nf, uint64_t nbatch, uint64_t nsamples, std::unique_ptr<DatasetRec> *out) {
    if (nbatch == 0 || nsamples == 0 || nsamples > nbatch * 8 || nsamples <= (nbatch - 1) * 8)
        return fail(RSR_EINVAL, "num_samples must satisfy 8*(num_batches-1) < num_samples <= 8*num_batches");
    if (nf > 255) return fail(RSR_EINVAL, "at most 255 features (LoadVar operands are u8)");
    const uint64_t n_eval = nbatch * 8;
    const uint64_t stride = round_up(n_eval, kStrideAlign);
    const size_t xbytes = (size_t)stride * std::max<uint32_t>(nf, 1) * sizeof(float);
    const size_t ybytes = (size_t)stride * sizeof(float);
    if (ctx->mem_in_use + xbytes + ybytes > ctx->opts.mem_budget_bytes)
        return fail(RSR_ENOMEM, "dataset exceeds the context's memory budget");
    auto rec = std::make_unique<DatasetRec>();
    cudaError_t e;
    if ((e = cudaMalloc(&rec->x, xbytes)) != cudaSuccess) return cuda_fail(e, "dataset features");
    if ((e = cudaMalloc(&rec->y, ybytes)) != cudaSuccess) { cudaFree(rec->x); return cuda_fail(e, "dataset targets"); }
    cudaMemsetAsync(rec->x, 0, xbytes, ctx->stream);
    cudaMemsetAsync(rec->y, 0, ybytes, ctx->stream);
    rec->num_features = nf;
    rec->num_batches = nbatch;
    rec->num_samples = nsamples;
    rec->stride = stride;
    rec->bytes = xbytes + ybytes;
    *out = std::move(rec);
    return RSR_OK;
}

rsr_dataset register_dataset(rsr_ctx *ctx, std::unique_ptr<DatasetRec> rec) {
    ctx->mem_in_use += rec->bytes;
    const uint64_t h = ctx->next_handle++;
    ctx->datasets.emplace(h, std::move(rec));
    return h;
}

}  // namespace rsr

using namespace rsr;

// ====================================================================== ABI
extern "C" {

const char *rsr_last_error(void) { return g_last_error.c_str(); }
const char *rsr_version(void) { return "rsr-b200 0.1 (sm_100a)"; }

void rsr_options_default(rsr_options *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(rsr_options);
    o->kernel = RSR_KERNEL_AUTO;
    o->use_graphs = 1;
}

int rsr_ctx_create(int device, const rsr_options *opts, rsr_ctx **out) {
    if (!out) return fail(RSR_EINVAL, "out is null");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(RSR_ENODEV, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(RSR_EINVAL, "device index out of range");
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return cuda_fail(e, "device properties");
    if (prop.major != 10) return fail(RSR_ENODEV, std::string("sm_100 device required, found ") + prop.name);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    auto *ctx = new rsr_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    ctx->smem_per_sm = prop.sharedMemPerMultiprocessor;
    ctx->smem_reserved = prop.reservedSharedMemPerBlock;
    rsr_options_default(&ctx->opts);
    if (opts) memcpy(&ctx->opts, opts, std::min<size_t>(sizeof(rsr_options), opts->struct_size ? opts->struct_size : sizeof(rsr_options)));
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking)) != cudaSuccess) {
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return cuda_fail(e, "stream");
    }
    for (auto &ev : ctx->ev) cudaEventCreate(&ev);
    if (ctx->opts.mem_budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        ctx->opts.mem_budget_bytes = (uint64_t)(fr * 0.9);
    }
    *out = ctx;
    return RSR_OK;
}

int rsr_ctx_destroy(rsr_ctx *ctx) {
    if (!ctx) return RSR_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->stream2);
    for (auto &kv : ctx->datasets) {
        cudaFree(kv.second->x);
        cudaFree(kv.second->y);
    }
    ctx->scratch.pool.release();
    ctx->scratch.partials.release();
    ctx->scratch.out.release();
    ctx->scratch.counters.release();
    ctx->scratch.staging.release();
    for (DevicePlan &d : ctx->pipe) {
        d.pool.release(); d.partials.release(); d.out.release(); d.counters.release(); d.staging.release();
    }
    ctx->results.release();
    if (ctx->l2buf) cudaFree(ctx->l2buf);
    for (auto &ev : ctx->ev) if (ev) cudaEventDestroy(ev);
    cudaStreamDestroy(ctx->stream);
    cudaStreamDestroy(ctx->stream2);
    delete ctx;
    return RSR_OK;
}

static int upload_soa(rsr_ctx *ctx, const float *ff, const float *tb, bool aosoa, uint32_t nf, uint64_t nbatch,
                      uint64_t nsamples, rsr_dataset *out) {
    if (!out) return fail(RSR_EINVAL, "out is null");
    if ((nf && !ff) || !tb) return fail(RSR_EINVAL, "feature or target pointer is null");
    std::unique_ptr<DatasetRec> rec;
    int rc = alloc_dataset(ctx, nf, nbatch, nsamples, &rec);
    if (rc) return rc;
    const uint64_t stride = rec->stride;
    cudaError_t e;
    if (aosoa) {
        // raw AoSoA upload, transposed on the device
        const size_t rawx = (size_t)nbatch * nf * 8 * sizeof(float), rawy = (size_t)nbatch * 8 * sizeof(float);
        void *tmp = nullptr;
        if ((e = cudaMalloc(&tmp, rawx + rawy)) != cudaSuccess) {
            cudaFree(rec->x); cudaFree(rec->y);
            return cuda_fail(e, "dataset staging");
        }
        if (rawx) cudaMemcpyAsync(tmp, ff, rawx, cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync((char *)tmp + rawx, tb, rawy, cudaMemcpyHostToDevice, ctx->stream);
        e = launch_aosoa_to_soa((const float *)tmp, (const float *)((char *)tmp + rawx), rec->x, rec->y, nf, nbatch,
                                stride, ctx->num_sms, ctx->stream);
        ctx->launches++;
        const cudaError_t se = cudaStreamSynchronize(ctx->stream);
        if (e == cudaSuccess) e = se;
        cudaFree(tmp);
    } else {
        // columns: features[f*n + i] with n = nsamples, zero padded
        for (uint32_t f = 0; f < nf; ++f)
            cudaMemcpyAsync(rec->x + (size_t)f * stride, ff + (size_t)f * nsamples, nsamples * sizeof(float),
                            cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(rec->y, tb, nsamples * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
        e = cudaStreamSynchronize(ctx->stream);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaFree(rec->x); cudaFree(rec->y);
        return cuda_fail(e, "dataset upload");
    }
    *out = register_dataset(ctx, std::move(rec));
    return RSR_OK;
}

int rsr_dataset_upload(rsr_ctx *ctx, const float *feature_flat, const float *target_batches, uint32_t num_features,
                       uint64_t num_batches, uint64_t num_samples, rsr_dataset *out) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return upload_soa(ctx, feature_flat, target_batches, true, num_features, num_batches, num_samples, out);
}

int rsr_dataset_upload_columns(rsr_ctx *ctx, const float *features, const float *targets, uint32_t num_features,
                               uint64_t n, rsr_dataset *out) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return upload_soa(ctx, features, targets, false, num_features, (n + 7) / 8, n, out);
}

int rsr_dataset_release(rsr_ctx *ctx, rsr_dataset ds) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->datasets.find(ds);
    if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle");
    if (it->second->refs.load() > 0) return fail(RSR_EBUSY, "dataset is referenced by a prepared batch or a job");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(it->second->x);
    cudaFree(it->second->y);
    ctx->mem_in_use -= it->second->bytes;
    ctx->datasets.erase(it);
    return RSR_OK;
}

int rsr_dataset_info(rsr_ctx *ctx, rsr_dataset ds, uint32_t *nf, uint64_t *nb, uint64_t *ns) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->datasets.find(ds);
    if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle");
    if (nf) *nf = it->second->num_features;
    if (nb) *nb = it->second->num_batches;
    if (ns) *ns = it->second->num_samples;
    return RSR_OK;
}

int rsr_compute_mse(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse) {
    if (!ctx || !prog || !mse) return fail(RSR_EINVAL, "null argument");
    uint64_t offs[6];
    rsr_population pop = single_pop(prog, offs);
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, pop, nullptr, ds, ctx->opts.kernel, false, MODE_MSE, mse, nullptr, nullptr);
}

int rsr_compute_mse_with_gradient(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse, float *grad) {
    if (!ctx || !prog || !mse || !grad) return fail(RSR_EINVAL, "null argument");
    uint64_t offs[6];
    rsr_population pop = single_pop(prog, offs);
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, pop, nullptr, ds, RSR_KERNEL_AUTO, true, MODE_MSE, mse, grad, nullptr);
}

int rsr_eval_points(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *out) {
    if (!ctx || !prog || !out) return fail(RSR_EINVAL, "null argument");
    uint64_t offs[6];
    rsr_population pop = single_pop(prog, offs);
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, pop, nullptr, ds, ctx->opts.kernel, false, MODE_POINTS, nullptr, nullptr, out);
}

int rsr_eval_mse_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp, int kernel,
                       float *mse_out) {
    if (!ctx || !pop || (!mse_out && pop->n_programs)) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, *pop, dsp, ds, kernel, false, MODE_MSE, mse_out, nullptr, nullptr);
}

int rsr_eval_mse_grad_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp,
                            float *mse_out, float *grad_out) {
    if (!ctx || !pop || ((!mse_out || !grad_out) && pop->n_programs)) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, *pop, dsp, ds, RSR_KERNEL_AUTO, true, MODE_MSE, mse_out, grad_out, nullptr);
}

int rsr_eval_sums_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp,
                        int gradient, double *sums_out) {
    if (!ctx || !pop || (!sums_out && pop->n_programs)) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    Plan plan;
    int rc = build_plan(ctx, *pop, dsp, ds, RSR_KERNEL_AUTO, gradient != 0, MODE_MSE, &plan);
    if (rc) return rc;
    plan.raw_sums = true;
    const size_t n = plan.progs.size();
    if (n == 0) return RSR_OK;
    if ((rc = upload_plan(ctx, plan, &ctx->scratch, ctx->stream))) return rc;
    if ((rc = enqueue_plan(ctx, plan, &ctx->scratch, ctx->stream, nullptr))) return rc;
    const size_t stride = gradient ? 33 : 1;
    std::vector<double> tmp(n * stride);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(tmp.data(), ctx->scratch.out.p, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                             ctx->stream)) != cudaSuccess)
        return cuda_fail(e, "sums download");
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_fail(e, "evaluation");
    ctx->last_d2h = tmp.size() * sizeof(double);
    for (size_t li = 0; li < n; ++li)
        memcpy(sums_out + (size_t)plan.orig[li] * stride, tmp.data() + li * stride, stride * sizeof(double));
    return RSR_OK;
}

int rsr_finalize_sums(uint32_t n, int gradient, const double *sums, uint64_t num_samples, float *mse_out,
                      float *grad_out) {
    if ((!sums || !mse_out || (gradient && !grad_out)) && n) return fail(RSR_EINVAL, "null argument");
    const size_t stride = gradient ? 33 : 1;
    const double ns = (double)num_samples;
    for (uint32_t p = 0; p < n; ++p) {
        const double s = sums[p * stride];
        const float m = (float)(s / ns);
        const bool bad = !(s <= (double)FLT_MAX) || !std::isfinite(m);
        mse_out[p] = bad ? FLT_MAX : m;
        if (gradient)
            for (int k = 0; k < 32; ++k) grad_out[(size_t)p * 32 + k] = bad ? 0.0f : (float)(sums[p * stride + 1 + k] / ns);
    }
    return RSR_OK;
}

int rsr_eval_points_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, int kernel, float *out) {
    if (!ctx || !pop || (!out && pop->n_programs)) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_oneshot(ctx, *pop, nullptr, ds, kernel, false, MODE_POINTS, nullptr, nullptr, out);
}

// ------------------------------------------------------------ prepared
int rsr_batch_prepare(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp, int kernel,
                      int with_gradient, rsr_batch **out) {
    if (!ctx || !pop || !out) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    auto *b = new rsr_batch();
    int rc = build_plan(ctx, *pop, dsp, ds, kernel, with_gradient != 0, MODE_MSE, &b->plan);
    if (!rc) rc = upload_plan(ctx, b->plan, &b->dev, ctx->stream);
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "prepare");
    if (rc) {
        delete b;
        return rc;
    }
    for (uint64_t h : b->plan.ds_handles) ctx->datasets[h]->refs++;
    for (auto &ev : b->ev) cudaEventCreate(&ev);
    b->pool_bytes = ctx->last_h2d;
    b->gev.resize(2 * b->plan.groups.size());
    for (auto &ev : b->gev) cudaEventCreate(&ev);
    b->group_ms.assign(b->plan.groups.size(), 0.0f);
    *out = b;
    return RSR_OK;
}

int rsr_batch_run(rsr_ctx *ctx, rsr_batch *b) {
    if (!ctx || !b) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaError_t e;
    if (ctx->opts.use_graphs) {
        if (!b->graph_ready) {
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                return cuda_fail(e, "graph capture");
            uint64_t before = ctx->launches.load();
            int rc = enqueue_plan(ctx, b->plan, &b->dev, ctx->stream, nullptr);
            e = cudaStreamEndCapture(ctx->stream, &g);
            if (rc) return rc;
            if (e != cudaSuccess) return cuda_fail(e, "graph capture");
            if ((e = cudaGraphInstantiate(&b->graph, g, 0)) != cudaSuccess) return cuda_fail(e, "graph instantiate");
            cudaGraphDestroy(g);
            b->graph_ready = true;
            ctx->launches = before;  // counted at replay
        }
        cudaEventRecord(b->ev[0], ctx->stream);
        if ((e = cudaGraphLaunch(b->graph, ctx->stream)) != cudaSuccess) return cuda_fail(e, "graph launch");
        uint64_t nl = 0;
        for (auto &g : b->plan.groups) nl += g.n_items ? 1 : 0;
        ctx->launches += nl + (b->plan.progs.empty() ? 0 : 1);
        cudaEventRecord(b->ev[2], ctx->stream);
        return RSR_OK;
    }
    cudaEventRecord(b->ev[0], ctx->stream);
    int rc = enqueue_plan(ctx, b->plan, &b->dev, ctx->stream, b->ev[1], b->gev.data());
    if (rc) return rc;
    cudaEventRecord(b->ev[2], ctx->stream);
    return RSR_OK;
}

int rsr_batch_results(rsr_ctx *ctx, rsr_batch *b, float *mse_out, float *grad_out) {
    if (!ctx || !b) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    int rc = fetch_results(ctx, b->plan, b->dev, ctx->stream, mse_out, grad_out, nullptr);
    if (rc) return rc;
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, b->ev[0], b->ev[2]) == cudaSuccess) b->total_ms = t;
    if (!ctx->opts.use_graphs && cudaEventElapsedTime(&t, b->ev[0], b->ev[1]) == cudaSuccess) b->eval_ms = t;
    else b->eval_ms = b->total_ms;
    return RSR_OK;
}

int rsr_batch_last_timing(rsr_ctx *ctx, rsr_batch *b, float *eval_ms, float *total_ms) {
    if (!ctx || !b) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaEventSynchronize(b->ev[2]);
    if (e != cudaSuccess) return cuda_fail(e, "timing");
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, b->ev[0], b->ev[2]) == cudaSuccess) b->total_ms = t;
    b->eval_ms = b->total_ms;
    if (!ctx->opts.use_graphs && cudaEventElapsedTime(&t, b->ev[0], b->ev[1]) == cudaSuccess) b->eval_ms = t;
    if (!ctx->opts.use_graphs)
        for (size_t g = 0; g < b->plan.groups.size(); ++g)
            if (b->plan.groups[g].n_items && cudaEventElapsedTime(&t, b->gev[2 * g], b->gev[2 * g + 1]) == cudaSuccess)
                b->group_ms[g] = t;
    if (eval_ms) *eval_ms = b->eval_ms;
    if (total_ms) *total_ms = b->total_ms;
    return RSR_OK;
}

int rsr_batch_describe(rsr_ctx *ctx, rsr_batch *b, char *buf, size_t len) {
    if (!ctx || !b || !buf || !len) return fail(RSR_EINVAL, "null argument");
    std::string s = "{\"programs\": " + std::to_string(b->plan.progs.size()) +
                    ", \"register_kernel_programs\": " + std::to_string(b->plan.n_reg) +
                    ", \"slot_kernel_programs\": " + std::to_string(b->plan.n_plain) +
                    ", \"work_items\": " + std::to_string(b->plan.items.size()) +
                    ", \"flops\": " + std::to_string(b->plan.flops) +
                    ", \"program_points\": " + std::to_string(b->plan.program_points) + ", \"groups\": [";
    for (size_t i = 0; i < b->plan.groups.size(); ++i) {
        const Group &g = b->plan.groups[i];
        const char *kn = g.kind == 0 ? "slot" : g.kind == 1 ? "register" : g.kind == 2 ? "adjoint" : "register_adjoint";
        s += (i ? ", " : "") + std::string("{\"kernel\": \"") + kn + "\", \"profile\": " + std::to_string(g.profile) +
             ", \"no_unary\": " + (((g.kind == 1 || g.kind == 3) ? (g.omit & 1u) != 0 : g.no_unary) ? "true" : "false") +
             ", \"no_matrix_operand\": " + (((g.kind == 1 || g.kind == 3) && (g.omit & 2u)) ? "true" : "false") +
             ", \"tmem_cols\": " + std::to_string(g.tmem_cols) + ", \"parts_per_item\": " + std::to_string(g.parts) +
             ", \"points_per_thread\": " + std::to_string(g.P) + ", \"programs_per_warp\": " + std::to_string(g.G) +
             ", \"items\": " + std::to_string(g.n_items) + ", \"flops\": " + std::to_string(g.flops) +
             ", \"program_points\": " + std::to_string(g.program_points) + ", \"grid\": " + std::to_string(g.grid) +
             ", \"warps_per_block\": " + std::to_string(g.warps_per_block) + ", \"smem_bytes\": " +
             std::to_string(g.smem) + ", \"last_ms\": " +
             std::to_string(b->group_ms.size() > i ? b->group_ms[i] : 0.0f) + "}";
    }
    s += "], \"upload_bytes\": " + std::to_string(b->pool_bytes) + "}";
    snprintf(buf, len, "%s", s.c_str());
    return RSR_OK;
}

int rsr_batch_destroy(rsr_ctx *ctx, rsr_batch *b) {
    if (!ctx || !b) return RSR_OK;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (uint64_t h : b->plan.ds_handles) {
        auto it = ctx->datasets.find(h);
        if (it != ctx->datasets.end()) it->second->refs--;
    }
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto &ev : b->ev) if (ev) cudaEventDestroy(ev);
    for (auto &ev : b->gev) if (ev) cudaEventDestroy(ev);
    delete b;
    return RSR_OK;
}

uint64_t rsr_ctx_launch_count(rsr_ctx *ctx) { return ctx ? ctx->launches.load() : 0; }

int rsr_ctx_last_transfer(rsr_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    if (h2d_bytes) *h2d_bytes = ctx->last_h2d;
    if (d2h_bytes) *d2h_bytes = ctx->last_d2h;
    return RSR_OK;
}

int rsr_flush_l2(rsr_ctx *ctx) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->l2buf) {
        ctx->l2bytes = 256ull << 20;
        cudaError_t e = cudaMalloc(&ctx->l2buf, ctx->l2bytes);
        if (e != cudaSuccess) return cuda_fail(e, "L2 flush buffer");
    }
    cudaError_t e = cudaMemsetAsync(ctx->l2buf, ctx->launches.load() & 0xFF, ctx->l2bytes, ctx->stream);
    return e == cudaSuccess ? RSR_OK : cuda_fail(e, "L2 flush");
}

int rsr_synchronize(rsr_ctx *ctx) {
    if (!ctx) return fail(RSR_EINVAL, "ctx is null");
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? RSR_OK : cuda_fail(e, "synchronize");
}

// Autotuner: times every (points per thread, programs per warp) candidate of
// the register kernel on this population and keeps, per kernel profile and
// dataset size class, the fastest.  Later plans of the context use it.
int rsr_autotune(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *dsp, int reps,
                 char *report, size_t report_len) {
    if (!ctx || !pop) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (reps < 1) reps = 3;
    const int Ps[3] = {2, 4, 8}, Gs[4] = {1, 2, 4, 8};
    struct Best { float ms = 1e30f; TuneChoice c; int bucket = 0; };
    std::map<int, Best> best;   // profile -> best
    std::string rep = "{\"candidates\": [";
    bool first = true;
    DevicePlan dev;
    std::vector<cudaEvent_t> ev;
    int rc = RSR_OK;
    for (int P : Ps)
        for (int G : Gs) {
            ctx->force = TuneChoice{P, G};
            Plan plan;
            rc = build_plan(ctx, *pop, dsp, ds, RSR_KERNEL_BATCHED, false, MODE_MSE, &plan);
            if (!rc) rc = upload_plan(ctx, plan, &dev, ctx->stream);
            if (rc) break;
            while (ev.size() < 2 * plan.groups.size()) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                ev.push_back(e);
            }
            std::vector<float> gmin(plan.groups.size(), 1e30f);
            for (int r = 0; r < reps + 1 && !rc; ++r) {
                rc = enqueue_plan(ctx, plan, &dev, ctx->stream, nullptr, ev.data());
                if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "autotune");
                for (size_t g = 0; !rc && r > 0 && g < plan.groups.size(); ++g) {
                    float t = 0.0f;
                    if (plan.groups[g].n_items && cudaEventElapsedTime(&t, ev[2 * g], ev[2 * g + 1]) == cudaSuccess)
                        gmin[g] = std::min(gmin[g], t);
                }
            }
            if (rc) break;
            // a profile may run as several launches (spill-depth classes):
            // its candidate time is their sum
            std::map<int, std::pair<float, uint64_t>> per;  // profile -> (ms, largest dataset)
            for (size_t g = 0; g < plan.groups.size(); ++g) {
                const Group &gr = plan.groups[g];
                if (gr.kind != 1 || !gr.n_items) continue;
                uint64_t max_eval = 0;
                for (uint32_t i = gr.item_begin; i < gr.item_begin + gr.n_items; ++i)
                    max_eval = std::max(max_eval, plan.datasets[plan.progs[plan.items[i].prog_begin].dataset].n_eval);
                auto &pp = per[gr.profile];
                pp.first += gmin[g];
                pp.second = std::max(pp.second, max_eval);
            }
            for (auto &kv : per) {
                Best &b = best[kv.first];
                if (kv.second.first < b.ms) {
                    b.ms = kv.second.first;
                    b.c = TuneChoice{P, G};
                    b.bucket = log2_bucket(kv.second.second);
                }
                rep += std::string(first ? "" : ", ") + "{\"profile\": " + std::to_string(kv.first) +
                       ", \"P\": " + std::to_string(P) + ", \"G\": " + std::to_string(G) +
                       ", \"ms\": " + std::to_string(kv.second.first) + "}";
                first = false;
            }
        }
    ctx->force = TuneChoice{};
    for (auto &e : ev) cudaEventDestroy(e);
    dev.pool.release(); dev.partials.release(); dev.out.release(); dev.counters.release();
    if (rc) return rc;
    rep += "], \"chosen\": [";
    first = true;
    for (auto &kv : best) {
        ctx->tune[{kv.first, kv.second.bucket}] = kv.second.c;
        rep += std::string(first ? "" : ", ") + "{\"profile\": " + std::to_string(kv.first) + ", \"P\": " +
               std::to_string(kv.second.c.P) + ", \"G\": " + std::to_string(kv.second.c.G) + ", \"ms\": " +
               std::to_string(kv.second.ms) + "}";
        first = false;
    }
    rep += "]}";
    if (report && report_len) snprintf(report, report_len, "%s", rep.c_str());
    return RSR_OK;
}

int rsr_measure_fp32_peak(rsr_ctx *ctx, double *lane_ops_per_s) {
    if (!ctx || !lane_ops_per_s) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaError_t e = measure_fp32_peak(ctx->num_sms, ctx->stream, lane_ops_per_s);
    ctx->launches += 2;
    return e == cudaSuccess ? RSR_OK : cuda_fail(e, "fp32 peak");
}

int rsr_validate_program(const rsr_program *prog, uint32_t num_features) {
    if (!prog) return fail(RSR_EINVAL, "prog is null");
    EncodedProgram E;
    std::string err;
    int rc = encode_program(prog->code, prog->len, prog->const_kinds, prog->n_consts, prog->params, prog->n_params,
                            num_features, &E, &err);
    if (rc) return fail(rc, err);
    return RSR_OK;
}

int rsr_program_encoding(const rsr_program *prog, uint32_t num_features, int form, uint32_t *out, uint32_t cap,
                         uint32_t *len) {
    if (!prog || !len || (cap && !out)) return fail(RSR_EINVAL, "null argument");
    EncodedProgram E;
    std::string err;
    int rc = encode_program(prog->code, prog->len, prog->const_kinds, prog->n_consts, prog->params, prog->n_params,
                            num_features, &E, &err);
    if (rc) return fail(rc, err);
    std::vector<uint32_t> v;
    if (form == 0 || form == 3) {
        v = E.slot_code;
        if (form == 3) {
            v.push_back(E.n_slots);
            v.push_back((E.result_zero ? PF_RESULT_ZERO : 0u) | (E.needs_zero_init ? PF_NEEDS_ZERO_INIT : 0u));
        }
    } else if (form == 1) {
        v = E.reg_code;
    } else if (form == 2) {
        v = E.tape_code;
    } else if (form == 5) {
        v = {E.adj_profile < 0 ? 0xFFFFFFFFu : (uint32_t)E.adj_profile, E.adj_tape};
        for (int t = 0; t < N_STACKS; ++t) v.push_back((uint32_t)E.adj_depth[t]);
        v.insert(v.end(), E.adj_code.begin(), E.adj_code.end());
    } else if (form == 4) {
        v.resize(noalloc_max_words());
        uint32_t nw = 0, ns = 0, fl = 0;
        const char *msg = "";
        if ((rc = noalloc_slot_form(*prog, num_features, v.data(), &nw, &ns, &fl, &msg))) return fail(rc, msg);
        v.resize(nw);
        v.push_back(ns);
        v.push_back(fl);
    } else {
        return fail(RSR_EINVAL, "unknown encoding form");
    }
    *len = (uint32_t)v.size();
    for (uint32_t i = 0; i < cap && i < v.size(); ++i) out[i] = v[i];
    return RSR_OK;
}

int rsr_program_analyze(const rsr_program *prog, uint32_t num_features, rsr_program_info *info) {
    if (!prog || !info) return fail(RSR_EINVAL, "null argument");
    EncodedProgram E;
    std::string err;
    int rc = encode_program(prog->code, prog->len, prog->const_kinds, prog->n_consts, prog->params, prog->n_params,
                            num_features, &E, &err);
    if (rc) return fail(rc, err);
    for (int t = 0; t < N_STACKS; ++t) {
        info->depth_ref[t] = (uint32_t)E.depth_ref[t];
        info->depth_fast[t] = (uint32_t)E.depth_fast[t];
    }
    info->n_uops_fast = (uint32_t)E.reg_code.size();
    info->n_uops_plain = (uint32_t)E.slot_code.size() / 3;
    info->fast_profile = E.profile;
    info->flops_per_point = E.flops_per_point;
    return RSR_OK;
}

}  // extern "C"
