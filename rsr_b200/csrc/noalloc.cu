// noalloc.cu -- rsr_compute_mse_noalloc: one program's MSE with no allocation.
//
// The slot-file kernel (plain_eval_kernel) and the MSE epilogue run with all
// of their device-side state -- program descriptor, dataset descriptor, code,
// constants, work items, per-chunk partial sums and the result -- in one
// file-scope __device__ array of kNoAllocScratchBytes.  Its address is taken
// with cudaGetSymbolAddress once per device, with that device current, on the
// first call for the device, which also loads every kernel the entry point
// launches (lazy module loading would otherwise allocate on a kernel's first
// launch); that first call should come before any stream capture on the
// device.  After it, a call performs no cudaMalloc/cudaFree,
// no pinned-host or managed allocation and no C++ heap allocation on its
// success path: the program is encoded into fixed-size arrays on the host
// stack, copied into the scratch array with one cudaMemcpyAsync, and the
// result comes back with one more.
//
// The scratch array is shared by every context on the device, so calls that
// overlap in time on one device (two contexts, or two threads with different
// contexts) race on it; calls through one context are serialised by the
// context's lock and finish before returning.
#include <cuda_runtime.h>
#include <stddef.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "encoder.h"
#include "kernels.h"
#include "runtime.h"

namespace rsr {
namespace {

constexpr size_t kNoAllocScratchBytes = 256 * 1024;
constexpr uint32_t kNoAllocMaxInstr = 512;      // reference instructions per program
constexpr uint32_t kNoAllocMaxParams = 1024;    // flat parameter floats (and constants) per program
constexpr uint32_t kNoAllocMaxChunks = 4096;    // 4096-point chunks: 16,777,216 points
constexpr uint32_t kChunk = 4096;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Byte layout of the scratch array.
struct Header {
    ProgDesc prog;
    DatasetDesc ds;
    float mse;
    uint32_t pad[3];
};
constexpr size_t kOffHeader = 0;
constexpr size_t kOffCode = 256;
constexpr size_t kOffConsts = kOffCode + kNoAllocMaxInstr * 3 * sizeof(uint32_t);
constexpr size_t kOffItems = kOffConsts + kNoAllocMaxParams * sizeof(float);
constexpr size_t kOffPartials = kOffItems + kNoAllocMaxChunks * sizeof(WorkItem);
constexpr size_t kScratchUsed = kOffPartials + kNoAllocMaxChunks * sizeof(double);
static_assert(sizeof(Header) <= kOffCode, "header overlaps the code");
static_assert(kOffItems % 16 == 0 && kOffPartials % 8 == 0, "misaligned scratch sections");
static_assert(kScratchUsed <= kNoAllocScratchBytes, "scratch array too small for its stated limits");

std::mutex g_setup_mu;
unsigned char *g_scratch[kMaxDevices] = {nullptr};

// Work items of one program: chunk c covers tiles [c*tpc, min(n_tiles, (c+1)*tpc)).
__global__ void noalloc_items_kernel(WorkItem *items, uint32_t n_chunks, uint32_t n_tiles, uint32_t tpc) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_chunks) return;
    WorkItem it{};
    it.prog_begin = 0;
    it.n_progs = 1;
    it.tile_begin = c * tpc;
    it.tile_end = min(n_tiles, (c + 1) * tpc);
    it.chunk = c;
    items[c] = it;
}

// Slot form of one program (reference stack positions), written into caller
// arrays with no heap use.  Same output and the same rejections as the slot
// part of encode_program (encoder.cpp), restricted to kNoAllocMaxInstr
// instructions and kNoAllocMaxParams constants.
int encode_slots_fixed(const rsr_program &p, uint32_t num_features, uint32_t *words, uint32_t *n_words,
                       uint32_t *n_slots, uint32_t *flags, const char **err) {
    if (p.len > kNoAllocMaxInstr) { *err = "program longer than 512 instructions"; return RSR_EINVAL; }
    if (p.n_consts > kNoAllocMaxParams || p.n_params > kNoAllocMaxParams) {
        *err = "more than 1024 constants or parameter floats";
        return RSR_EINVAL;
    }
    if (p.len > 0 && !p.code) { *err = "code is null"; return RSR_EINVAL; }
    if (p.n_consts > 0 && !p.const_kinds) { *err = "const_kinds is null"; return RSR_EINVAL; }
    if (p.n_params > 0 && !p.params) { *err = "params is null"; return RSR_EINVAL; }
    uint32_t flat[kNoAllocMaxParams + 1];
    flat[0] = 0;
    for (uint32_t c = 0; c < p.n_consts; ++c) {
        if (p.const_kinds[c] > 6) { *err = "constant has unknown kind"; return RSR_EPROGRAM; }
        flat[c + 1] = flat[c] + (uint32_t)kind_width(p.const_kinds[c]);
    }
    if (flat[p.n_consts] != p.n_params) { *err = "params length does not match the constants"; return RSR_EPROGRAM; }
    // pass 1: stack replay; slots are recorded as (type << 8 | position) and
    // resolved once the per-type depths are known
    int sp[N_STACKS] = {0, 0, 0, 0, 0}, depth[N_STACKS] = {0, 0, 0, 0, 0};
    bool root = false, stale_any = false;
    uint32_t nw = 0;
    for (uint32_t pc = 0; pc < p.len; ++pc) {
        const int op = (int)(p.code[pc] & 0xFFu);
        const uint32_t a = (p.code[pc] >> 8) & 0xFFFFu;
        if (op >= N_OPCODES) { *err = "unknown opcode"; return RSR_EPROGRAM; }
        uint32_t w0, in[3] = {0, 0, 0};
        int out;
        bool stale = false;
        if (is_load(op)) {
            out = load_stack(op);
            if (out < 0) continue;  // Bool / Int loads push nothing
            if (!is_const_load(op)) {
                if (num_features && a + kStackWidth[out] > num_features) {
                    *err = "feature offset out of range";
                    return RSR_EPROGRAM;
                }
                w0 = (uint32_t)op | (a << 8);
            } else {
                if (a >= p.n_consts) { *err = "constant index out of range"; return RSR_EPROGRAM; }
                stale = p.const_kinds[a] != const_kind_for_load(op);
                w0 = stale ? (uint32_t)SLOT_NOP : ((uint32_t)op | (flat[a] << 8));
            }
        } else {
            const OpSig &g = op_sig(op);
            int cnt[N_STACKS] = {0, 0, 0, 0, 0}, base[N_STACKS];
            for (int i = 0; i < g.n_in; ++i) cnt[g.in[i]]++;
            for (int t = 0; t < N_STACKS; ++t) {
                if (sp[t] < cnt[t]) { *err = "stack underflow"; return RSR_EPROGRAM; }
                base[t] = sp[t] - cnt[t];
            }
            for (int i = 0; i < g.n_in; ++i) in[i] = ((uint32_t)g.in[i] << 8) | (uint32_t)base[g.in[i]]++;
            for (int t = 0; t < N_STACKS; ++t) sp[t] -= cnt[t];
            out = g.out;
            w0 = (uint32_t)op;
        }
        const int pos = sp[out];
        if (pos >= 32) { *err = "more than 32 values on a stack"; return RSR_EPROGRAM; }
        sp[out]++;
        if (sp[out] > depth[out]) depth[out] = sp[out];
        if (out == SF && pos == 0 && !stale) root = true;
        stale_any |= stale;
        words[nw] = w0;
        words[nw + 1] = ((uint32_t)out << 8) | (uint32_t)pos;
        words[nw + 2] = in[0];
        words[nw + 3] = in[1];
        words[nw + 4] = in[2];
        nw += 5;
    }
    // pass 2: resolve slots, compacting 5 staging words to the 3-word form
    uint32_t sbase[N_STACKS], acc = 0;
    for (int t = 0; t < N_STACKS; ++t) {
        sbase[t] = acc;
        acc += (uint32_t)depth[t] * (uint32_t)kStackWidth[t];
    }
    auto slot = [&](uint32_t tp) { return sbase[tp >> 8] + (tp & 0xFFu) * (uint32_t)kStackWidth[tp >> 8]; };
    uint32_t o = 0;
    for (uint32_t i = 0; i < nw; i += 5) {
        const uint32_t w0 = words[i], dst = slot(words[i + 1]);
        const int n_in = (w0 & 0xFFu) == SLOT_NOP || is_load((int)(w0 & 0xFFu)) ? 0 : op_sig((int)(w0 & 0xFFu)).n_in;
        const uint32_t i0 = n_in > 0 ? slot(words[i + 2]) : 0, i1 = n_in > 1 ? slot(words[i + 3]) : 0,
                       i2 = n_in > 2 ? slot(words[i + 4]) : 0;
        words[o] = w0;
        words[o + 1] = dst | (i0 << 16);
        words[o + 2] = i1 | (i2 << 16);
        o += 3;
    }
    *n_words = o;
    *n_slots = acc;
    *flags = (root ? 0u : PF_RESULT_ZERO) | (stale_any ? PF_NEEDS_ZERO_INIT : 0u);
    return RSR_OK;
}

// Set-up of the current device, once: the scratch array's address, and every
// kernel this entry point launches loaded ahead of its first real use (with
// lazy module loading a kernel's code and local memory are allocated on its
// first launch), so that no later call allocates.
int scratch_for(int device, cudaStream_t st, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return fail(RSR_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, noalloc_items_kernel)) != cudaSuccess)
            return cuda_fail(e, "noalloc kernel load");
        noalloc_items_kernel<<<1, 32, 0, st>>>(nullptr, 0u, 0u, 1u);  // no chunks: returns at once
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "noalloc kernel load");
        if ((e = preload_plain_mse(st)) != cudaSuccess) return cuda_fail(e, "noalloc kernel load");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "noalloc kernel load");
        g_scratch[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch[device];
    return RSR_OK;
}

}  // namespace

// The fixed-array slot encoder behind a diagnostic entry point
// (rsr_program_encoding, form 4), so that tests can hold it against the
// slot form of encode_program.  words must hold kNoAllocMaxInstr * 5 words.
int noalloc_slot_form(const rsr_program &p, uint32_t num_features, uint32_t *words, uint32_t *n_words,
                      uint32_t *n_slots, uint32_t *flags, const char **err) {
    return encode_slots_fixed(p, num_features, words, n_words, n_slots, flags, err);
}
uint32_t noalloc_max_words() { return kNoAllocMaxInstr * 5; }

}  // namespace rsr

using namespace rsr;

extern "C" int rsr_compute_mse_noalloc(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse) {
    if (!ctx || !prog || !mse) return fail(RSR_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    unsigned char *scratch = nullptr;
    int rc = scratch_for(ctx->device, ctx->stream, &scratch);
    if (rc) return rc;
    auto it = ctx->datasets.find(ds);
    if (it == ctx->datasets.end()) return fail(RSR_ENOTFOUND, "unknown dataset handle");
    const DatasetDesc dd = it->second->desc();
    const uint64_t n_chunks64 = (dd.n_eval + kChunk - 1) / kChunk;
    if (n_chunks64 > kNoAllocMaxChunks) return fail(RSR_EINVAL, "dataset larger than 16,777,216 points");

    // host image: header | code | constants, on the stack
    struct Image {
        Header h;
        unsigned char pad[kOffCode - sizeof(Header)];
        uint32_t code[kNoAllocMaxInstr * 5];  // 5 staging words per instruction, 3 after encoding
    };
    static_assert(offsetof(Image, code) == kOffCode, "image layout");
    Image img;
    memset(&img.h, 0, sizeof(img.h));
    uint32_t n_words = 0, n_slots = 0, flags = 0;
    const char *err = "";
    if ((rc = encode_slots_fixed(*prog, dd.num_features, img.code, &n_words, &n_slots, &flags, &err)))
        return fail(rc, err);
    const uint32_t n_chunks = (uint32_t)std::max<uint64_t>(1, n_chunks64);
    ProgDesc &pd = img.h.prog;
    pd.uop_off = 0;
    pd.uop_len = n_words;
    pd.const_off = 0;
    pd.n_consts = prog->n_params;
    pd.n_slots = n_slots;
    pd.flags = flags;
    pd.dataset = 0;
    pd.part_off = 0;
    pd.n_parts = n_chunks;
    img.h.ds = dd;
    img.h.mse = 0.0f;

    // points per lane: the largest whose per-warp staging fits 110 KB
    int P = 4;
    while (P > 1 && plain_smem_per_warp(n_words, prog->n_params, n_slots, P) > 110 * 1024) P >>= 1;
    // (an empty program stages nothing; keep the per-warp size non-zero)
    const size_t per = std::max<size_t>(16, plain_smem_per_warp(n_words, prog->n_params, n_slots, P));
    if (per > 200 * 1024) return fail(RSR_EINVAL, "program needs more shared memory than one block holds");
    const uint32_t wpb = (uint32_t)std::max<size_t>(1, std::min<size_t>(kPlainThreads / 32, (200 * 1024) / per));
    const uint32_t tile_pts = 32u * (uint32_t)P;
    const uint32_t n_tiles = (uint32_t)((dd.n_eval + tile_pts - 1) / tile_pts);
    const uint32_t tpc = kChunk / tile_pts;

    cudaStream_t st = ctx->stream;
    // header and code in one copy (the result word starts at zero with it),
    // constants in a second
    if ((e = cudaMemcpyAsync(scratch + kOffHeader, &img, kOffCode + (size_t)n_words * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "scratch upload");
    if (prog->n_params &&
        (e = cudaMemcpyAsync(scratch + kOffConsts, prog->params, (size_t)prog->n_params * sizeof(float),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_fail(e, "scratch upload");
    WorkItem *items = reinterpret_cast<WorkItem *>(scratch + kOffItems);
    noalloc_items_kernel<<<(n_chunks + 127) / 128, 128, 0, st>>>(items, n_chunks, n_tiles, tpc);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "kernel launch");

    Header *dh = reinterpret_cast<Header *>(scratch + kOffHeader);
    LaunchArgs a{};
    a.progs = &dh->prog;
    a.datasets = &dh->ds;
    a.items = items;
    a.code = reinterpret_cast<const uint32_t *>(scratch + kOffCode);
    a.consts = reinterpret_cast<const float *>(scratch + kOffConsts);
    a.partials = reinterpret_cast<double *>(scratch + kOffPartials);
    a.n_items = n_chunks;
    a.mode = MODE_MSE;
    a.smem_code_words = n_words;
    a.smem_const_floats = prog->n_params;
    a.smem_slots = n_slots;
    a.progs_per_warp = 1;
    if ((e = launch_plain(a, P, wpb, per * wpb, st)) != cudaSuccess) return cuda_fail(e, "kernel launch");
    if ((e = launch_finalize_mse(&dh->prog, &dh->ds, a.partials, 1, &dh->mse, st)) != cudaSuccess)
        return cuda_fail(e, "kernel launch");
    ctx->launches += 3;
    float m = 0.0f;
    if ((e = cudaMemcpyAsync(&m, &dh->mse, sizeof(float), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "result download");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "evaluation");
    *mse = m;
    return RSR_OK;
}
