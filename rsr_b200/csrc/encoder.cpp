// encoder.cpp -- validation, value-graph analysis and emission of the slot,
// tape and register encodings (uops.h) of a reference program.
//
// The analysis replays the reference VM's stack discipline
// (src/engine/eval/evaluator.rs:20-150, src/engine/eval/state.rs:12-37) on
// value ids instead of numbers, which gives for every instruction the stack
// positions it reads and writes and the expression tree behind stack_f[0].
#include "encoder.h"

#include <algorithm>
#include <array>
#include <cstring>

#include "../../include/rsr_gpu.h"

namespace rsr {
namespace {

struct SigTable {
    OpSig s[N_OPCODES];
    SigTable() {
        for (auto &x : s) x = OpSig{0, {-1, -1, -1}, -1, 0};
        auto set = [&](int op, std::initializer_list<int> in, int out, int fl) {
            OpSig g{0, {-1, -1, -1}, out, fl};
            for (int t : in) g.in[g.n_in++] = t;
            s[op] = g;
        };
        const int F = SF, V2 = SV2, V3 = SV3, M2 = SM2, M3 = SM3;
        // loads (pushes only; B/I loads are no-ops in eval_simd, domain.rs:286-293)
        set(LOAD_VAR_F, {}, F, 0); set(LOAD_CONST_F, {}, F, 0);
        set(LOAD_VAR_V2, {}, V2, 0); set(LOAD_CONST_V2, {}, V2, 0);
        set(LOAD_VAR_V3, {}, V3, 0); set(LOAD_CONST_V3, {}, V3, 0);
        set(LOAD_VAR_M2, {}, M2, 0); set(LOAD_CONST_M2, {}, M2, 0);
        set(LOAD_VAR_M3, {}, M3, 0); set(LOAD_CONST_M3, {}, M3, 0);
        // basic (basic/mod.rs:198-217)
        for (int op : {ADD_F, SUB_F, MUL_F, DIV_F}) set(op, {F, F}, F, 1);
        for (int op : {SIN_F, COS_F, EXP_F, SQR_F, SQRT_F, LN_F}) set(op, {F}, F, 1);
        // linalg (linalg/mod.rs:317-432)
        set(MAKE_VEC2, {F, F}, V2, 0); set(MAKE_VEC3, {F, F, F}, V3, 0);
        set(GET_X_V2, {V2}, F, 0); set(GET_Y_V2, {V2}, F, 0);
        set(GET_X_V3, {V3}, F, 0); set(GET_Y_V3, {V3}, F, 0); set(GET_Z_V3, {V3}, F, 0);
        set(ADD_V2, {V2, V2}, V2, 2); set(SUB_V2, {V2, V2}, V2, 2); set(SCALE_V2, {F, V2}, V2, 2);
        set(DOT_V2, {V2, V2}, F, 3); set(NORM_V2, {V2}, F, 4);
        set(ADD_V3, {V3, V3}, V3, 3); set(SUB_V3, {V3, V3}, V3, 3); set(SCALE_V3, {F, V3}, V3, 3);
        set(DOT_V3, {V3, V3}, F, 5); set(NORM_V3, {V3}, F, 6); set(CROSS_V3, {V3, V3}, V3, 9);
        set(MAKE_MAT2, {V2, V2}, M2, 0); set(ADD_M2, {M2, M2}, M2, 4); set(SUB_M2, {M2, M2}, M2, 4);
        set(SCALE_M2, {F, M2}, M2, 4); set(MUL_M2, {M2, M2}, M2, 12); set(MUL_M2V2, {M2, V2}, V2, 6);
        set(DET_M2, {M2}, F, 3); set(TRACE_M2, {M2}, F, 1); set(TRANSPOSE_M2, {M2}, M2, 0);
        set(INVERSE_M2, {M2}, M2, 8);
        set(MAKE_MAT3, {V3, V3, V3}, M3, 0); set(ADD_M3, {M3, M3}, M3, 9); set(SUB_M3, {M3, M3}, M3, 9);
        set(SCALE_M3, {F, M3}, M3, 9); set(MUL_M3, {M3, M3}, M3, 45); set(MUL_M3V3, {M3, V3}, V3, 15);
        set(DET_M3, {M3}, F, 14); set(TRACE_M3, {M3}, F, 2); set(TRANSPOSE_M3, {M3}, M3, 0);
        set(INVERSE_M3, {M3}, M3, 51);
    }
};
const SigTable &sigs() {
    static SigTable t;
    return t;
}

constexpr int kKindWidth[7] = {1, 0, 0, 2, 3, 4, 9};
constexpr int kMseEpilogueFlops = 3;
// Reverse sweep of the MSE epilogue: the seed 2 (pred - y) (multiply; the
// difference is the forward pass's).
constexpr int kMseEpilogueRevFlops = 1;

// Unfused FP32 lane-ops of each opcode's reverse rule (the adjoint kernel's
// work beside the forward pass), counted from the rules: one multiply per
// product term and one add per adjoint accumulation.  E.g. MulF: ga += g b,
// gb += g a (4); DivF: q = g / b, ga += q, gb -= q * out (4 + the divide);
// CrossV3: ga += b x g, gb += g x a (2 x (9 + 3)); MulM3V3: gM += g v^T
// (9 + 9), gv += M^T g (15 + 3); InverseM3: gA -= X^T G X^T with X the
// inverse (2 x 45 + 9).  A LoadConst adds its adjoint into the parameter
// sums (one add per component); a LoadVar's adjoint is dropped (0).
int reverse_flops(int op, int const_width) {
    switch (op) {
        case LOAD_CONST_F: case LOAD_CONST_V2: case LOAD_CONST_V3: case LOAD_CONST_M2: case LOAD_CONST_M3:
            return const_width;
        case ADD_F: case SUB_F: return 2;
        case MUL_F: return 4;
        case DIV_F: return 5;
        case SIN_F: case COS_F: case SQR_F: case SQRT_F: return 3;
        case EXP_F: case LN_F: return 2;
        case MAKE_VEC2: return 2;
        case MAKE_VEC3: return 3;
        case GET_X_V2: case GET_Y_V2: case GET_X_V3: case GET_Y_V3: case GET_Z_V3: return 1;
        case ADD_V2: case SUB_V2: return 4;
        case ADD_V3: case SUB_V3: return 6;
        case MAKE_MAT2: case TRANSPOSE_M2: return 4;
        case ADD_M2: case SUB_M2: return 8;
        case ADD_M3: case SUB_M3: return 18;
        case MAKE_MAT3: case TRANSPOSE_M3: return 9;
        case SCALE_V2: return 8;
        case SCALE_V3: return 12;
        case SCALE_M2: return 16;
        case SCALE_M3: return 36;
        case DOT_V2: return 8;
        case DOT_V3: return 12;
        case NORM_V2: return 5;
        case NORM_V3: return 7;
        case CROSS_V3: return 24;
        case MUL_M2: return 32;
        case MUL_M3: return 108;
        case MUL_M2V2: return 16;
        case MUL_M3V3: return 36;
        case DET_M2: return 8;
        case DET_M3: return 45;
        case TRACE_M2: return 2;
        case TRACE_M3: return 3;
        case INVERSE_M2: return 28;
        case INVERSE_M3: return 99;
        default: return 0;
    }
}

struct Node {
    int opcode = 0;
    uint32_t arg = 0;    // feature offset (LoadVar) or flat param offset (LoadConst)
    int out = -1;        // result stack
    int n_in = 0;
    int in[3] = {-1, -1, -1};
    int pos = 0;         // reference stack position of the result
    bool stale = false;  // LoadConst of a mismatched variant: writes nothing
    int alias = -1;      // stale: node whose value sits in that slot (-1: zero)
};

bool leaf(const Node &n) { return is_load(n.opcode) && !n.stale; }

// Values that an opcode's reverse rule reads (the adjoint kernel's
// tape_reverse): bit k < 3 for input k, bit 3 for the output.
int reverse_reads(int op) {
    switch (op) {
        case MUL_F: return 1 | 2;
        case DIV_F: return 2 | 8;
        case SIN_F: case COS_F: case SQR_F: case LN_F: return 1;
        case EXP_F: case SQRT_F: return 8;
        case SCALE_V2: case SCALE_V3: case SCALE_M2: case SCALE_M3: return 1 | 2;
        case DOT_V2: case DOT_V3: case CROSS_V3: return 1 | 2;
        case NORM_V2: case NORM_V3: return 1 | 8;
        case MUL_M2: case MUL_M3: case MUL_M2V2: case MUL_M3V3: return 1 | 2;
        case DET_M2: case DET_M3: return 1;
        case INVERSE_M2: case INVERSE_M3: return 1 | 8;
        default: return 0;
    }
}

// First-fit allocation of runs of `width` slots over time intervals: a slot
// is free for an interval starting at t0 when its last holder ended before t0.
struct SlotPool {
    std::vector<int> busy_until;  // per slot, -1 = never used
    uint32_t take(int width, int t0, int t1) {
        for (uint32_t s = 0;; ++s) {
            bool ok = true;
            for (int k = 0; k < width && ok; ++k)
                ok = s + k >= busy_until.size() || busy_until[s + k] < t0;
            if (!ok) continue;
            if (busy_until.size() < s + width) busy_until.resize(s + width, -1);
            for (int k = 0; k < width; ++k) busy_until[s + k] = t1;
            return s;
        }
    }
};

// Working storage of one encoding thread, kept between programs so that an
// encoding allocates only while a program is larger than any before it.
struct Scratch {
    std::vector<uint32_t> flat;
    std::vector<Node> nodes;
    std::vector<int> instr_node, work;
    std::vector<char> live;
    // accumulator form
    std::vector<uint32_t> writes, code;
    std::vector<int> size;
    // tape form
    std::vector<int> idx, pos, vend, astart;
    std::vector<uint32_t> vs, as;
    SlotPool vals;
};
thread_local Scratch tls;

// Tape form for the adjoint kernel.  Live nodes in program order; node t runs
// forward at time t and in reverse at time 2N-1-t.  A value lives from its
// definition to its last forward read, or to the reverse step of the last
// node whose reverse rule reads it; an adjoint lives from the reverse step of
// its latest consumer (its first contribution) to its own reverse step.
// Values and adjoints share one slot file, allocated first-fit by lifetime
// in order of start time; the input through which an adjoint receives its
// first contribution carries kTapeZeroFirst, so the reverse step clears those
// slots before adding to them (the root's adjoint is written by the seed).
// Feature loads have no tape entry: their value slot is kTapeFeature |
// feature offset, read from the dataset where it is used, and their adjoint
// field is a sink past the slot file, which takes contributions and is never
// read; the reverse rules of matrix products and inverses skip a feature
// matrix's contributions outright, so the sink is as wide as the widest
// feature that other rules send contributions from.  Words: header (result value slot, result adjoint
// slot), then 5 per node: op | aux << 8 | out_width << 28 (aux: the load's
// operand, a copy's has_alias | width << 1, else the input widths in three
// nibbles), vo | ao << 16, and vi | ai << 16 for inputs 0..2.
void emit_tape(const std::vector<Node> &nodes, const std::vector<char> &live, int root, EncodedProgram *E) {
    std::vector<int> &idx = tls.idx;  // tape order -> node id
    std::vector<int> &pos = tls.pos;
    idx.clear();
    pos.assign(nodes.size(), -1);
    for (size_t i = 0; i < nodes.size(); ++i)
        if (live[i]) {
            pos[i] = (int)idx.size();
            idx.push_back((int)i);
        }
    const int N = (int)idx.size();
    const int rev = 2 * N - 1;
    std::vector<int> &vend = tls.vend, &astart = tls.astart;
    vend.assign(N, -1);
    astart.assign(N, 1 << 30);
    // first[u]: (consumer, input) of u's first adjoint contribution -- the
    // latest consumer in program order, its lowest input that reads u
    std::vector<int> &first = tls.work;
    first.assign(2 * (size_t)N, -1);
    // sink_width: the widest feature whose adjoint contributions are made
    // (the matrix input of a matrix product or inverse skips them)
    uint32_t sink_width = 0;
    for (int t = 0; t < N; ++t) {
        const Node &n = nodes[idx[t]];
        const int rr = n.stale ? 0 : reverse_reads(n.opcode);
        if (rr & 8) vend[t] = std::max(vend[t], rev - t);
        auto use = [&](int in_node, int k) {
            const int u = pos[in_node];
            vend[u] = std::max(vend[u], t);                                // forward read
            if (k >= 0 && ((rr >> k) & 1)) vend[u] = std::max(vend[u], rev - t);
            astart[u] = std::min(astart[u], rev - t);                      // adjoint contribution
            if (first[2 * u] != t) {
                first[2 * u] = t;
                first[2 * u + 1] = k < 0 ? 0 : k;
            }
            const Node &un = nodes[in_node];
            if (!un.stale && is_load(un.opcode) && !is_const_load(un.opcode)) {
                const int op = n.stale ? -1 : n.opcode;
                const bool skipped = ((op == MUL_M2V2 || op == MUL_M3V3) && k == 0) || op == MUL_M2 ||
                                     op == MUL_M3 || op == INVERSE_M2 || op == INVERSE_M3;
                if (!skipped) sink_width = std::max(sink_width, (uint32_t)kStackWidth[un.out]);
            }
        };
        if (n.stale) {
            if (n.alias >= 0) use(n.alias, -1);
        } else {
            for (int k = 0; k < n.n_in; ++k) use(n.in[k], k);
        }
    }
    const int rt = root >= 0 ? pos[root] : -1;
    if (rt >= 0) {
        vend[rt] = std::max(vend[rt], N);          // read for the prediction
        astart[rt] = std::min(astart[rt], N - 1);  // seeded before the reverse sweep
    }
    auto is_feature = [&](int t) {
        const Node &n = nodes[idx[t]];
        return !n.stale && is_load(n.opcode) && !is_const_load(n.opcode) && n.arg < kTapeFeature;
    };
    // one slot file: every value and adjoint interval, first-fit in order of
    // start time (the order that packs intervals of one width optimally)
    struct Interval { int t0, t1, w, node; bool adj; };
    std::vector<Interval> iv;
    iv.reserve(2 * (size_t)N);
    for (int t = 0; t < N; ++t) {
        if (is_feature(t)) continue;
        const int w = kStackWidth[nodes[idx[t]].out];
        iv.push_back({t, std::max(vend[t], t), w, t, false});
        if (astart[t] <= rev - t) iv.push_back({astart[t], rev - t, w, t, true});
    }
    std::stable_sort(iv.begin(), iv.end(), [](const Interval &a, const Interval &b) { return a.t0 < b.t0; });
    SlotPool &slots = tls.vals;
    slots.busy_until.clear();
    std::vector<uint32_t> &vs = tls.vs, &as = tls.as;
    vs.assign(N, 0);
    as.assign(N, 0);
    for (const Interval &x : iv) (x.adj ? as : vs)[x.node] = slots.take(x.w, x.t0, x.t1);
    const uint32_t sink = (uint32_t)slots.busy_until.size();
    for (int t = 0; t < N; ++t)
        if (is_feature(t)) {
            vs[t] = kTapeFeature | nodes[idx[t]].arg;  // read from the dataset where used
            as[t] = sink;
        }
    if (rt >= 0 && is_feature(rt)) sink_width = std::max(sink_width, (uint32_t)kStackWidth[nodes[idx[rt]].out]);  // the seed
    E->n_tape_val = sink + sink_width;
    E->n_tape_adj = 0;
    E->tape_code.clear();
    E->tape_code.push_back(rt >= 0 ? vs[rt] : 0xFFFFFFFFu);
    E->tape_code.push_back(rt >= 0 ? as[rt] : 0u);
    // input k of node t carries the clear flag when it is the first
    // contribution to that value's adjoint (never the root's: the seed is)
    auto in_word = [&](int t, int k, int in_node) {
        const int u = pos[in_node];
        uint32_t a = as[u];
        if (!is_feature(u) && u != rt && first[2 * u] == t && first[2 * u + 1] == k) a |= kTapeZeroFirst;
        return vs[u] | (a << 16);
    };
    for (int t = 0; t < N; ++t) {
        const Node &n = nodes[idx[t]];
        if (is_feature(t)) continue;  // no tape entry: consumers read the dataset
        uint32_t w0, in[3] = {0, 0, 0};
        if (n.stale) {
            // copy of the value left in that slot, or zero; aux = has_alias | width << 1
            w0 = (uint32_t)SLOT_NOP | (((n.alias >= 0 ? 1u : 0u) | ((uint32_t)kStackWidth[n.out] << 1)) << 8);
            if (n.alias >= 0) in[0] = in_word(t, 0, n.alias);
        } else if (is_load(n.opcode)) {
            w0 = (uint32_t)n.opcode | (n.arg << 8);
        } else {
            uint32_t widths = 0;
            for (int k = 0; k < n.n_in; ++k) {
                in[k] = in_word(t, k, n.in[k]);
                widths |= (uint32_t)kStackWidth[nodes[n.in[k]].out] << (4 * k);
            }
            w0 = (uint32_t)n.opcode | (widths << 8);
        }
        w0 |= (uint32_t)kStackWidth[n.out] << 28;
        E->tape_code.push_back(w0);
        E->tape_code.push_back(vs[t] | (as[t] << 16));
        E->tape_code.push_back(in[0]);
        E->tape_code.push_back(in[1]);
        E->tape_code.push_back(in[2]);
    }
}

}  // namespace

const OpSig &op_sig(int opcode) { return sigs().s[opcode]; }
bool is_load(int opcode) { return opcode >= 0 && opcode <= LOAD_CONST_M3; }
bool is_const_load(int opcode) { return is_load(opcode) && (opcode & 1); }
int kind_width(int kind) { return (kind >= 0 && kind < 7) ? kKindWidth[kind] : 0; }
int load_stack(int opcode) {
    switch (opcode) {
        case LOAD_VAR_F: case LOAD_CONST_F: return SF;
        case LOAD_VAR_V2: case LOAD_CONST_V2: return SV2;
        case LOAD_VAR_V3: case LOAD_CONST_V3: return SV3;
        case LOAD_VAR_M2: case LOAD_CONST_M2: return SM2;
        case LOAD_VAR_M3: case LOAD_CONST_M3: return SM3;
        default: return -1;
    }
}
int const_kind_for_load(int opcode) {
    switch (opcode) {
        case LOAD_CONST_F: return 0; case LOAD_CONST_V2: return 3; case LOAD_CONST_V3: return 4;
        case LOAD_CONST_M2: return 5; case LOAD_CONST_M3: return 6; default: return -1;
    }
}

namespace {

// ---------------------------------------------------- accumulator form
enum OpClass { C_LOAD, C_BIN, C_DOT, C_SCALE, C_MULMV, C_UNARY_F, C_GET, C_NORM, C_DET, C_TRACE, C_MAT_UN, C_MAKE };

OpClass op_class(int op) {
    switch (op) {
        case ADD_F: case SUB_F: case MUL_F: case DIV_F: case ADD_V2: case SUB_V2: case ADD_V3: case SUB_V3:
        case CROSS_V3: case ADD_M2: case SUB_M2: case MUL_M2: case ADD_M3: case SUB_M3: case MUL_M3:
            return C_BIN;
        case DOT_V2: case DOT_V3: return C_DOT;
        case SCALE_V2: case SCALE_V3: case SCALE_M2: case SCALE_M3: return C_SCALE;
        case MUL_M2V2: case MUL_M3V3: return C_MULMV;
        case SIN_F: case COS_F: case EXP_F: case SQR_F: case SQRT_F: case LN_F: return C_UNARY_F;
        case GET_X_V2: case GET_Y_V2: case GET_X_V3: case GET_Y_V3: case GET_Z_V3: return C_GET;
        case NORM_V2: case NORM_V3: return C_NORM;
        case DET_M2: case DET_M3: return C_DET;
        case TRACE_M2: case TRACE_M3: return C_TRACE;
        case TRANSPOSE_M2: case TRANSPOSE_M3: case INVERSE_M2: case INVERSE_M3: return C_MAT_UN;
        case MAKE_VEC2: case MAKE_VEC3: case MAKE_MAT2: case MAKE_MAT3: return C_MAKE;
        default: return C_LOAD;
    }
}

// (binary-op index within its type's block, index of the reversed form)
struct BinIdx { int op, rop; };
BinIdx bin_index(int opcode) {
    switch (opcode) {
        case ADD_F: return {0, 0};  case SUB_F: return {1, 2};  case MUL_F: return {3, 3};  case DIV_F: return {4, 5};
        case ADD_V2: return {0, 0}; case SUB_V2: return {1, 2};
        case ADD_V3: return {0, 0}; case SUB_V3: return {1, 2}; case CROSS_V3: return {3, 4};
        case ADD_M2: case ADD_M3: return {0, 0};
        case SUB_M2: case SUB_M3: return {1, 2};
        case MUL_M2: case MUL_M3: return {3, 4};
        default: return {0, 0};
    }
}

class AccEmitter {
   public:
    explicit AccEmitter(const std::vector<Node> &nodes)
        : code(tls.code), nodes_(nodes), writes_(tls.writes), size_(tls.size) {
        code.clear();
        writes_.assign(nodes.size(), 0);
        size_.assign(nodes.size(), 0);
    }

    bool analyze(int id) {  // accumulator write sets and subtree sizes; false if unsupported
        const Node &n = nodes_[id];
        if (is_load(n.opcode)) {
            if (n.stale) return false;
            writes_[id] = 1u << n.out;
            size_[id] = 1;
            types_ |= 1u << n.out;
            return true;
        }
        uint32_t w = 1u << n.out;
        int sz = 1;
        for (int i = 0; i < n.n_in; ++i) {
            if (!analyze(n.in[i])) return false;
            w |= writes_[n.in[i]];
            sz += size_[n.in[i]];
        }
        writes_[id] = w;
        size_[id] = sz;
        types_ |= w;
        return true;
    }

    // Emits the subtree of `id`; leaves its value in the accumulator of its type.
    void gen(int id) {
        const Node &n = nodes_[id];
        const int op = n.opcode;
        if (is_load(op)) {
            emit(kBlockBase[n.out] + (is_const_load(op) ? KV_LDC : KV_LDX), n.arg);
            return;
        }
        const Node *in[3] = {n.n_in > 0 ? &nodes_[n.in[0]] : nullptr, n.n_in > 1 ? &nodes_[n.in[1]] : nullptr,
                             n.n_in > 2 ? &nodes_[n.in[2]] : nullptr};
        switch (op_class(op)) {
            case C_BIN: {
                const int t = n.out, base = kBlockBase[t] + KV_BIN;
                const BinIdx b = bin_index(op);
                const bool la = leaf(*in[0]), lb = leaf(*in[1]);
                if (lb) {                       // acc = a op leaf
                    gen(n.in[0]);
                    emit(base + 3 * b.op + src_of(*in[1]), in[1]->arg);
                } else if (la) {                // acc = leaf op b
                    gen(n.in[1]);
                    emit(base + 3 * b.rop + src_of(*in[0]), in[0]->arg);
                } else if (size_[n.in[1]] > size_[n.in[0]]) {  // b first: acc = a op S[b]
                    gen(n.in[1]);
                    const int slot = push(t);
                    gen(n.in[0]);
                    emit(base + 3 * b.op + SRC_S, slot);
                    pop(t);
                } else {                        // a first: acc = S[a] op b
                    gen(n.in[0]);
                    const int slot = push(t);
                    gen(n.in[1]);
                    emit(base + 3 * b.rop + SRC_S, slot);
                    pop(t);
                }
                break;
            }
            case C_DOT: {
                const int t = in[0]->out, nb = kBinOps[t];
                const int base = kBlockBase[t] + kv_dot(nb);
                if (leaf(*in[1])) { gen(n.in[0]); emit(base + src_of(*in[1]), in[1]->arg); }
                else if (leaf(*in[0])) { gen(n.in[1]); emit(base + src_of(*in[0]), in[0]->arg); }
                else {
                    gen(n.in[0]);
                    const int slot = push(t);
                    gen(n.in[1]);
                    emit(base + SRC_S, slot);
                    pop(t);
                }
                break;
            }
            case C_SCALE: {  // in[0] scalar, in[1] vector/matrix
                const int t = n.out;
                const int base = kBlockBase[t] + (t == SM2 || t == SM3 ? (int)KM_SCALE : kv_scale(kBinOps[t]));
                cross_type(n, base, SF, t);
                break;
            }
            case C_MULMV: {  // in[0] matrix, in[1] vector
                const int t = n.out, tm = in[0]->out;
                const int w = t == SV2 ? 2 : 3;
                cross_type(n, kBlockBase[t] + kv_mulm(kBinOps[t], w), tm, t);
                break;
            }
            case C_UNARY_F:
                gen(n.in[0]);
                emit(K_F_UN + (op - SIN_F), 0);
                break;
            case C_NORM: case C_GET: {
                const int t = in[0]->out, nb = kBinOps[t];
                gen(n.in[0]);
                int k = kv_norm(nb);
                if (op == GET_X_V2 || op == GET_X_V3) k += 1;
                if (op == GET_Y_V2 || op == GET_Y_V3) k += 2;
                if (op == GET_Z_V3) k += 3;
                emit(kBlockBase[t] + k, 0);
                break;
            }
            case C_DET: case C_TRACE: case C_MAT_UN: {
                const int t = in[0]->out;
                gen(n.in[0]);
                int k = op == DET_M2 || op == DET_M3 ? KM_DET : op == TRACE_M2 || op == TRACE_M3 ? KM_TRACE
                      : op == TRANSPOSE_M2 || op == TRANSPOSE_M3 ? KM_TRANSPOSE : KM_INVERSE;
                emit(kBlockBase[t] + k, 0);
                break;
            }
            case C_MAKE: {  // operands pushed in order, the last stays in its accumulator
                const int tin = in[0]->out, t = n.out;
                int first = -1;
                for (int i = 0; i + 1 < n.n_in; ++i) {
                    gen(n.in[i]);
                    const int slot = push(tin);
                    if (i == 0) first = slot;
                }
                gen(n.in[n.n_in - 1]);
                const int k = t == SM2 || t == SM3 ? (int)KM_MAKE : kv_make(kBinOps[t], t == SV2 ? 2 : 3);
                emit(kBlockBase[t] + k, (uint32_t)first);
                for (int i = 0; i + 1 < n.n_in; ++i) pop(tin);
                break;
            }
            case C_LOAD: break;
        }
    }

    uint32_t writes_of(int id) const { return writes_[id]; }
    int size_of(int id) const { return size_[id]; }

    std::vector<uint32_t> &code;
    int max_sp[N_STACKS] = {0, 0, 0, 0, 0};
    uint32_t types_ = 0;  // accumulator types used

   private:
    // Ops whose second operand has another type (Scale: scalar, MulMV:
    // matrix): the operand of the result type is evaluated last; the other
    // one is fused if it is a leaf, kept in its accumulator if the result
    // subtree does not overwrite it, pushed to its stack otherwise.
    // base + {0 A, 1 X, 2 C, 3 S}.
    void cross_type(const Node &n, int base, int tother, int t) {
        const Node &o = nodes_[n.in[0]];
        if (leaf(o)) {
            gen(n.in[1]);
            emit(base + 1 + src_of(o), o.arg);
            return;
        }
        gen(n.in[0]);
        if (writes_[n.in[1]] & (1u << tother)) {
            const int slot = push(tother);
            gen(n.in[1]);
            emit(base + 3, slot);
            pop(tother);
        } else {
            gen(n.in[1]);
            emit(base + 0, 0);
        }
        (void)t;
    }
    static int src_of(const Node &leafn) { return is_const_load(leafn.opcode) ? SRC_C : SRC_X; }
    int push(int t) {
        const int slot = sp_[t]++;
        max_sp[t] = std::max(max_sp[t], sp_[t]);
        emit(kBlockBase[t] + KV_PUSH, (uint32_t)slot);
        return slot;
    }
    void pop(int t) { sp_[t]--; }
    void emit(int kind, uint32_t arg) { code.push_back(uop_word((uint32_t)kind, arg)); }

    const std::vector<Node> &nodes_;
    std::vector<uint32_t> &writes_;
    std::vector<int> &size_;
    int sp_[N_STACKS] = {0, 0, 0, 0, 0};
};

// Register-adjoint code (uops.h, kAdjHeaderWords) of a tree an AccEmitter
// has analysed: the accumulator form's evaluation order, a load directly
// after a PUSH fused into the PUSH's word, every PUSH to its own stack slot,
// tape stores of the forward values the reverse rules read (carried by the
// op's own forward entry where the value is of the op's type, else a TAPE
// entry), and one reverse entry per micro-op.  An input value that is still a plain feature or constant load
// is not taped: its reference names the feature or constant (kTapeRefX,
// kTapeRefC).  Tape references hold (first | second << 16):
//   F MUL: A before; DIV: A after; RDIV: A before, A after;
//   sin cos sqr ln: A before; exp sqrt: A after;
//   V CROSS/RCROSS, M MUL/RMUL, DOT, DET: the accumulator before;
//   SCALE, MULM: the accumulator before, and (A forms) the other operand's
//   accumulator (A_F, or the matrix);
//   NORM: -, the vector (the rule recomputes the norm from it);
//   INVERSE: after, before.
int kind_block(int kind);

class AdjEmitter {
   public:
    AdjEmitter(const std::vector<Node> &nodes, const AccEmitter &an) : nodes_(nodes), an_(an) {}

    void gen(int id) {
        const Node &n = nodes_[id];
        const int opc = n.opcode;
        if (is_load(opc)) {
            op(kBlockBase[n.out] + (is_const_load(opc) ? KV_LDC : KV_LDX), n.arg);
            return;
        }
        const Node *in[3] = {n.n_in > 0 ? &nodes_[n.in[0]] : nullptr, n.n_in > 1 ? &nodes_[n.in[1]] : nullptr,
                             n.n_in > 2 ? &nodes_[n.in[2]] : nullptr};
        switch (op_class(opc)) {
            case C_BIN: {
                const int t = n.out, base = kBlockBase[t] + KV_BIN;
                const BinIdx b = bin_index(opc);
                int j, src;
                uint32_t arg;
                if (leaf(*in[1])) {
                    gen(n.in[0]);
                    j = b.op, src = src_of(*in[1]), arg = in[1]->arg;
                } else if (leaf(*in[0])) {
                    gen(n.in[1]);
                    j = b.rop, src = src_of(*in[0]), arg = in[0]->arg;
                } else if (an_.size_of(n.in[1]) > an_.size_of(n.in[0])) {
                    gen(n.in[1]);
                    arg = (uint32_t)push(t);
                    gen(n.in[0]);
                    j = b.op, src = SRC_S;
                } else {
                    gen(n.in[0]);
                    arg = (uint32_t)push(t);
                    gen(n.in[1]);
                    j = b.rop, src = SRC_S;
                }
                const int kind = base + 3 * j + src;
                const bool before = (t == SF && (j == 3 || j == 5)) || (t != SF && t != SV2 && (j == 3 || j == 4));
                const bool after = t == SF && (j == 4 || j == 5);
                uint32_t ta = 0, tb = 0;
                if (before) ta = tape_in(t);
                if (after) (before ? tb : ta) = take(t);
                op(kind, arg, ta, tb);
                if (after) store_after(t, before ? tb : ta);
                break;
            }
            case C_DOT: {
                const int t = in[0]->out;
                const int base = kBlockBase[t] + kv_dot(kBinOps[t]);
                uint32_t arg;
                int src;
                if (leaf(*in[1])) { gen(n.in[0]); src = src_of(*in[1]); arg = in[1]->arg; }
                else if (leaf(*in[0])) { gen(n.in[1]); src = src_of(*in[0]); arg = in[0]->arg; }
                else { gen(n.in[0]); arg = (uint32_t)push(t); gen(n.in[1]); src = SRC_S; }
                const uint32_t ta = tape_in(t);
                op(base + src, arg, ta);
                break;
            }
            case C_SCALE: {
                const int t = n.out;
                cross_type(n, kBlockBase[t] + (t == SM2 || t == SM3 ? (int)KM_SCALE : kv_scale(kBinOps[t])), SF, t);
                break;
            }
            case C_MULMV: {
                const int t = n.out;
                cross_type(n, kBlockBase[t] + kv_mulm(kBinOps[t], t == SV2 ? 2 : 3), in[0]->out, t);
                break;
            }
            case C_UNARY_F: {
                gen(n.in[0]);
                const int u = opc - SIN_F;  // sin cos exp sqr sqrt ln
                const bool after = u == 2 || u == 4;
                const uint32_t ta = after ? take(SF) : tape_in(SF);
                op(K_F_UN + u, 0, ta);
                if (after) store_after(SF, ta);
                break;
            }
            case C_NORM: case C_GET: {
                const int t = in[0]->out, nb = kBinOps[t];
                gen(n.in[0]);
                int k = kv_norm(nb);
                if (opc == GET_X_V2 || opc == GET_X_V3) k += 1;
                if (opc == GET_Y_V2 || opc == GET_Y_V3) k += 2;
                if (opc == GET_Z_V3) k += 3;
                if (op_class(opc) == C_NORM) {
                    // the reverse rule recomputes the norm from the vector
                    const uint32_t tb = tape_in(t);
                    op(kBlockBase[t] + k, 0, 0, tb);
                } else {
                    op(kBlockBase[t] + k, 0);
                }
                break;
            }
            case C_DET: case C_TRACE: case C_MAT_UN: {
                const int t = in[0]->out;
                gen(n.in[0]);
                if (opc == DET_M2 || opc == DET_M3) {
                    const uint32_t ta = tape_in(t);
                    op(kBlockBase[t] + KM_DET, 0, ta);
                } else if (opc == TRACE_M2 || opc == TRACE_M3) {
                    op(kBlockBase[t] + KM_TRACE, 0);
                } else if (opc == TRANSPOSE_M2 || opc == TRANSPOSE_M3) {
                    op(kBlockBase[t] + KM_TRANSPOSE, 0);
                } else {
                    const uint32_t tb = tape_in(t), ta = take(t);
                    op(kBlockBase[t] + KM_INVERSE, 0, ta, tb);
                    store_after(t, ta);
                }
                break;
            }
            case C_MAKE: {  // operands pushed to consecutive slots reserved up front
                const int tin = in[0]->out, t = n.out;
                const int first = n_push[tin];
                n_push[tin] += n.n_in - 1;
                for (int i = 0; i + 1 < n.n_in; ++i) {
                    gen(n.in[i]);
                    op(kBlockBase[tin] + KV_PUSH, (uint32_t)(first + i));
                }
                gen(n.in[n.n_in - 1]);
                const int k = t == SM2 || t == SM3 ? (int)KM_MAKE : kv_make(kBinOps[t], t == SV2 ? 2 : 3);
                op(kBlockBase[t] + k, (uint32_t)first);
                break;
            }
            case C_LOAD: break;
        }
    }

    // The code: header, forward entries, reverse entries in reverse order.
    void finish(std::vector<uint32_t> *out) const {
        out->clear();
        out->push_back((uint32_t)(fwd.size() / 2));
        out->push_back((uint32_t)(rev.size() / 2));
        out->insert(out->end(), fwd.begin(), fwd.end());
        for (size_t i = rev.size(); i >= 2; i -= 2) {
            out->push_back(rev[i - 2]);
            out->push_back(rev[i - 1]);
        }
    }

    std::vector<uint32_t> fwd, rev;
    uint32_t tape = 0;
    int n_push[N_STACKS] = {0, 0, 0, 0, 0};

   private:
    // Scale / mat-vec: the operand of another type (tother) is fused when it
    // is a leaf, pushed when the result subtree overwrites its accumulator,
    // else read from its accumulator (A form, taped); base + {0 A, 1 X, 2 C, 3 S}.
    void cross_type(const Node &n, int base, int tother, int t) {
        const Node &o = nodes_[n.in[0]];
        if (leaf(o)) {
            gen(n.in[1]);
            const uint32_t ta = tape_in(t);
            op(base + 1 + src_of(o), o.arg, ta);
            return;
        }
        gen(n.in[0]);
        if (an_.writes_of(n.in[1]) & (1u << tother)) {
            const int slot = push(tother);
            gen(n.in[1]);
            const uint32_t ta = tape_in(t);
            op(base + 3, (uint32_t)slot, ta);
        } else {
            gen(n.in[1]);
            const uint32_t ta = tape_in(t), tb = tape_in(tother);
            op(base + 0, 0, ta, tb);
        }
    }
    static int src_of(const Node &leafn) { return is_const_load(leafn.opcode) ? SRC_C : SRC_X; }
    uint32_t take(int t) {
        const uint32_t s = tape;
        tape += (uint32_t)kStackWidth[t];
        return s;
    }
    // A TAPE entry of its own: a store the op's entry cannot carry.
    void tape_entry(int t, uint32_t slot) {
        fwd.push_back(uop_word((uint32_t)kTapeKind[t], slot));
        fwd.push_back(kNoTapes);
        push_open_ = false;
    }
    // Tape store of accumulator t after the op just emitted: carried by that
    // op's entry when it is the op's own type.
    void store_after(int t, uint32_t slot) {
        uint32_t &tapes = fwd.back();
        if (kind_block((int)(fwd[fwd.size() - 2] & 0xFFu)) == t && (tapes >> 16) == kNoTape)
            tapes = (tapes & 0xFFFFu) | (slot << 16);
        else
            tape_entry(t, slot);
    }
    // Reference to the current value of accumulator t as an input of the next
    // op: the feature or constant it was loaded from when no op has changed
    // it since, else a new tape slot, stored before the op runs (by the op's
    // entry, or by a TAPE entry for another type's accumulator).
    uint32_t tape_in(int t) {
        if (plain_[t]) return plain_[t];
        const uint32_t s = take(t);
        pending_[n_pending_++] = {t, s};
        return s;
    }
    void op(int kind, uint32_t arg, uint32_t ta = 0, uint32_t tb = 0) {
        const int t = kind_block(kind), k = kind - kBlockBase[t];
        uint32_t before = kNoTape;
        for (int q = 0; q < n_pending_; ++q) {
            if (pending_[q].t == t && before == kNoTape) before = pending_[q].slot;
            else tape_entry(pending_[q].t, pending_[q].slot);
        }
        n_pending_ = 0;
        const bool load = k == KV_LDX || k == KV_LDC;
        if (load && push_open_ && arg < (1u << kLdOffsetBits)) {
            // a load right after a PUSH joins the PUSH's word (push_load_arg),
            // in the forward stream and in the PUSH's reverse entry, whose
            // rule then also reverses the load
            const uint32_t pw = fwd[fwd.size() - 2];
            const uint32_t fused = uop_word(pw & 0xFFu, push_load_arg((pw >> 8) & 15u, (uint32_t)t + 1u,
                                                                      k == KV_LDC ? 1u : 0u, arg));
            fwd[fwd.size() - 2] = fused;
            rev[rev.size() - 2] = fused;
        } else {
            fwd.push_back(uop_word((uint32_t)kind, arg));
            fwd.push_back(before | (kNoTape << 16));
            rev.push_back(uop_word((uint32_t)kind, arg));
            rev.push_back(ta | (tb << 16));
        }
        push_open_ = k == KV_PUSH && !load;
        const bool fits = arg + (uint32_t)kStackWidth[t] <= kTapeRefIndex;
        if (k == KV_LDX) plain_[t] = fits ? kTapeRefX | arg : 0u;
        else if (k == KV_LDC) plain_[t] = fits ? kTapeRefC | arg : 0u;
        else if (k != KV_PUSH) plain_[t] = plain_[SF] = 0u;  // the op's own type and A_F may change
    }
    uint32_t plain_[N_STACKS] = {0, 0, 0, 0, 0};
    bool push_open_ = false;  // the last forward entry is a PUSH without a load
    struct Pending { int t; uint32_t slot; };
    Pending pending_[2];      // tape stores before the next op (at most two: A-form scale / mat-vec)
    int n_pending_ = 0;
    int push(int t) {
        const int slot = n_push[t]++;
        op(kBlockBase[t] + KV_PUSH, (uint32_t)slot);
        return slot;
    }

    const std::vector<Node> &nodes_;
    const AccEmitter &an_;
};

// Peephole passes over the accumulator form: a load directly followed by a
// unary op on the loaded value becomes the op's operand load, and a PUSH
// directly followed by a load carries the load.
int kind_block(int kind) { return kind >= K_M3 ? SM3 : kind >= K_M2 ? SM2 : kind >= K_V3 ? SV3 : kind >= K_V2 ? SV2 : SF; }

int post_op_of(int kind, int t) {
    const int k = kind - kBlockBase[t];
    if (t == SF) return (k >= K_F_UN - K_F && k < K_F_END - K_F) ? k - (K_F_UN - K_F) + 1 : 0;
    if (t == SV2 || t == SV3) {
        const int kn = kv_norm(kBinOps[t]), w = kStackWidth[t];
        return (k >= kn && k <= kn + w) ? k - kn + 1 : 0;
    }
    if (k == KM_DET) return 1;
    if (k == KM_TRACE) return 2;
    if (k == KM_TRANSPOSE) return 3;
    if (k == KM_INVERSE) return 4;
    return 0;
}

bool is_unary_kind(int kind, int t) { return post_op_of(kind, t) != 0; }

// The passes rewrite the code in place: a word is written at or before the
// position just read, after the words it depends on were read.
void fuse_loads(std::vector<uint32_t> *code) {
    std::vector<uint32_t> &c = *code;
    // 1. a load directly followed by a unary op on the loaded value
    size_t w = 0;
    for (size_t i = 0; i < c.size(); ++i) {
        const int kind = (int)(c[i] & 0xFFu);
        const int t = kind_block(kind), k = kind - kBlockBase[t];
        if ((k == KV_LDX || k == KV_LDC) && i + 1 < c.size()) {
            const int kn = (int)(c[i + 1] & 0xFFu);
            if (kind_block(kn) == t && is_unary_kind(kn, t) && (c[i] >> 8) < (1u << kLdOffsetBits)) {
                c[w++] = uop_word((uint32_t)kn, unary_load_arg(c[i] >> 8, k == KV_LDX ? 1u : 2u));
                ++i;
                continue;
            }
        }
        c[w++] = c[i];
    }
    c.resize(w);
    // 2. a PUSH directly followed by a load
    w = 0;
    for (size_t i = 0; i < c.size(); ++i) {
        const int kind = (int)(c[i] & 0xFFu);
        const int t = kind_block(kind), k = kind - kBlockBase[t];
        if (k == KV_PUSH && i + 1 < c.size()) {
            const int kn = (int)(c[i + 1] & 0xFFu), tn = kind_block(kn), kk = kn - kBlockBase[tn];
            if ((kk == KV_LDX || kk == KV_LDC) && (c[i + 1] >> 8) < (1u << kLdOffsetBits)) {
                c[w++] = uop_word((uint32_t)kind, push_load_arg(c[i] >> 8, (uint32_t)tn + 1u, kk == KV_LDC ? 1u : 0u,
                                                               c[i + 1] >> 8));
                ++i;
                continue;
            }
        }
        c[w++] = c[i];
    }
    c.resize(w);
}

void set_err(std::string *err, const std::string &m) {
    if (err) *err = m;
}

}  // namespace

int encode_program(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t n_consts,
                   const float *params, uint32_t n_params, uint32_t num_features, EncodedProgram *out,
                   std::string *err, bool fuse, unsigned forms) {
    EncodedProgram &E = *out;
    E.reset();
    if (len > 0 && !code) { set_err(err, "code is null"); return RSR_EINVAL; }
    if (n_consts > 0 && !kinds) { set_err(err, "const_kinds is null"); return RSR_EINVAL; }
    if (n_params > 0 && !params) { set_err(err, "params is null"); return RSR_EINVAL; }
    // flat parameter offsets (get_flat_start_idx, evaluator.rs:232-245)
    std::vector<uint32_t> &flat = tls.flat;
    flat.assign(n_consts + 1, 0);
    for (uint32_t c = 0; c < n_consts; ++c) {
        if (kinds[c] > 6) { set_err(err, "constant " + std::to_string(c) + " has unknown kind"); return RSR_EPROGRAM; }
        flat[c + 1] = flat[c] + kKindWidth[kinds[c]];
    }
    if (flat[n_consts] != n_params) {
        set_err(err, "params holds " + std::to_string(n_params) + " floats, constants need " +
                         std::to_string(flat[n_consts]));
        return RSR_EPROGRAM;
    }
    E.n_params = n_params;
    E.consts.assign(params, params + n_params);

    // ---- replay the stack discipline on value ids
    std::vector<Node> &nodes = tls.nodes;
    nodes.clear();
    // the reference's stacks hold at most kRefStackSlots values each
    int stack[N_STACKS][kRefStackSlots];
    int sp[N_STACKS] = {0, 0, 0, 0, 0};
    std::vector<int> &instr_node = tls.instr_node;  // node id per kept instruction
    instr_node.clear();
    int last[N_STACKS][kRefStackSlots];
    for (auto &row : last) std::fill(row, row + kRefStackSlots, -1);
    for (uint32_t pc = 0; pc < len; ++pc) {
        int op = code[pc] & 0xFF;
        uint32_t a = (code[pc] >> 8) & 0xFFFF;
        if (op >= N_OPCODES) { set_err(err, "pc " + std::to_string(pc) + ": unknown opcode " + std::to_string(op)); return RSR_EPROGRAM; }
        Node n;
        n.opcode = op;
        const OpSig &g = op_sig(op);
        if (is_load(op)) {
            int t = load_stack(op);
            if (t < 0) continue;  // LoadVarB/I, LoadConstB/I push nothing
            n.out = t;
            if (!is_const_load(op)) {
                if (num_features && a + kStackWidth[t] > num_features) {
                    set_err(err, "pc " + std::to_string(pc) + ": feature offset " + std::to_string(a) +
                                     " out of range for " + std::to_string(num_features) + " features");
                    return RSR_EPROGRAM;
                }
                n.arg = a;
            } else {
                if (a >= n_consts) { set_err(err, "pc " + std::to_string(pc) + ": constant index out of range"); return RSR_EPROGRAM; }
                if (kinds[a] != const_kind_for_load(op)) {
                    n.stale = true;
                    int p = sp[t];
                    n.alias = p < kRefStackSlots ? last[t][p] : -1;
                } else {
                    n.arg = flat[a];
                }
            }
        } else {
            int cnt[N_STACKS] = {0, 0, 0, 0, 0};
            for (int i = 0; i < g.n_in; ++i) cnt[g.in[i]]++;
            int base[N_STACKS];
            for (int t = 0; t < N_STACKS; ++t) {
                if (sp[t] < cnt[t]) {
                    set_err(err, "pc " + std::to_string(pc) + ": stack underflow");
                    return RSR_EPROGRAM;
                }
                base[t] = sp[t] - cnt[t];
            }
            n.n_in = g.n_in;
            for (int i = 0; i < g.n_in; ++i) n.in[i] = stack[g.in[i]][base[g.in[i]]++];
            for (int t = 0; t < N_STACKS; ++t) sp[t] -= cnt[t];
            n.out = g.out;
        }
        int t = n.out;
        n.pos = sp[t];
        if (n.pos >= kRefStackSlots) {
            set_err(err, "pc " + std::to_string(pc) + ": more than 32 values on a stack");
            return RSR_EPROGRAM;
        }
        int id = (int)nodes.size();
        nodes.push_back(n);
        instr_node.push_back(id);
        stack[t][sp[t]++] = id;
        if (!n.stale) last[t][n.pos] = id;
        E.depth_ref[t] = std::max(E.depth_ref[t], sp[t]);
    }
    int root = last[SF][0];
    E.result_zero = root < 0;

    // live tree (DAG through stale aliases) behind stack_f[0]
    std::vector<char> &live = tls.live;
    live.assign(nodes.size(), 0);
    if (root >= 0) {
        std::vector<int> &work = tls.work;
        work.assign(1, root);
        while (!work.empty()) {
            int id = work.back();
            work.pop_back();
            if (live[id]) continue;
            live[id] = 1;
            const Node &n = nodes[id];
            for (int i = 0; i < n.n_in; ++i) work.push_back(n.in[i]);
            if (n.stale && n.alias >= 0) work.push_back(n.alias);
        }
    }
    uint32_t flops = 0, rev_flops = 0;
    bool has_stale_live = false;
    for (size_t i = 0; i < nodes.size(); ++i) {
        if (!live[i]) continue;
        flops += op_sig(nodes[i].opcode).flops;
        rev_flops += (uint32_t)reverse_flops(nodes[i].opcode, is_const_load(nodes[i].opcode) && !nodes[i].stale
                                                                   ? kStackWidth[nodes[i].out] : 0);
        if (nodes[i].opcode == INVERSE_M2 || nodes[i].opcode == INVERSE_M3) E.differentiable = false;
        if (nodes[i].stale) has_stale_live = true;
    }
    E.flops_per_point = flops + kMseEpilogueFlops;
    E.adj_flops_per_point = E.flops_per_point + rev_flops + kMseEpilogueRevFlops;
    {
        uint32_t types = 1u << SF;
        for (size_t i = 0; i < nodes.size(); ++i)
            if (live[i]) types |= 1u << nodes[i].out;
        for (int p = 0; p < N_PROFILES; ++p)
            if ((types & ~kProfileTypes[p]) == 0) { E.tape_profile = p; break; }
    }

    // ---- slot form: reference positions
    if (forms & FORM_SLOT) {
    uint32_t sbase[N_STACKS], acc = 0;
    for (int t = 0; t < N_STACKS; ++t) {
        sbase[t] = acc;
        acc += E.depth_ref[t] * kStackWidth[t];
    }
    E.n_slots = acc;
    auto slot_of = [&](int id) -> uint32_t {
        const Node &n = nodes[id];
        return sbase[n.out] + n.pos * kStackWidth[n.out];
    };
    for (int id : instr_node) {
        const Node &n = nodes[id];
        uint32_t w0 = n.stale ? (uint32_t)SLOT_NOP : ((uint32_t)n.opcode | (n.arg << 8));
        uint32_t in[3] = {0, 0, 0};
        for (int i = 0; i < n.n_in; ++i) in[i] = slot_of(n.in[i]);
        E.slot_code.push_back(w0);
        E.slot_code.push_back(slot_of(id) | (in[0] << 16));
        E.slot_code.push_back(in[1] | (in[2] << 16));
        if (n.stale) E.needs_zero_init = true;
    }
    }

    // ---- tape form: value and adjoint slots allocated by lifetime
    if (forms & FORM_TAPE) emit_tape(nodes, live, root, &E);

    // ---- accumulator form
    if ((forms & FORM_ACC) && root >= 0 && !has_stale_live && n_params < (1u << kLdOffsetBits)) {
        AccEmitter em(nodes);
        if (em.analyze(root)) {
            em.gen(root);
            if (fuse) fuse_loads(&em.code);
            bool fits = true;
            for (int t = 0; t < N_STACKS; ++t) {
                E.depth_fast[t] = em.max_sp[t];
                fits = fits && em.max_sp[t] <= kMaxAccStack;
            }
            for (int p = 0; fits && p < N_PROFILES; ++p)
                if ((em.types_ & ~kProfileTypes[p]) == 0) { E.profile = p; break; }
            if (E.profile >= 0) E.reg_code.assign(em.code.begin(), em.code.end());
        }
    }

    // ---- register adjoint form
    if ((forms & FORM_ADJ) && root >= 0 && !has_stale_live && n_params < (1u << kLdOffsetBits)) {
        AccEmitter an(nodes);
        if (an.analyze(root)) {
            AdjEmitter em(nodes, an);
            em.gen(root);
            bool fits = em.tape <= kTapeRefIndex;
            for (int t = 0; t < N_STACKS; ++t) {
                E.adj_depth[t] = em.n_push[t];
                fits = fits && em.n_push[t] <= kMaxAccStack;
            }
            for (int p = 0; fits && p < N_PROFILES; ++p)
                if ((an.types_ & ~kProfileTypes[p]) == 0) { E.adj_profile = p; break; }
            if (E.adj_profile >= 0) {
                em.finish(&E.adj_code);
                E.adj_tape = em.tape;
            }
        }
    }
    return RSR_OK;
}

}  // namespace rsr
