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

// ------------------------------------------------------- register form
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

struct Plan {
    int fused = -1;        // operand index taken from a feature/constant directly
    int order[3] = {0, 1, 2};
    int n_kids = 0;        // stack operands in evaluation order (operand indices)
    std::array<int, N_STACKS> need{};
};

class RegEmitter {
   public:
    RegEmitter(const std::vector<Node> &nodes) : nodes_(nodes), plans_(nodes.size()) {}

    bool plan(int id) {  // fills plans_ bottom-up; false if unsupported
        const Node &n = nodes_[id];
        Plan &p = plans_[id];
        if (is_load(n.opcode)) {
            if (n.stale) return false;
            p.need.fill(0);
            p.need[n.out] = 1;
            return true;
        }
        for (int i = 0; i < n.n_in; ++i)
            if (!plan(n.in[i])) return false;
        OpClass c = op_class(n.opcode);
        // choose a fused (leaf) operand
        if (c == C_BIN || c == C_DOT) {
            if (leaf(nodes_[n.in[1]])) p.fused = 1;
            else if (leaf(nodes_[n.in[0]])) p.fused = 0;
        } else if (c == C_SCALE || c == C_MULMV) {
            if (leaf(nodes_[n.in[0]])) p.fused = 0;
        }
        int kids[3], nk = 0;
        for (int i = 0; i < n.n_in; ++i)
            if (i != p.fused) kids[nk++] = i;
        p.n_kids = nk;
        // best evaluation order of the stack operands
        int perm[3] = {0, 1, 2};
        int best_cost = 1 << 30;
        std::array<int, N_STACKS> best_need{};
        int best_order[3] = {0, 1, 2};
        do {
            std::array<int, N_STACKS> cur{}, peak{};
            for (int j = 0; j < nk; ++j) {
                int k = n.in[kids[perm[j]]];
                const auto &kn = plans_[k].need;
                for (int t = 0; t < N_STACKS; ++t) peak[t] = std::max(peak[t], cur[t] + kn[t]);
                cur[nodes_[k].out] += 1;
            }
            if (n.out >= 0) {
                int consumed = 0;
                for (int j = 0; j < nk; ++j) consumed += nodes_[n.in[kids[j]]].out == n.out;
                peak[n.out] = std::max(peak[n.out], cur[n.out] - consumed + 1);
            }
            int cost = 0;
            for (int t = 0; t < N_STACKS; ++t) cost += peak[t] * kStackWidth[t];
            if (cost < best_cost) {
                best_cost = cost;
                best_need = peak;
                for (int j = 0; j < nk; ++j) best_order[j] = kids[perm[j]];
            }
        } while (std::next_permutation(perm, perm + nk));
        p.need = best_need;
        for (int j = 0; j < nk; ++j) p.order[j] = best_order[j];
        return true;
    }

    // Emits the subtree of `id`; leaves its value on top of its stack.
    void gen(int id) {
        const Node &n = nodes_[id];
        const Plan &p = plans_[id];
        if (is_load(n.opcode)) {
            int t = n.out;
            static const int ldx[N_STACKS] = {U_F_LDX, U_V2_LDX, U_V3_LDX, U_M2_LDX, U_M3_LDX};
            static const int ldc[N_STACKS] = {U_F_LDC, U_V2_LDC, U_V3_LDC, U_M2_LDC, U_M3_LDC};
            emit(is_const_load(n.opcode) ? ldc[t] : ldx[t], push(t), n.arg);
            return;
        }
        int pos[3] = {-1, -1, -1};
        for (int j = 0; j < p.n_kids; ++j) {
            int i = p.order[j];
            gen(n.in[i]);
            pos[i] = sp_[nodes_[n.in[i]].out] - 1;
        }
        // pop the stack operands
        for (int i = 0; i < n.n_in; ++i)
            if (i != p.fused) sp_[nodes_[n.in[i]].out] -= 1;
        const Node *fz = p.fused >= 0 ? &nodes_[n.in[p.fused]] : nullptr;
        bool fzc = fz && is_const_load(fz->opcode);
        uint32_t farg = fz ? fz->arg : 0;
        int op = n.opcode;
        switch (op_class(op)) {
            case C_BIN: {
                int t = n.out;
                int r = sp_[t];
                int kind = bin_kind(op, p.fused, fzc, pos, r);
                emit(kind, r, farg);
                push(t);
                break;
            }
            case C_DOT: {
                int t = nodes_[n.in[0]].out;
                int base = t == SV2 ? U_V2_DOT_T : U_V3_DOT_T;
                if (p.fused < 0) emit(base, std::min(pos[0], pos[1]), 0);
                else emit(base + (fzc ? 2 : 1), pos[1 - p.fused], farg);
                use_t(1);
                emit(U_F_FROM_T0, push(SF), 0);
                break;
            }
            case C_SCALE: {
                int t = n.out;
                static const int sc[N_STACKS] = {0, U_V2_SCALE_T, U_V3_SCALE_T, U_M2_SCALE_T, U_M3_SCALE_T};
                if (p.fused == 0) {
                    emit(sc[t] + (fzc ? 2 : 1), pos[1], farg);
                } else {
                    emit(U_F_TO_T0, pos[0], 0);
                    use_t(1);
                    emit(sc[t], pos[1], 0);
                }
                push(t);
                break;
            }
            case C_MULMV: {
                int tv = n.out;
                int base = tv == SV2 ? U_V2_MULM_T : U_V3_MULM_T;
                if (p.fused == 0) {
                    emit(base + (fzc ? 2 : 1), pos[1], farg);
                } else {
                    emit(tv == SV2 ? U_M2_TO_T : U_M3_TO_T, pos[0], 0);
                    use_t(tv == SV2 ? 4 : 9);
                    emit(base, pos[1], 0);
                }
                push(tv);
                break;
            }
            case C_UNARY_F: {
                static const int k[] = {U_F_SIN, U_F_COS, U_F_EXP, U_F_SQR, U_F_SQRT, U_F_LN};
                emit(k[op - SIN_F], pos[0], 0);
                push(SF);
                break;
            }
            case C_GET: {
                int kind = op == GET_X_V2 ? U_V2_GETX_T : op == GET_Y_V2 ? U_V2_GETY_T
                         : op == GET_X_V3 ? U_V3_GETX_T : op == GET_Y_V3 ? U_V3_GETY_T : U_V3_GETZ_T;
                emit(kind, pos[0], 0);
                use_t(1);
                emit(U_F_FROM_T0, push(SF), 0);
                break;
            }
            case C_NORM:
                emit(op == NORM_V2 ? U_V2_NORM_T : U_V3_NORM_T, pos[0], 0);
                use_t(1);
                emit(U_F_FROM_T0, push(SF), 0);
                break;
            case C_DET: case C_TRACE: {
                int kind = op == DET_M2 ? U_M2_DET_T : op == DET_M3 ? U_M3_DET_T
                         : op == TRACE_M2 ? U_M2_TRACE_T : U_M3_TRACE_T;
                emit(kind, pos[0], 0);
                use_t(1);
                emit(U_F_FROM_T0, push(SF), 0);
                break;
            }
            case C_MAT_UN: {
                int kind = op == TRANSPOSE_M2 ? U_M2_TRANSPOSE : op == TRANSPOSE_M3 ? U_M3_TRANSPOSE
                         : op == INVERSE_M2 ? U_M2_INVERSE : U_M3_INVERSE;
                emit(kind, pos[0], 0);
                push(n.out);
                break;
            }
            case C_MAKE: {
                if (op == MAKE_VEC2 || op == MAKE_VEC3) {
                    static const int tt[3] = {U_F_TO_T0, U_F_TO_T1, U_F_TO_T2};
                    for (int i = 0; i < n.n_in; ++i) emit(tt[i], pos[i], 0);
                    use_t(n.n_in);
                    emit(op == MAKE_VEC2 ? U_V2_FROM_T : U_V3_FROM_T, push(n.out), 0);
                } else if (op == MAKE_MAT2) {
                    emit(U_V2_TO_T0, pos[0], 0);
                    emit(U_V2_TO_T2, pos[1], 0);
                    use_t(4);
                    emit(U_M2_FROM_T, push(SM2), 0);
                } else {
                    emit(U_V3_TO_T0, pos[0], 0);
                    emit(U_V3_TO_T3, pos[1], 0);
                    emit(U_V3_TO_T6, pos[2], 0);
                    use_t(9);
                    emit(U_M3_FROM_T, push(SM3), 0);
                }
                break;
            }
            case C_LOAD: break;
        }
    }

    const Plan &plan_of(int id) const { return plans_[id]; }
    std::vector<uint32_t> code;
    int max_sp[N_STACKS] = {0, 0, 0, 0, 0};
    int max_t = 0;

   private:
    int push(int t) {
        int p = sp_[t]++;
        max_sp[t] = std::max(max_sp[t], sp_[t]);
        return p;
    }
    void use_t(int n) { max_t = std::max(max_t, n); }
    void emit(int kind, int slot, uint32_t arg) { code.push_back(uop_word(kind, slot, arg)); }

    static int bin_kind(int op, int fused, bool fzc, const int *pos, int r) {
        // base kinds: {stack-stack, reversed, X, reversed X, C, reversed C}
        struct K { int s, rs, x, rx, c, rc; };
        K k{};
        switch (op) {
            case ADD_F: k = {U_F_ADD, U_F_ADD, U_F_ADDX, U_F_ADDX, U_F_ADDC, U_F_ADDC}; break;
            case MUL_F: k = {U_F_MUL, U_F_MUL, U_F_MULX, U_F_MULX, U_F_MULC, U_F_MULC}; break;
            case SUB_F: k = {U_F_SUB, U_F_RSUB, U_F_SUBX, U_F_RSUBX, U_F_SUBC, U_F_RSUBC}; break;
            case DIV_F: k = {U_F_DIV, U_F_RDIV, U_F_DIVX, U_F_RDIVX, U_F_DIVC, U_F_RDIVC}; break;
            case ADD_V2: k = {U_V2_ADD, U_V2_ADD, U_V2_ADDX, U_V2_ADDX, U_V2_ADDC, U_V2_ADDC}; break;
            case SUB_V2: k = {U_V2_SUB, U_V2_RSUB, U_V2_SUBX, U_V2_RSUBX, U_V2_SUBC, U_V2_RSUBC}; break;
            case ADD_V3: k = {U_V3_ADD, U_V3_ADD, U_V3_ADDX, U_V3_ADDX, U_V3_ADDC, U_V3_ADDC}; break;
            case SUB_V3: k = {U_V3_SUB, U_V3_RSUB, U_V3_SUBX, U_V3_RSUBX, U_V3_SUBC, U_V3_RSUBC}; break;
            case CROSS_V3: k = {U_V3_CROSS, U_V3_RCROSS, U_V3_CROSSX, U_V3_RCROSSX, U_V3_CROSSC, U_V3_RCROSSC}; break;
            case ADD_M2: k = {U_M2_ADD, U_M2_ADD, U_M2_ADDX, U_M2_ADDX, U_M2_ADDC, U_M2_ADDC}; break;
            case SUB_M2: k = {U_M2_SUB, U_M2_RSUB, U_M2_SUBX, U_M2_RSUBX, U_M2_SUBC, U_M2_RSUBC}; break;
            case MUL_M2: k = {U_M2_MUL, U_M2_RMUL, U_M2_MULX, U_M2_RMULX, U_M2_MULC, U_M2_RMULC}; break;
            case ADD_M3: k = {U_M3_ADD, U_M3_ADD, U_M3_ADDX, U_M3_ADDX, U_M3_ADDC, U_M3_ADDC}; break;
            case SUB_M3: k = {U_M3_SUB, U_M3_RSUB, U_M3_SUBX, U_M3_RSUBX, U_M3_SUBC, U_M3_RSUBC}; break;
            case MUL_M3: k = {U_M3_MUL, U_M3_RMUL, U_M3_MULX, U_M3_RMULX, U_M3_MULC, U_M3_RMULC}; break;
        }
        if (fused == 1) return fzc ? k.c : k.x;   // stack[r] = stack[r] op leaf
        if (fused == 0) return fzc ? k.rc : k.rx; // stack[r] = leaf op stack[r]
        return pos[0] == r ? k.s : k.rs;          // operands at r, r+1
    }

    const std::vector<Node> &nodes_;
    std::vector<Plan> plans_;
    int sp_[N_STACKS] = {0, 0, 0, 0, 0};
};

void set_err(std::string *err, const std::string &m) {
    if (err) *err = m;
}

}  // namespace

int encode_program(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t n_consts,
                   const float *params, uint32_t n_params, uint32_t num_features, EncodedProgram *out,
                   std::string *err) {
    EncodedProgram &E = *out;
    E = EncodedProgram();
    if (len > 0 && !code) { set_err(err, "code is null"); return RSR_EINVAL; }
    if (n_consts > 0 && !kinds) { set_err(err, "const_kinds is null"); return RSR_EINVAL; }
    if (n_params > 0 && !params) { set_err(err, "params is null"); return RSR_EINVAL; }
    // flat parameter offsets (get_flat_start_idx, evaluator.rs:232-245)
    std::vector<uint32_t> flat(n_consts + 1, 0);
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
    std::vector<Node> nodes;
    nodes.reserve(len);
    std::vector<int> stack[N_STACKS];
    std::vector<int> instr_node;  // node id per kept instruction
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
                    int p = (int)stack[t].size();
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
                if ((int)stack[t].size() < cnt[t]) {
                    set_err(err, "pc " + std::to_string(pc) + ": stack underflow");
                    return RSR_EPROGRAM;
                }
                base[t] = (int)stack[t].size() - cnt[t];
            }
            n.n_in = g.n_in;
            for (int i = 0; i < g.n_in; ++i) n.in[i] = stack[g.in[i]][base[g.in[i]]++];
            for (int t = 0; t < N_STACKS; ++t) stack[t].resize(stack[t].size() - cnt[t]);
            n.out = g.out;
        }
        int t = n.out;
        n.pos = (int)stack[t].size();
        if (n.pos >= kRefStackSlots) {
            set_err(err, "pc " + std::to_string(pc) + ": more than 32 values on a stack");
            return RSR_EPROGRAM;
        }
        int id = (int)nodes.size();
        nodes.push_back(n);
        instr_node.push_back(id);
        stack[t].push_back(id);
        if (!n.stale) last[t][n.pos] = id;
        E.depth_ref[t] = std::max(E.depth_ref[t], (int)stack[t].size());
    }
    int root = last[SF][0];
    E.result_zero = root < 0;

    // live tree (DAG through stale aliases) behind stack_f[0]
    std::vector<char> live(nodes.size(), 0);
    if (root >= 0) {
        std::vector<int> work{root};
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
    uint32_t flops = 0;
    bool has_stale_live = false;
    for (size_t i = 0; i < nodes.size(); ++i) {
        if (!live[i]) continue;
        flops += op_sig(nodes[i].opcode).flops;
        if (nodes[i].opcode == INVERSE_M2 || nodes[i].opcode == INVERSE_M3) E.differentiable = false;
        if (nodes[i].stale) has_stale_live = true;
    }
    E.flops_per_point = flops + kMseEpilogueFlops;

    // ---- slot form: reference positions
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

    // ---- tape form: every live value gets its own slots (SSA)
    {
        std::vector<uint32_t> tslot(nodes.size(), 0);
        uint32_t tacc = 0;
        for (size_t i = 0; i < nodes.size(); ++i) {
            if (!live[i]) continue;
            tslot[i] = tacc;
            tacc += kStackWidth[nodes[i].out];
        }
        E.n_tape_slots = tacc;
        E.tape_code.push_back(root >= 0 ? tslot[root] : 0xFFFFFFFFu);  // header: result slot
        for (size_t i = 0; i < nodes.size(); ++i) {
            if (!live[i]) continue;
            const Node &n = nodes[i];
            uint32_t w0, in[3] = {0, 0, 0};
            if (n.stale) {
                // copy of the value left in that slot, or zero; aux = has_alias | width << 1
                w0 = (uint32_t)SLOT_NOP | (((n.alias >= 0 ? 1u : 0u) | ((uint32_t)kStackWidth[n.out] << 1)) << 8);
                if (n.alias >= 0) in[0] = tslot[n.alias];
            } else {
                w0 = (uint32_t)n.opcode | (n.arg << 8);
                for (int k = 0; k < n.n_in; ++k) in[k] = tslot[n.in[k]];
            }
            E.tape_code.push_back(w0);
            E.tape_code.push_back(tslot[i] | (in[0] << 16));
            E.tape_code.push_back(in[1] | (in[2] << 16));
        }
    }

    // ---- register form
    if (root >= 0 && !has_stale_live) {
        RegEmitter em(nodes);
        if (em.plan(root)) {
            em.gen(root);
            const auto &need = em.plan_of(root).need;
            for (int t = 0; t < N_STACKS; ++t) E.depth_fast[t] = std::max(need[t], em.max_sp[t]);
            for (int p = 0; p < N_PROFILES; ++p) {
                bool ok = em.max_t <= kProfiles[p].n_transfer;
                for (int t = 0; t < N_STACKS; ++t) ok = ok && E.depth_fast[t] <= kProfiles[p].cap[t];
                if (ok) { E.profile = p; break; }
            }
            if (E.profile >= 0) E.reg_code = std::move(em.code);
        }
    }
    return RSR_OK;
}

}  // namespace rsr
