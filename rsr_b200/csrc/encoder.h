// encoder.h -- host-side analysis of reference programs and emission of the
// two device encodings described in uops.h.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "uops.h"

namespace rsr {

// Static properties of each reference opcode: operand stacks in
// expected_types order (basic/mod.rs:209-217, linalg/mod.rs:375-432) and the
// result stack (-1: none).
struct OpSig {
    int n_in;
    int in[3];
    int out;
    int flops;  // unfused FP32 lane-ops
};
const OpSig &op_sig(int opcode);
int load_stack(int opcode);       // stack a LoadVar*/LoadConst* pushes to, -1 for B/I loads
bool is_load(int opcode);
bool is_const_load(int opcode);
int kind_width(int kind);         // flat params per Scalar variant (program.rs:84-98)
int const_kind_for_load(int opcode);

struct EncodedProgram {
    // common
    uint32_t n_params = 0;
    std::vector<float> consts;            // flat parameters (kernel constant pool)
    uint32_t flops_per_point = 0;         // incl. MSE epilogue
    uint32_t adj_flops_per_point = 0;     // forward + reverse sweep (adjoint kernel), incl. epilogues
    bool differentiable = true;
    bool result_zero = false;             // stack_f[0] is never written
    int depth_ref[N_STACKS] = {0, 0, 0, 0, 0};
    // slot form
    std::vector<uint32_t> slot_code;      // 3 words per instruction
    uint32_t n_slots = 0;
    bool needs_zero_init = false;
    // register form
    int profile = -1;                     // -1: register kernel not applicable
    int depth_fast[N_STACKS] = {0, 0, 0, 0, 0};
    std::vector<uint32_t> reg_code;
    // adjoint (slot form with one slot range per value, never reused)
    std::vector<uint32_t> tape_code;      // 2 header words + 5 words per live node
    uint32_t n_tape_val = 0, n_tape_adj = 0;  // scalar value / adjoint slots
    int tape_profile = P_ALL;             // smallest kernel profile covering the live values' types
    // register adjoint (uops.h, kAdjHeaderWords): empty when the program
    // needs the slot-file adjoint
    std::vector<uint32_t> adj_code;
    uint32_t adj_tape = 0;                // tape slots (scalar values)
    int adj_depth[N_STACKS] = {0, 0, 0, 0, 0};  // stack slots per type (one per PUSH)
    int adj_profile = -1;

    // Back to the default state; the vectors keep their capacity, so an
    // EncodedProgram reused across calls stops allocating.
    void reset() {
        std::vector<float> c = std::move(consts);
        std::vector<uint32_t> sc = std::move(slot_code), rc = std::move(reg_code), tc = std::move(tape_code),
                              ac = std::move(adj_code);
        *this = EncodedProgram();
        c.clear(); sc.clear(); rc.clear(); tc.clear(); ac.clear();
        consts = std::move(c); slot_code = std::move(sc); reg_code = std::move(rc); tape_code = std::move(tc);
        adj_code = std::move(ac);
    }
};

// Validates and encodes.  num_features == 0 skips feature-range checks.
// Returns 0 or an rsr_status code, with a message in *err.
// Device forms to emit (validation and the analysis run for every call).
enum EncodeForms : unsigned { FORM_SLOT = 1u, FORM_TAPE = 2u, FORM_ACC = 4u, FORM_ADJ = 8u, FORM_ALL = 15u };
int encode_program(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t n_consts,
                   const float *params, uint32_t n_params, uint32_t num_features, EncodedProgram *out,
                   std::string *err, bool fuse_loads = true, unsigned forms = FORM_ALL);

}  // namespace rsr
