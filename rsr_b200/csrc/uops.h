// uops.h -- device instruction formats shared by the host encoder and the
// kernels.
//
// Two encodings of a reference program (src/engine/expr/program.rs:18-23):
//
//  * Slot form, for the slot-file kernel.  Every reference instruction keeps
//    the stack positions the reference VM gives it (state.rs:12-37), mapped to
//    a flat file of scalar slots, so the kernel reproduces eval_simd exactly,
//    including stack_f[0] as the result (evaluator.rs:147-149) and constant
//    loads of a mismatched variant that leave a slot unwritten
//    (evaluator.rs:37-40).  Three words per instruction:
//       w0 = opcode | aux << 8        (aux: feature offset or flat param offset)
//       w1 = out_slot | in0_slot << 16
//       w2 = in1_slot | in2_slot << 16
//
//  * Register form, for the register-stack kernel.  The expression tree that
//    produces the result is re-emitted with its subtrees evaluated in the order
//    that needs the fewest stack slots (values are pure, so every value is
//    bit-identical to the reference's); leaf loads are fused into their
//    consumer; cross-stack operands move through transfer registers T[0..8].
//    One word per micro-op:
//       bits 0-2 stack position, bits 3-10 micro-op kind, bits 11-31 argument.
#pragma once
#include <stdint.h>

namespace rsr {

// Reference opcodes (compose_engine! order, domain.rs:46-63 + basic + linalg).
enum Opcode : uint8_t {
    LOAD_VAR_F = 0, LOAD_CONST_F, LOAD_VAR_B, LOAD_CONST_B, LOAD_VAR_I, LOAD_CONST_I,
    LOAD_VAR_V2, LOAD_CONST_V2, LOAD_VAR_V3, LOAD_CONST_V3, LOAD_VAR_M2, LOAD_CONST_M2,
    LOAD_VAR_M3, LOAD_CONST_M3,
    ADD_F = 14, SUB_F, MUL_F, DIV_F, SIN_F, COS_F, EXP_F, SQR_F, SQRT_F, LN_F,
    MAKE_VEC2 = 24, MAKE_VEC3, GET_X_V2, GET_Y_V2, GET_X_V3, GET_Y_V3, GET_Z_V3,
    ADD_V2, SUB_V2, SCALE_V2, DOT_V2, NORM_V2,
    ADD_V3, SUB_V3, SCALE_V3, DOT_V3, NORM_V3, CROSS_V3,
    MAKE_MAT2, ADD_M2, SUB_M2, SCALE_M2, MUL_M2, MUL_M2V2, DET_M2, TRACE_M2, TRANSPOSE_M2, INVERSE_M2,
    MAKE_MAT3, ADD_M3, SUB_M3, SCALE_M3, MUL_M3, MUL_M3V3, DET_M3, TRACE_M3, TRANSPOSE_M3, INVERSE_M3,
    N_OPCODES,
    // slot form only: a LoadConst* of a mismatched variant (no write)
    SLOT_NOP = 200
};

// Typed stacks (VmState fields, state.rs:14-36).
enum Stack : int { SF = 0, SV2 = 1, SV3 = 2, SM2 = 3, SM3 = 4, N_STACKS = 5 };
static constexpr int kStackWidth[N_STACKS] = {1, 2, 3, 4, 9};
static constexpr int kRefStackSlots = 32;

// ----------------------------------------------------- register micro-ops
// Argument source suffixes: S = stack position s+1, X = feature, C = constant.
enum UopKind : uint8_t {
    // F stack
    U_F_LDX = 0, U_F_LDC, U_F_FROM_T0, U_F_TO_T0, U_F_TO_T1, U_F_TO_T2,
    U_F_ADD, U_F_SUB, U_F_RSUB, U_F_MUL, U_F_DIV, U_F_RDIV,
    U_F_ADDX, U_F_SUBX, U_F_RSUBX, U_F_MULX, U_F_DIVX, U_F_RDIVX,
    U_F_ADDC, U_F_SUBC, U_F_RSUBC, U_F_MULC, U_F_DIVC, U_F_RDIVC,
    U_F_SIN, U_F_COS, U_F_EXP, U_F_SQR, U_F_SQRT, U_F_LN,
    // V2 stack
    U_V2_LDX = 32, U_V2_LDC, U_V2_FROM_T, U_V2_TO_T0, U_V2_TO_T2,
    U_V2_ADD, U_V2_SUB, U_V2_RSUB, U_V2_ADDX, U_V2_SUBX, U_V2_RSUBX, U_V2_ADDC, U_V2_SUBC, U_V2_RSUBC,
    U_V2_SCALE_T, U_V2_SCALE_X, U_V2_SCALE_C,
    U_V2_DOT_T, U_V2_DOTX_T, U_V2_DOTC_T, U_V2_NORM_T, U_V2_GETX_T, U_V2_GETY_T,
    U_V2_MULM_T, U_V2_MULMX, U_V2_MULMC,
    // V3 stack
    U_V3_LDX = 64, U_V3_LDC, U_V3_FROM_T, U_V3_TO_T0, U_V3_TO_T3, U_V3_TO_T6,
    U_V3_ADD, U_V3_SUB, U_V3_RSUB, U_V3_CROSS, U_V3_RCROSS,
    U_V3_ADDX, U_V3_SUBX, U_V3_RSUBX, U_V3_CROSSX, U_V3_RCROSSX,
    U_V3_ADDC, U_V3_SUBC, U_V3_RSUBC, U_V3_CROSSC, U_V3_RCROSSC,
    U_V3_SCALE_T, U_V3_SCALE_X, U_V3_SCALE_C,
    U_V3_DOT_T, U_V3_DOTX_T, U_V3_DOTC_T, U_V3_NORM_T, U_V3_GETX_T, U_V3_GETY_T, U_V3_GETZ_T,
    U_V3_MULM_T, U_V3_MULMX, U_V3_MULMC,
    // M2 stack
    U_M2_LDX = 104, U_M2_LDC, U_M2_FROM_T, U_M2_TO_T,
    U_M2_ADD, U_M2_SUB, U_M2_RSUB, U_M2_MUL, U_M2_RMUL,
    U_M2_ADDX, U_M2_SUBX, U_M2_RSUBX, U_M2_MULX, U_M2_RMULX,
    U_M2_ADDC, U_M2_SUBC, U_M2_RSUBC, U_M2_MULC, U_M2_RMULC,
    U_M2_SCALE_T, U_M2_SCALE_X, U_M2_SCALE_C,
    U_M2_DET_T, U_M2_TRACE_T, U_M2_TRANSPOSE, U_M2_INVERSE,
    // M3 stack
    U_M3_LDX = 136, U_M3_LDC, U_M3_FROM_T, U_M3_TO_T,
    U_M3_ADD, U_M3_SUB, U_M3_RSUB, U_M3_MUL, U_M3_RMUL,
    U_M3_ADDX, U_M3_SUBX, U_M3_RSUBX, U_M3_MULX, U_M3_RMULX,
    U_M3_ADDC, U_M3_SUBC, U_M3_RSUBC, U_M3_MULC, U_M3_RMULC,
    U_M3_SCALE_T, U_M3_SCALE_X, U_M3_SCALE_C,
    U_M3_DET_T, U_M3_TRACE_T, U_M3_TRANSPOSE, U_M3_INVERSE,
    U_END = 168
};

static inline constexpr uint32_t uop_word(uint32_t kind, uint32_t slot, uint32_t arg) {
    return (slot & 0x7u) | ((kind & 0xFFu) << 3) | (arg << 11);
}
static constexpr int kMaxRegSlots = 8;

// Register-stack kernel profiles: which stacks are held in registers and how
// many positions each has.  A program runs on the first profile it fits.
struct ProfileCaps {
    int cap[N_STACKS];
    int n_transfer;   // transfer registers T[0..n)
};
enum Profile : int { P_F = 0, P_FV3 = 1, P_FV2M2 = 2, P_FV3M3 = 3, P_ALL = 4, N_PROFILES = 5 };
static constexpr ProfileCaps kProfiles[N_PROFILES] = {
    {{8, 0, 0, 0, 0}, 1},
    {{8, 0, 4, 0, 0}, 3},
    {{6, 3, 0, 3, 0}, 4},
    {{6, 0, 3, 0, 2}, 9},
    {{6, 2, 3, 2, 2}, 9},
};

// Program descriptor for the kernels (one per program in a launch).
struct ProgDesc {
    uint32_t uop_off;     // first word in the launch's code pool
    uint32_t uop_len;     // words (slot form: 3 per instruction)
    uint32_t const_off;   // first float in the launch's constant pool
    uint32_t n_consts;    // floats
    uint32_t n_slots;     // slot form: scalar slots needed
    uint32_t flags;       // PF_* below
    uint32_t dataset;     // index into the launch's dataset table
    uint32_t part_off;    // first partial-sum slot of this program
    uint32_t n_parts;     // partial-sum slots (chunks) of this program
    uint32_t n_tape;      // adjoint kernel: scalar tape slots
};
enum : uint32_t { PF_RESULT_ZERO = 1u, PF_NEEDS_ZERO_INIT = 2u, PF_DIFFERENTIABLE = 4u };

// Dataset descriptor (structure-of-arrays copy of a Dataset).
struct DatasetDesc {
    const float *x;       // x[f * stride + i]
    const float *y;       // y[i]
    uint64_t stride;      // multiple of 128 points
    uint64_t n_eval;      // num_batches * 8: points evaluated and counted
    uint64_t num_samples; // divisor
    uint32_t num_features;
    uint32_t pad;
};

// Work item: a chunk of point tiles for a group of programs that share a
// dataset.  Tiles are 32 * points_per_thread points.
struct WorkItem {
    uint32_t prog_begin;  // index into the launch's program list
    uint32_t n_progs;     // programs evaluated on each tile (programs per warp)
    uint32_t tile_begin;
    uint32_t tile_end;
    uint32_t chunk;       // partial-sum slot offset within each program
    uint32_t pad;
};

}  // namespace rsr
