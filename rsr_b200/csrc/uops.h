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
//  * Accumulator form, for the register (batched) kernel.  Each value type
//    has one accumulator register set (A_F, A_V2, A_V3, A_M2, A_M3), P data
//    points wide; every micro-op reads and writes accumulators, and a value
//    that must wait while a sibling subtree is evaluated is pushed to a
//    per-type stack in shared memory at a slot fixed by the encoder.  Leaf
//    operands (features, constants) are fused into the consuming op.  Sibling
//    subtrees are evaluated largest first; values are pure, so every result is
//    bit-identical to the reference's.  One word per micro-op:
//       bits 0-7 micro-op kind, bits 8-31 argument (feature offset, flat
//       param offset or stack slot).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define RSR_HD __host__ __device__
#else
#define RSR_HD
#endif

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

// --------------------------------------------------- accumulator micro-ops
// Sources of the second operand: X feature, C constant, S shared-memory stack
// slot, A the accumulator of the operand's own type.
enum AccSrc : int { SRC_X = 0, SRC_C = 1, SRC_S = 2 };
// Binary operations on one type: a = a op b, R-forms b op a.
enum AccBin : int { BIN_ADD = 0, BIN_SUB, BIN_RSUB, BIN_MUL, BIN_DIV, BIN_RDIV, BIN_CROSS, BIN_RCROSS,
                    BIN_MMUL, BIN_RMMUL };

// Kind numbering: one block per accumulator type.
//   F  (base 0):   LDX LDC PUSH, {ADD SUB RSUB MUL DIV RDIV} x {X C S}, SIN COS EXP SQR SQRT LN
//   V2 (base 32):  LDX LDC PUSH, {ADD SUB RSUB} x {X C S}, SCALE{A X C S}, DOT{X C S}, NORM GETX GETY,
//                  MULM{A X C S}, MAKE
//   V3 (base 64):  LDX LDC PUSH, {ADD SUB RSUB CROSS RCROSS} x {X C S}, SCALE{A X C S}, DOT{X C S},
//                  NORM GETX GETY GETZ, MULM{A X C S}, MAKE
//   M2 (base 104), M3 (base 136): LDX LDC PUSH, {ADD SUB RSUB MUL RMUL} x {X C S}, SCALE{A X C S},
//                  DET TRACE TRANSPOSE INVERSE, MAKE
enum AccKind : int {
    K_F = 0, K_F_LDX = 0, K_F_LDC = 1, K_F_PUSH = 2, K_F_BIN = 3, K_F_UN = 21, K_F_END = 27,
    K_V2 = 32, K_V3 = 64, K_M2 = 104, K_M3 = 136, K_END = 163,
    // offsets within the V2 / V3 blocks
    KV_LDX = 0, KV_LDC = 1, KV_PUSH = 2, KV_BIN = 3,
    // offsets within the M blocks
    KM_LDX = 0, KM_LDC = 1, KM_PUSH = 2, KM_BIN = 3, KM_SCALE = 18, KM_DET = 22, KM_TRACE = 23,
    KM_TRANSPOSE = 24, KM_INVERSE = 25, KM_MAKE = 26,
};
// number of binary ops in each block
static constexpr int kBinOps[5] = {6, 3, 5, 5, 5};
// Register adjoint (kernels_adj.cu): one TAPE kind per block, just past the
// block's last kind; arg = first tape slot.  It stores the type's
// accumulator to the tape, for the reverse rules that read forward values.
static constexpr int kTapeKind[5] = {K_F + 27, K_V2 + 27, K_V3 + 34, K_M2 + 27, K_M3 + 27};
static constexpr int kBlockBase[5] = {K_F, K_V2, K_V3, K_M2, K_M3};
// V-block offsets after the binary ops
RSR_HD static constexpr int kv_scale(int nbin) { return KV_BIN + 3 * nbin; }       // 4 kinds: A X C S
RSR_HD static constexpr int kv_dot(int nbin) { return kv_scale(nbin) + 4; }        // 3 kinds: X C S
RSR_HD static constexpr int kv_norm(int nbin) { return kv_dot(nbin) + 3; }         // NORM, GETX, GETY[, GETZ]
RSR_HD static constexpr int kv_mulm(int nbin, int w) { return kv_norm(nbin) + 1 + w; }  // 4 kinds: A X C S
RSR_HD static constexpr int kv_make(int nbin, int w) { return kv_mulm(nbin, w) + 4; }

RSR_HD static inline constexpr uint32_t uop_word(uint32_t kind, uint32_t arg) { return (kind & 0xFFu) | (arg << 8); }

// Fused loads.  A unary op (F unary, NORM/GET, DET/TRACE/TRANSPOSE/INVERSE)
// may first load its operand, and a PUSH may be followed by a load:
//   unary arg:  bits 0-11 feature or param offset, bits 12-13 load first
//               (0 none, 1 feature, 2 constant)
//   PUSH arg:   bits 0-3 slot, bits 4-6 then load into accumulator type
//               (0 none, 1 + type), bit 7 constant (else feature),
//               bits 8-19 offset
static constexpr uint32_t kLdOffsetBits = 12;
RSR_HD static inline constexpr uint32_t unary_load_arg(uint32_t off, uint32_t src1) { return off | (src1 << 12); }
RSR_HD static inline constexpr uint32_t push_load_arg(uint32_t slot, uint32_t type1, uint32_t is_const, uint32_t off) {
    return slot | (type1 << 4) | (is_const << 7) | (off << 8);
}

// Tape value slot that stands for a feature column (adjoint kernel): the
// low 15 bits are the feature offset.
constexpr uint32_t kTapeFeature = 0x8000u;
// Tape adjoint slot fields (16 bits).  Value and adjoint slots share one slot
// file, so on an input field kTapeZeroFirst asks the reverse step to clear
// that input's adjoint slots before adding to them: the step holds the first
// contribution to that adjoint, and its slots may still hold an earlier value.
constexpr uint32_t kTapeZeroFirst = 0x8000u;

// Register-kernel profiles: the accumulator types a kernel instance holds.

enum Profile : int { P_F = 0, P_FV3 = 1, P_FV2M2 = 2, P_FV3M3 = 3, P_ALL = 4, N_PROFILES = 5 };
static constexpr uint32_t kProfileTypes[N_PROFILES] = {
    1u << SF, (1u << SF) | (1u << SV3), (1u << SF) | (1u << SV2) | (1u << SM2), (1u << SF) | (1u << SV3) | (1u << SM3),
    0x1Fu};
static constexpr int kMaxAccStack = 16;   // shared-memory stack slots per type

// Register adjoint code of a program (EncodedProgram::adj_code): word 0 the
// number F of forward entries, word 1 the number R of reverse entries, then
// F forward entries of two words each -- the micro-op word (accumulator
// form, a load after a PUSH fused into the PUSH's word but no load fused
// into a unary op, every PUSH to its own stack slot so that spilled values
// survive the forward sweep; TAPE kinds for the tape stores an op's entry
// cannot carry) and its tape stores (kNoTape) -- then R reverse entries of
// two words each, in the order the reverse sweep runs them: the forward word
// of the micro-op being reversed, and its tape references (first | second
// << 16; which forward values they hold depends on the kind,
// kernels_adj.cu).  A reference is a tape slot (below kTapeRefC), or, where
// the forward value was a plain feature or constant load not changed since,
// that feature (kTapeRefX | index) or constant (kTapeRefC | index), which
// the reverse sweep reads again instead of a tape slot; a value of width W
// reads W consecutive slots, features or constants.
static constexpr int kAdjHeaderWords = 2;
static constexpr uint32_t kTapeRefX = 0x8000u, kTapeRefC = 0x4000u, kTapeRefIndex = 0x3FFFu;
// Second word of a forward entry: the tape slot its op stores the op type's
// accumulator to before running (low half) and after (high half), kNoTape
// for none.
static constexpr uint32_t kNoTape = 0xFFFFu, kNoTapes = 0xFFFFFFFFu;

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
    uint32_t n_tape;      // adjoint kernel: value slots | adjoint slots << 16
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
