/*
 * rsr_oracle.c -- CPU restatement of rsr's fitness-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
 * rsr_b200/: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg load it.  The product path never calls it.
 *
 * It restates, in plain C with IEEE single-precision arithmetic and no
 * contraction (built with -ffp-contract=off), the reference algorithm:
 *
 *   typed-stack VM ........ src/engine/eval/evaluator.rs:20-150 (eval_simd)
 *                           src/engine/eval/state.rs:12-49 (32 zeroed slots/type)
 *   scalar ops ............ src/domains/basic/eval.rs:4-63
 *   linalg ops ............ src/domains/linalg/eval.rs:4-506
 *   compute_mse ........... src/engine/eval/evaluator.rs:153-174
 *   dual-number gradient .. src/engine/eval/evaluator.rs:177-388,
 *                           src/engine/eval/autodiff.rs:12-124,221-873,
 *                           dispatch src/domains/basic/mod.rs:205-220,
 *                           src/domains/linalg/mod.rs:502-690
 *   flat parameter order .. src/engine/expr/program.rs:84-145
 *   ISA numbering ......... src/engine/domain.rs:46-63, basic/mod.rs:9-20,
 *                           linalg/mod.rs:9-51
 *
 * Parity status.  The reference is Rust and cannot be built in this image
 * (no cargo/rustc, no crate cache), and its tests hold no golden vectors.
 * add/sub/mul/div/sqrt/compare are pinned by IEEE-754 itself and by the
 * known-answer targets of the reference's own tests (tests/basic.rs,
 * tests/linalg.rs).  sin/cos/exp/ln come from the third-party crate `wide`
 * 1.1.1 (Cargo.lock:506-508), whose source is absent: they are restated here
 * from the published Cephes method (S. L. Moshier, Cephes Math Library:
 * sinf.c/cosf.c/expf.c/logf.c), the method `wide` follows.  Their bit-level
 * parity with `wide` is UNPINNED; only error bounds against libm double are
 * checked.  The reduce_add lane order of `wide` is likewise unpinned.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <pthread.h>

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ ISA */
/* Instruction numbering follows the variant order of compose_engine!
 * (domain.rs:46-63) with BasicOpCode (basic/mod.rs:9-20) and LinalgOpCode
 * (linalg/mod.rs:9-51) appended in declaration order. */
enum {
    LOAD_VAR_F = 0, LOAD_CONST_F, LOAD_VAR_B, LOAD_CONST_B, LOAD_VAR_I, LOAD_CONST_I,
    LOAD_VAR_V2, LOAD_CONST_V2, LOAD_VAR_V3, LOAD_CONST_V3, LOAD_VAR_M2, LOAD_CONST_M2,
    LOAD_VAR_M3, LOAD_CONST_M3,
    ADD_F = 14, SUB_F, MUL_F, DIV_F, SIN_F, COS_F, EXP_F, SQR_F, SQRT_F, LN_F,
    MAKE_VEC2 = 24, MAKE_VEC3, GET_X_V2, GET_Y_V2, GET_X_V3, GET_Y_V3, GET_Z_V3,
    ADD_V2, SUB_V2, SCALE_V2, DOT_V2, NORM_V2,
    ADD_V3, SUB_V3, SCALE_V3, DOT_V3, NORM_V3, CROSS_V3,
    MAKE_MAT2, ADD_M2, SUB_M2, SCALE_M2, MUL_M2, MUL_M2V2, DET_M2, TRACE_M2, TRANSPOSE_M2, INVERSE_M2,
    MAKE_MAT3, ADD_M3, SUB_M3, SCALE_M3, MUL_M3, MUL_M3V3, DET_M3, TRACE_M3, TRANSPOSE_M3, INVERSE_M3,
    N_OPCODES
};

/* Scalar variants (scalar.rs:4-12) and their flat parameter widths
 * (program.rs:84-98; Int/Bool contribute none). */
enum { K_FLOAT = 0, K_INT, K_BOOL, K_VEC2, K_VEC3, K_MAT2, K_MAT3 };
static const int kind_width[7] = {1, 0, 0, 2, 3, 4, 9};

ORC_API int orc_n_opcodes(void) { return N_OPCODES; }

/* ------------------------------------------------------ transcendentals */
/* Cephes single-precision method, restated; Horner evaluation, unfused. */
static float pow2i(int k) { /* 2^k for k in [-126, 127] */
    union { uint32_t u; float f; } v;
    v.u = (uint32_t)(k + 127) << 23;
    return v.f;
}

ORC_API float orc_sinf(float x);
ORC_API float orc_cosf(float x);

static float sincos_core(float x, int want_cos) {
    const float TWO_OVER_PI = 0.636619772367581343f;
    const float DP1 = 1.5703125f, DP2 = 4.837512969970703125e-4f, DP3 = 7.54978995489188216e-8f;
    if (isnan(x) || isinf(x)) return NAN;
    float xa = fabsf(x);
    float yq = rintf(xa * TWO_OVER_PI);
    if (yq > 16777216.0f) return want_cos ? 1.0f : 0.0f; /* reduction meaningless */
    int q = (int)yq;
    float r = ((xa - yq * DP1) - yq * DP2) - yq * DP3;
    float r2 = r * r;
    float s = ((-1.9515295891e-4f * r2 + 8.3321608736e-3f) * r2 - 1.6666654611e-1f) * (r2 * r) + r;
    float c = ((2.443315711809948e-5f * r2 - 1.388731625493765e-3f) * r2 + 4.166664568298827e-2f) * (r2 * r2)
              + (1.0f - 0.5f * r2);
    float sv, cv;
    switch (q & 3) {
        case 0: sv = s; cv = c; break;
        case 1: sv = c; cv = -s; break;
        case 2: sv = -s; cv = -c; break;
        default: sv = -c; cv = s; break;
    }
    if (want_cos) return cv;
    return (x < 0.0f) ? -sv : sv;
}
ORC_API float orc_sinf(float x) { return sincos_core(x, 0); }
ORC_API float orc_cosf(float x) { return sincos_core(x, 1); }

ORC_API float orc_expf(float x) {
    if (isnan(x)) return x;
    if (x > 88.72283905206835f) return INFINITY;
    if (x < -103.278929903431851103f) return 0.0f;
    float z = floorf(1.44269504088896341f * x + 0.5f);
    float r = (x - z * 0.693359375f) - z * -2.12194440e-4f;
    int n = (int)z;
    float rr = r * r;
    float p = ((((1.9875691500e-4f * r + 1.3981999507e-3f) * r + 8.3334519073e-3f) * r + 4.1665795894e-2f) * r
               + 1.6666665459e-1f) * r + 5.0000001201e-1f;
    float y = (p * rr + r) + 1.0f;
    int n1 = n >> 1, n2 = n - n1;
    return (y * pow2i(n1)) * pow2i(n2);
}

ORC_API float orc_logf(float x) {
    const float SQRTHF = 0.707106781186547524f;
    if (isnan(x)) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (isinf(x)) return x;
    union { uint32_t u; float f; } v;
    v.f = x;
    int e_adj = 0;
    if (((v.u >> 23) & 0xFF) == 0) { v.f = x * 33554432.0f; e_adj = -25; } /* subnormal: scale by 2^25 */
    int e = (int)((v.u >> 23) & 0xFF) - 126 + e_adj;
    v.u = (v.u & 0x807FFFFFu) | (126u << 23); /* mantissa in [0.5, 1) */
    float m = v.f;
    if (m < SQRTHF) { e -= 1; m = (m + m) - 1.0f; } else { m = m - 1.0f; }
    float z = m * m;
    float y = ((((((((7.0376836292e-2f * m - 1.1514610310e-1f) * m + 1.1676998740e-1f) * m - 1.2420140846e-1f) * m
                  + 1.4249322787e-1f) * m - 1.6668057665e-1f) * m + 2.0000714765e-1f) * m - 2.4999993993e-1f) * m
               + 3.3333331174e-1f) * m * z;
    float fe = (float)e;
    y = y + -2.12194440e-4f * fe;
    y = y + -0.5f * z;
    float r = m + y;
    return r + 0.693359375f * fe;
}

/* ---------------------------------------------------------- programs */
typedef struct {
    const uint32_t *code;
    uint32_t len;
    const uint8_t *kinds;
    uint32_t n_consts;
    const float *params;
    uint32_t n_params;
} prog_t;

static inline uint32_t w_op(uint32_t w) { return w & 0xFFu; }
static inline uint32_t w_arg(uint32_t w) { return (w >> 8) & 0xFFFFu; }

/* get_flat_start_idx (evaluator.rs:232-245) */
static uint32_t flat_start(const prog_t *p, uint32_t cidx) {
    uint32_t s = 0;
    for (uint32_t c = 0; c < cidx && c < p->n_consts; ++c) s += kind_width[p->kinds[c]];
    return s;
}

/* ------------------------------------------------------ plain VM state */
typedef struct {
    float f[32], v2[32][2], v3[32][3], m2[32][4], m3[32][9];
    int sf, sv2, sv3, sm2, sm3;
} vm_t;

static void det_m3(const float *m, float *out) {
    *out = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7]) + m[6] * (m[1] * m[5] - m[2] * m[4]);
}

/* One instruction of eval_simd on one lane.  Returns 0, or -1 on a stack
 * error (the reference has undefined behaviour there; callers validate). */
static int vm_step(vm_t *s, const prog_t *p, const float *feat, uint32_t w) {
    uint32_t op = w_op(w), a = w_arg(w);
    float *A, *B, t[9];
    switch (op) {
    case LOAD_VAR_F: s->f[s->sf++] = feat[a]; break;
    case LOAD_CONST_F: /* a mismatched variant leaves the slot unwritten (evaluator.rs:37-40) */
        if (a < p->n_consts && p->kinds[a] == K_FLOAT) s->f[s->sf] = p->params[flat_start(p, a)];
        s->sf++; break;
    case LOAD_VAR_B: case LOAD_CONST_B: case LOAD_VAR_I: case LOAD_CONST_I: break; /* no-ops (domain.rs:286-293) */
    case LOAD_VAR_V2: s->v2[s->sv2][0] = feat[a]; s->v2[s->sv2][1] = feat[a + 1]; s->sv2++; break;
    case LOAD_CONST_V2:
        if (a < p->n_consts && p->kinds[a] == K_VEC2) { uint32_t o = flat_start(p, a); for (int i = 0; i < 2; ++i) s->v2[s->sv2][i] = p->params[o + i]; }
        s->sv2++; break;
    case LOAD_VAR_V3: for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = feat[a + i]; s->sv3++; break;
    case LOAD_CONST_V3:
        if (a < p->n_consts && p->kinds[a] == K_VEC3) { uint32_t o = flat_start(p, a); for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = p->params[o + i]; }
        s->sv3++; break;
    case LOAD_VAR_M2: for (int i = 0; i < 4; ++i) s->m2[s->sm2][i] = feat[a + i]; s->sm2++; break;
    case LOAD_CONST_M2:
        if (a < p->n_consts && p->kinds[a] == K_MAT2) { uint32_t o = flat_start(p, a); for (int i = 0; i < 4; ++i) s->m2[s->sm2][i] = p->params[o + i]; }
        s->sm2++; break;
    case LOAD_VAR_M3: for (int i = 0; i < 9; ++i) s->m3[s->sm3][i] = feat[a + i]; s->sm3++; break;
    case LOAD_CONST_M3:
        if (a < p->n_consts && p->kinds[a] == K_MAT3) { uint32_t o = flat_start(p, a); for (int i = 0; i < 9; ++i) s->m3[s->sm3][i] = p->params[o + i]; }
        s->sm3++; break;
    /* basic/eval.rs:4-63 */
    case ADD_F: s->sf -= 2; s->f[s->sf] = s->f[s->sf] + s->f[s->sf + 1]; s->sf++; break;
    case SUB_F: s->sf -= 2; s->f[s->sf] = s->f[s->sf] - s->f[s->sf + 1]; s->sf++; break;
    case MUL_F: s->sf -= 2; s->f[s->sf] = s->f[s->sf] * s->f[s->sf + 1]; s->sf++; break;
    case DIV_F: s->sf -= 2; s->f[s->sf] = s->f[s->sf] / s->f[s->sf + 1]; s->sf++; break;
    case SIN_F: s->f[s->sf - 1] = orc_sinf(s->f[s->sf - 1]); break;
    case COS_F: s->f[s->sf - 1] = orc_cosf(s->f[s->sf - 1]); break;
    case EXP_F: s->f[s->sf - 1] = orc_expf(s->f[s->sf - 1]); break;
    case SQR_F: s->f[s->sf - 1] = s->f[s->sf - 1] * s->f[s->sf - 1]; break;
    case SQRT_F: s->f[s->sf - 1] = sqrtf(s->f[s->sf - 1]); break;
    case LN_F: s->f[s->sf - 1] = orc_logf(s->f[s->sf - 1]); break;
    /* linalg/eval.rs */
    case MAKE_VEC2: s->sf -= 2; s->v2[s->sv2][0] = s->f[s->sf]; s->v2[s->sv2][1] = s->f[s->sf + 1]; s->sv2++; break;
    case MAKE_VEC3: s->sf -= 3; for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = s->f[s->sf + i]; s->sv3++; break;
    case GET_X_V2: s->sv2--; s->f[s->sf++] = s->v2[s->sv2][0]; break;
    case GET_Y_V2: s->sv2--; s->f[s->sf++] = s->v2[s->sv2][1]; break;
    case GET_X_V3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][0]; break;
    case GET_Y_V3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][1]; break;
    case GET_Z_V3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][2]; break;
    case ADD_V2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; A[0] = A[0] + B[0]; A[1] = A[1] + B[1]; s->sv2++; break;
    case SUB_V2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; A[0] = A[0] - B[0]; A[1] = A[1] - B[1]; s->sv2++; break;
    case SCALE_V2: { s->sf--; s->sv2--; float k = s->f[s->sf]; A = s->v2[s->sv2]; A[0] = A[0] * k; A[1] = A[1] * k; s->sv2++; break; }
    case DOT_V2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; s->f[s->sf++] = (A[0] * B[0]) + (A[1] * B[1]); break;
    case NORM_V2: A = s->v2[s->sv2 - 1]; s->f[s->sf++] = sqrtf((A[0] * A[0]) + (A[1] * A[1])); s->sv2--; break;
    case ADD_V3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = A[i] + B[i]; s->sv3++; break;
    case SUB_V3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = A[i] - B[i]; s->sv3++; break;
    case SCALE_V3: { s->sf--; s->sv3--; float k = s->f[s->sf]; A = s->v3[s->sv3]; for (int i = 0; i < 3; ++i) A[i] = A[i] * k; s->sv3++; break; }
    case DOT_V3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; s->f[s->sf++] = (A[0] * B[0]) + (A[1] * B[1]) + (A[2] * B[2]); break;
    case NORM_V3: A = s->v3[s->sv3 - 1]; s->f[s->sf++] = sqrtf((A[0] * A[0]) + (A[1] * A[1]) + (A[2] * A[2])); s->sv3--; break;
    case CROSS_V3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1];
        t[0] = A[1] * B[2] - A[2] * B[1]; t[1] = A[2] * B[0] - A[0] * B[2]; t[2] = A[0] * B[1] - A[1] * B[0];
        memcpy(A, t, 3 * sizeof(float)); s->sv3++; break;
    case MAKE_MAT2: s->sv2 -= 2; A = s->m2[s->sm2];
        A[0] = s->v2[s->sv2][0]; A[1] = s->v2[s->sv2][1]; A[2] = s->v2[s->sv2 + 1][0]; A[3] = s->v2[s->sv2 + 1][1]; s->sm2++; break;
    case ADD_M2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = A[i] + B[i]; s->sm2++; break;
    case SUB_M2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = A[i] - B[i]; s->sm2++; break;
    case SCALE_M2: { s->sf--; s->sm2--; float k = s->f[s->sf]; A = s->m2[s->sm2]; for (int i = 0; i < 4; ++i) A[i] = A[i] * k; s->sm2++; break; }
    case MUL_M2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1];
        t[0] = A[0] * B[0] + A[2] * B[1]; t[1] = A[1] * B[0] + A[3] * B[1];
        t[2] = A[0] * B[2] + A[2] * B[3]; t[3] = A[1] * B[2] + A[3] * B[3];
        memcpy(A, t, 4 * sizeof(float)); s->sm2++; break;
    case MUL_M2V2: s->sm2--; s->sv2--; A = s->m2[s->sm2]; B = s->v2[s->sv2];
        t[0] = A[0] * B[0] + A[2] * B[1]; t[1] = A[1] * B[0] + A[3] * B[1]; B[0] = t[0]; B[1] = t[1]; s->sv2++; break;
    case DET_M2: s->sm2--; A = s->m2[s->sm2]; s->f[s->sf++] = (A[0] * A[3]) - (A[1] * A[2]); break;
    case TRACE_M2: s->sm2--; A = s->m2[s->sm2]; s->f[s->sf++] = A[0] + A[3]; break;
    case TRANSPOSE_M2: A = s->m2[s->sm2 - 1]; { float x = A[1]; A[1] = A[2]; A[2] = x; } break;
    case INVERSE_M2: {
        A = s->m2[s->sm2 - 1];
        float det = (A[0] * A[3]) - (A[1] * A[2]);
        int sing = fabsf(det) < 1e-9f;
        float inv = 1.0f / (sing ? 1.0f : det);
        t[0] = sing ? 1.0f : A[3] * inv; t[1] = sing ? 0.0f : -A[1] * inv;
        t[2] = sing ? 0.0f : -A[2] * inv; t[3] = sing ? 1.0f : A[0] * inv;
        memcpy(A, t, 4 * sizeof(float)); break; }
    case MAKE_MAT3: s->sv3 -= 3; A = s->m3[s->sm3];
        for (int c = 0; c < 3; ++c) for (int i = 0; i < 3; ++i) A[3 * c + i] = s->v3[s->sv3 + c][i]; s->sm3++; break;
    case ADD_M3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = A[i] + B[i]; s->sm3++; break;
    case SUB_M3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = A[i] - B[i]; s->sm3++; break;
    case SCALE_M3: { s->sf--; s->sm3--; float k = s->f[s->sf]; A = s->m3[s->sm3]; for (int i = 0; i < 9; ++i) A[i] = A[i] * k; s->sm3++; break; }
    case MUL_M3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1];
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
            t[3 * c + r] = A[r] * B[3 * c] + A[3 + r] * B[3 * c + 1] + A[6 + r] * B[3 * c + 2];
        memcpy(A, t, 9 * sizeof(float)); s->sm3++; break;
    case MUL_M3V3: s->sm3--; s->sv3--; A = s->m3[s->sm3]; B = s->v3[s->sv3];
        for (int r = 0; r < 3; ++r) t[r] = A[r] * B[0] + A[3 + r] * B[1] + A[6 + r] * B[2];
        memcpy(B, t, 3 * sizeof(float)); s->sv3++; break;
    case DET_M3: s->sm3--; det_m3(s->m3[s->sm3], &s->f[s->sf]); s->sf++; break;
    case TRACE_M3: s->sm3--; A = s->m3[s->sm3]; s->f[s->sf++] = A[0] + A[4] + A[8]; break;
    case TRANSPOSE_M3: A = s->m3[s->sm3 - 1];
        t[0] = A[0]; t[1] = A[3]; t[2] = A[6]; t[3] = A[1]; t[4] = A[4]; t[5] = A[7]; t[6] = A[2]; t[7] = A[5]; t[8] = A[8];
        memcpy(A, t, 9 * sizeof(float)); break;
    case INVERSE_M3: {
        float *m = s->m3[s->sm3 - 1], det;
        det_m3(m, &det);
        int sing = fabsf(det) < 1e-9f;
        float inv = 1.0f / (sing ? 1.0f : det);
        float adj[9] = {
            (m[4] * m[8] - m[5] * m[7]) * inv, -(m[1] * m[8] - m[2] * m[7]) * inv, (m[1] * m[5] - m[2] * m[4]) * inv,
            -(m[3] * m[8] - m[5] * m[6]) * inv, (m[0] * m[8] - m[2] * m[6]) * inv, -(m[0] * m[5] - m[2] * m[3]) * inv,
            (m[3] * m[7] - m[4] * m[6]) * inv, -(m[0] * m[7] - m[1] * m[6]) * inv, (m[0] * m[4] - m[1] * m[3]) * inv};
        for (int i = 0; i < 9; ++i) m[i] = sing ? ((i % 4 == 0) ? 1.0f : 0.0f) : adj[i];
        break; }
    default: return -1;
    }
    return 0;
}

/* eval_simd for one data point (one SIMD lane): zeroed state, result stack_f[0]. */
static float eval_point(const prog_t *p, const float *feat) {
    vm_t s;
    memset(&s, 0, sizeof(s));
    for (uint32_t pc = 0; pc < p->len; ++pc) vm_step(&s, p, feat, p->code[pc]);
    return s.f[0];
}

/* ------------------------------------------------------ validation */
/* Per-type stack simulation: checks underflow, the 32-slot limit
 * (state.rs:14), feature and constant indices.  Returns 0 if valid. */
static const signed char op_pops[N_OPCODES][5] = {
    /* F, V2, V3, M2, M3 pops; pushes are in op_push below */
    [ADD_F] = {2}, [SUB_F] = {2}, [MUL_F] = {2}, [DIV_F] = {2},
    [SIN_F] = {1}, [COS_F] = {1}, [EXP_F] = {1}, [SQR_F] = {1}, [SQRT_F] = {1}, [LN_F] = {1},
    [MAKE_VEC2] = {2}, [MAKE_VEC3] = {3},
    [GET_X_V2] = {0, 1}, [GET_Y_V2] = {0, 1}, [GET_X_V3] = {0, 0, 1}, [GET_Y_V3] = {0, 0, 1}, [GET_Z_V3] = {0, 0, 1},
    [ADD_V2] = {0, 2}, [SUB_V2] = {0, 2}, [SCALE_V2] = {1, 1}, [DOT_V2] = {0, 2}, [NORM_V2] = {0, 1},
    [ADD_V3] = {0, 0, 2}, [SUB_V3] = {0, 0, 2}, [SCALE_V3] = {1, 0, 1}, [DOT_V3] = {0, 0, 2}, [NORM_V3] = {0, 0, 1},
    [CROSS_V3] = {0, 0, 2},
    [MAKE_MAT2] = {0, 2}, [ADD_M2] = {0, 0, 0, 2}, [SUB_M2] = {0, 0, 0, 2}, [SCALE_M2] = {1, 0, 0, 1},
    [MUL_M2] = {0, 0, 0, 2}, [MUL_M2V2] = {0, 1, 0, 1}, [DET_M2] = {0, 0, 0, 1}, [TRACE_M2] = {0, 0, 0, 1},
    [TRANSPOSE_M2] = {0, 0, 0, 1}, [INVERSE_M2] = {0, 0, 0, 1},
    [MAKE_MAT3] = {0, 0, 3}, [ADD_M3] = {0, 0, 0, 0, 2}, [SUB_M3] = {0, 0, 0, 0, 2}, [SCALE_M3] = {1, 0, 0, 0, 1},
    [MUL_M3] = {0, 0, 0, 0, 2}, [MUL_M3V3] = {0, 0, 1, 0, 1}, [DET_M3] = {0, 0, 0, 0, 1}, [TRACE_M3] = {0, 0, 0, 0, 1},
    [TRANSPOSE_M3] = {0, 0, 0, 0, 1}, [INVERSE_M3] = {0, 0, 0, 0, 1},
};
static const signed char op_push[N_OPCODES] = {
    [LOAD_VAR_F] = 0, [LOAD_CONST_F] = 0, [LOAD_VAR_B] = -1, [LOAD_CONST_B] = -1, [LOAD_VAR_I] = -1, [LOAD_CONST_I] = -1,
    [LOAD_VAR_V2] = 1, [LOAD_CONST_V2] = 1, [LOAD_VAR_V3] = 2, [LOAD_CONST_V3] = 2, [LOAD_VAR_M2] = 3,
    [LOAD_CONST_M2] = 3, [LOAD_VAR_M3] = 4, [LOAD_CONST_M3] = 4,
    [ADD_F] = 0, [SUB_F] = 0, [MUL_F] = 0, [DIV_F] = 0, [SIN_F] = 0, [COS_F] = 0, [EXP_F] = 0, [SQR_F] = 0,
    [SQRT_F] = 0, [LN_F] = 0,
    [MAKE_VEC2] = 1, [MAKE_VEC3] = 2, [GET_X_V2] = 0, [GET_Y_V2] = 0, [GET_X_V3] = 0, [GET_Y_V3] = 0, [GET_Z_V3] = 0,
    [ADD_V2] = 1, [SUB_V2] = 1, [SCALE_V2] = 1, [DOT_V2] = 0, [NORM_V2] = 0,
    [ADD_V3] = 2, [SUB_V3] = 2, [SCALE_V3] = 2, [DOT_V3] = 0, [NORM_V3] = 0, [CROSS_V3] = 2,
    [MAKE_MAT2] = 3, [ADD_M2] = 3, [SUB_M2] = 3, [SCALE_M2] = 3, [MUL_M2] = 3, [MUL_M2V2] = 1, [DET_M2] = 0,
    [TRACE_M2] = 0, [TRANSPOSE_M2] = 3, [INVERSE_M2] = 3,
    [MAKE_MAT3] = 4, [ADD_M3] = 4, [SUB_M3] = 4, [SCALE_M3] = 4, [MUL_M3] = 4, [MUL_M3V3] = 2, [DET_M3] = 0,
    [TRACE_M3] = 0, [TRANSPOSE_M3] = 4, [INVERSE_M3] = 4,
};
static const int type_width[5] = {1, 2, 3, 4, 9};

ORC_API int orc_validate(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t n_consts,
                         uint32_t n_params, uint32_t num_features) {
    int sp[5] = {0, 0, 0, 0, 0};
    uint32_t need = 0;
    for (uint32_t c = 0; c < n_consts; ++c) { if (kinds[c] > K_MAT3) return -5; need += kind_width[kinds[c]]; }
    if (need != n_params) return -6;
    for (uint32_t pc = 0; pc < len; ++pc) {
        uint32_t op = w_op(code[pc]), a = w_arg(code[pc]);
        if (op >= N_OPCODES) return -1;
        if (op <= LOAD_CONST_M3) {
            int t = op_push[op];
            if (t < 0) continue;
            if ((op & 1) == 0) { if (a + type_width[t] > num_features) return -3; }
            else if (a >= n_consts) return -4;
        } else {
            for (int t = 0; t < 5; ++t) { sp[t] -= op_pops[op][t]; if (sp[t] < 0) return -2; }
        }
        int t = op_push[op];
        if (t >= 0) { sp[t] += 1; if (sp[t] > 32) return -7; }
    }
    return 0;
}

/* ---------------------------------------------------------- exports */
static prog_t mkprog(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk, const float *params,
                     uint32_t np) {
    prog_t p = {code, len, kinds, nk, params, np};
    return p;
}

/* Per-point predictions over an AoSoA dataset (dataset.rs:96-154 layout:
 * feature_flat[b*F + f] holds 8 consecutive points). out has nbatch*8. */
ORC_API void orc_eval_points(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                             const float *params, uint32_t np, const float *feature_flat, uint32_t nf,
                             uint64_t nbatch, float *out) {
    prog_t p = mkprog(code, len, kinds, nk, params, np);
    float feat[256];
    for (uint64_t b = 0; b < nbatch; ++b)
        for (int l = 0; l < 8; ++l) {
            for (uint32_t f = 0; f < nf; ++f) feat[f] = feature_flat[(b * nf + f) * 8 + l];
            out[b * 8 + l] = eval_point(&p, feat);
        }
}

/* reduce_add of an f32x8: halving-tree order, unpinned against `wide`. */
static float reduce8(const float *v) {
    float a0 = v[0] + v[4], a1 = v[1] + v[5], a2 = v[2] + v[6], a3 = v[3] + v[7];
    return (a0 + a2) + (a1 + a3);
}

/* compute_mse (evaluator.rs:153-174): per-lane f32 accumulation over all
 * padded batches, reduce_add, divide by num_samples, non-finite -> f32::MAX. */
ORC_API float orc_mse_ref32(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                            const float *params, uint32_t np, const float *feature_flat, const float *target,
                            uint32_t nf, uint64_t nbatch, uint64_t nsamples) {
    prog_t p = mkprog(code, len, kinds, nk, params, np);
    float acc[8] = {0}, feat[256];
    for (uint64_t b = 0; b < nbatch; ++b)
        for (int l = 0; l < 8; ++l) {
            for (uint32_t f = 0; f < nf; ++f) feat[f] = feature_flat[(b * nf + f) * 8 + l];
            float d = eval_point(&p, feat) - target[b * 8 + l];
            acc[l] = acc[l] + d * d;
        }
    float mse = reduce8(acc) / (float)nsamples;
    return isfinite(mse) ? mse : FLT_MAX;
}

/* FP64 oracle: f32 predictions, squared error summed in double over all
 * padded points, divided by num_samples.  Non-finite -> inf (the caller
 * classifies). */
ORC_API double orc_mse_f64(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                           const float *params, uint32_t np, const float *feature_flat, const float *target,
                           uint32_t nf, uint64_t nbatch, uint64_t nsamples) {
    prog_t p = mkprog(code, len, kinds, nk, params, np);
    double acc = 0.0;
    float feat[256];
    for (uint64_t b = 0; b < nbatch; ++b)
        for (int l = 0; l < 8; ++l) {
            for (uint32_t f = 0; f < nf; ++f) feat[f] = feature_flat[(b * nf + f) * 8 + l];
            double d = (double)eval_point(&p, feat) - (double)target[b * 8 + l];
            acc += d * d;
        }
    return acc / (double)nsamples;
}

/* ------------------------------------------------------ dual numbers */
/* DualSimd restated per lane (autodiff.rs:12-124). */
typedef struct { float v, g; } dual;
static inline dual dconst(float v) { dual d = {v, 0.0f}; return d; }
static inline dual dadd(dual a, dual b) { dual r = {a.v + b.v, a.g + b.g}; return r; }
static inline dual dsub(dual a, dual b) { dual r = {a.v - b.v, a.g - b.g}; return r; }
static inline dual dmul(dual a, dual b) { dual r = {a.v * b.v, (a.v * b.g) + (a.g * b.v)}; return r; }
static inline dual ddiv(dual a, dual b) { dual r = {a.v / b.v, ((a.g * b.v) - (a.v * b.g)) / (b.v * b.v)}; return r; }
static inline dual dsin(dual a) { dual r = {orc_sinf(a.v), a.g * orc_cosf(a.v)}; return r; }
static inline dual dcos(dual a) { dual r = {orc_cosf(a.v), a.g * (-orc_sinf(a.v))}; return r; }
static inline dual dexp(dual a) { float e = orc_expf(a.v); dual r = {e, a.g * e}; return r; }
static inline dual dsqr(dual a) { dual r = {a.v * a.v, (2.0f * a.v) * a.g}; return r; }
static inline dual dsqrt(dual a) { float s = sqrtf(a.v); dual r = {s, a.g / (2.0f * s)}; return r; }
static inline dual dln(dual a) { dual r = {orc_logf(a.v), a.g / a.v}; return r; }

typedef struct {
    dual f[32], v2[32][2], v3[32][3], m2[32][4], m3[32][9];
    int sf, sv2, sv3, sm2, sm3;
} dvm_t;

static dual det_m3_dual(const dual *m) {
    return dadd(dsub(dmul(m[0], dsub(dmul(m[4], m[8]), dmul(m[5], m[7]))),
                     dmul(m[3], dsub(dmul(m[1], m[8]), dmul(m[2], m[7])))),
                dmul(m[6], dsub(dmul(m[1], m[5]), dmul(m[2], m[4]))));
}

/* eval_simd_dual on one lane, seeded on flat parameter k (evaluator.rs:228-388). */
static dual eval_point_dual(const prog_t *p, const float *feat, uint32_t k) {
    dvm_t s;
    memset(&s, 0, sizeof(s));
    for (uint32_t pc = 0; pc < p->len; ++pc) {
        uint32_t op = w_op(p->code[pc]), a = w_arg(p->code[pc]);
        dual *A, *B, t[9];
        switch (op) {
        case LOAD_VAR_F: s.f[s.sf++] = dconst(feat[a]); break;
        case LOAD_VAR_V2: for (int i = 0; i < 2; ++i) s.v2[s.sv2][i] = dconst(feat[a + i]); s.sv2++; break;
        case LOAD_VAR_V3: for (int i = 0; i < 3; ++i) s.v3[s.sv3][i] = dconst(feat[a + i]); s.sv3++; break;
        case LOAD_VAR_M2: for (int i = 0; i < 4; ++i) s.m2[s.sm2][i] = dconst(feat[a + i]); s.sm2++; break;
        case LOAD_VAR_M3: for (int i = 0; i < 9; ++i) s.m3[s.sm3][i] = dconst(feat[a + i]); s.sm3++; break;
        case LOAD_CONST_F: case LOAD_CONST_V2: case LOAD_CONST_V3: case LOAD_CONST_M2: case LOAD_CONST_M3: {
            static const int want[] = {[LOAD_CONST_F] = K_FLOAT, [LOAD_CONST_V2] = K_VEC2, [LOAD_CONST_V3] = K_VEC3,
                                       [LOAD_CONST_M2] = K_MAT2, [LOAD_CONST_M3] = K_MAT3};
            int kind = want[op], w = kind_width[kind];
            dual *dst = op == LOAD_CONST_F ? &s.f[s.sf] : op == LOAD_CONST_V2 ? s.v2[s.sv2]
                      : op == LOAD_CONST_V3 ? s.v3[s.sv3] : op == LOAD_CONST_M2 ? s.m2[s.sm2] : s.m3[s.sm3];
            if (a < p->n_consts && p->kinds[a] == kind) {
                uint32_t o = flat_start(p, a);
                for (int i = 0; i < w; ++i) { dst[i].v = p->params[o + i]; dst[i].g = (o + i == k) ? 1.0f : 0.0f; }
            }
            if (op == LOAD_CONST_F) s.sf++; else if (op == LOAD_CONST_V2) s.sv2++; else if (op == LOAD_CONST_V3) s.sv3++;
            else if (op == LOAD_CONST_M2) s.sm2++; else s.sm3++;
            break; }
        case ADD_F: s.sf -= 2; s.f[s.sf] = dadd(s.f[s.sf], s.f[s.sf + 1]); s.sf++; break;
        case SUB_F: s.sf -= 2; s.f[s.sf] = dsub(s.f[s.sf], s.f[s.sf + 1]); s.sf++; break;
        case MUL_F: s.sf -= 2; s.f[s.sf] = dmul(s.f[s.sf], s.f[s.sf + 1]); s.sf++; break;
        case DIV_F: s.sf -= 2; s.f[s.sf] = ddiv(s.f[s.sf], s.f[s.sf + 1]); s.sf++; break;
        case SIN_F: s.f[s.sf - 1] = dsin(s.f[s.sf - 1]); break;
        case COS_F: s.f[s.sf - 1] = dcos(s.f[s.sf - 1]); break;
        case EXP_F: s.f[s.sf - 1] = dexp(s.f[s.sf - 1]); break;
        case SQR_F: s.f[s.sf - 1] = dsqr(s.f[s.sf - 1]); break;
        case SQRT_F: s.f[s.sf - 1] = dsqrt(s.f[s.sf - 1]); break;
        case LN_F: s.f[s.sf - 1] = dln(s.f[s.sf - 1]); break;
        case MAKE_VEC2: s.sf -= 2; s.v2[s.sv2][0] = s.f[s.sf]; s.v2[s.sv2][1] = s.f[s.sf + 1]; s.sv2++; break;
        case MAKE_VEC3: s.sf -= 3; for (int i = 0; i < 3; ++i) s.v3[s.sv3][i] = s.f[s.sf + i]; s.sv3++; break;
        case GET_X_V2: s.sv2--; s.f[s.sf++] = s.v2[s.sv2][0]; break;
        case GET_Y_V2: s.sv2--; s.f[s.sf++] = s.v2[s.sv2][1]; break;
        case GET_X_V3: s.sv3--; s.f[s.sf++] = s.v3[s.sv3][0]; break;
        case GET_Y_V3: s.sv3--; s.f[s.sf++] = s.v3[s.sv3][1]; break;
        case GET_Z_V3: s.sv3--; s.f[s.sf++] = s.v3[s.sv3][2]; break;
        case ADD_V2: s.sv2 -= 2; A = s.v2[s.sv2]; B = s.v2[s.sv2 + 1]; for (int i = 0; i < 2; ++i) A[i] = dadd(A[i], B[i]); s.sv2++; break;
        case SUB_V2: s.sv2 -= 2; A = s.v2[s.sv2]; B = s.v2[s.sv2 + 1]; for (int i = 0; i < 2; ++i) A[i] = dsub(A[i], B[i]); s.sv2++; break;
        case SCALE_V2: { s.sf--; s.sv2--; dual q = s.f[s.sf]; A = s.v2[s.sv2]; for (int i = 0; i < 2; ++i) A[i] = dmul(A[i], q); s.sv2++; break; }
        case DOT_V2: s.sv2 -= 2; A = s.v2[s.sv2]; B = s.v2[s.sv2 + 1]; s.f[s.sf++] = dadd(dmul(A[0], B[0]), dmul(A[1], B[1])); break;
        case NORM_V2: A = s.v2[s.sv2 - 1]; s.f[s.sf++] = dsqrt(dadd(dmul(A[0], A[0]), dmul(A[1], A[1]))); s.sv2--; break;
        case ADD_V3: s.sv3 -= 2; A = s.v3[s.sv3]; B = s.v3[s.sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = dadd(A[i], B[i]); s.sv3++; break;
        case SUB_V3: s.sv3 -= 2; A = s.v3[s.sv3]; B = s.v3[s.sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = dsub(A[i], B[i]); s.sv3++; break;
        case SCALE_V3: { s.sf--; s.sv3--; dual q = s.f[s.sf]; A = s.v3[s.sv3]; for (int i = 0; i < 3; ++i) A[i] = dmul(A[i], q); s.sv3++; break; }
        case DOT_V3: { /* dual_dot_v3 (autodiff.rs:127-134) */
            s.sv3 -= 2; A = s.v3[s.sv3]; B = s.v3[s.sv3 + 1];
            dual r;
            r.v = (A[0].v * B[0].v) + (A[1].v * B[1].v) + (A[2].v * B[2].v);
            r.g = (A[0].v * B[0].g + A[0].g * B[0].v) + (A[1].v * B[1].g + A[1].g * B[1].v)
                + (A[2].v * B[2].g + A[2].g * B[2].v);
            s.f[s.sf++] = r; break; }
        case NORM_V3: A = s.v3[s.sv3 - 1];
            s.f[s.sf++] = dsqrt(dadd(dadd(dmul(A[0], A[0]), dmul(A[1], A[1])), dmul(A[2], A[2]))); s.sv3--; break;
        case CROSS_V3: s.sv3 -= 2; A = s.v3[s.sv3]; B = s.v3[s.sv3 + 1];
            t[0] = dsub(dmul(A[1], B[2]), dmul(A[2], B[1])); t[1] = dsub(dmul(A[2], B[0]), dmul(A[0], B[2]));
            t[2] = dsub(dmul(A[0], B[1]), dmul(A[1], B[0])); memcpy(A, t, 3 * sizeof(dual)); s.sv3++; break;
        case MAKE_MAT2: s.sv2 -= 2; A = s.m2[s.sm2];
            A[0] = s.v2[s.sv2][0]; A[1] = s.v2[s.sv2][1]; A[2] = s.v2[s.sv2 + 1][0]; A[3] = s.v2[s.sv2 + 1][1]; s.sm2++; break;
        case ADD_M2: s.sm2 -= 2; A = s.m2[s.sm2]; B = s.m2[s.sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = dadd(A[i], B[i]); s.sm2++; break;
        case SUB_M2: s.sm2 -= 2; A = s.m2[s.sm2]; B = s.m2[s.sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = dsub(A[i], B[i]); s.sm2++; break;
        case SCALE_M2: { s.sf--; s.sm2--; dual q = s.f[s.sf]; A = s.m2[s.sm2]; for (int i = 0; i < 4; ++i) A[i] = dmul(A[i], q); s.sm2++; break; }
        case MUL_M2: s.sm2 -= 2; A = s.m2[s.sm2]; B = s.m2[s.sm2 + 1];
            t[0] = dadd(dmul(A[0], B[0]), dmul(A[2], B[1])); t[1] = dadd(dmul(A[1], B[0]), dmul(A[3], B[1]));
            t[2] = dadd(dmul(A[0], B[2]), dmul(A[2], B[3])); t[3] = dadd(dmul(A[1], B[2]), dmul(A[3], B[3]));
            memcpy(A, t, 4 * sizeof(dual)); s.sm2++; break;
        case MUL_M2V2: s.sm2--; s.sv2--; A = s.m2[s.sm2]; B = s.v2[s.sv2];
            t[0] = dadd(dmul(A[0], B[0]), dmul(A[2], B[1])); t[1] = dadd(dmul(A[1], B[0]), dmul(A[3], B[1]));
            B[0] = t[0]; B[1] = t[1]; s.sv2++; break;
        case DET_M2: s.sm2--; A = s.m2[s.sm2]; s.f[s.sf++] = dsub(dmul(A[0], A[3]), dmul(A[1], A[2])); break;
        case TRACE_M2: s.sm2--; A = s.m2[s.sm2]; s.f[s.sf++] = dadd(A[0], A[3]); break;
        case TRANSPOSE_M2: A = s.m2[s.sm2 - 1]; { dual x = A[1]; A[1] = A[2]; A[2] = x; } break;
        case INVERSE_M2: case INVERSE_M3: break; /* the reference's dual dispatch is a no-op (linalg/mod.rs:643,687) */
        case MAKE_MAT3: s.sv3 -= 3; A = s.m3[s.sm3];
            for (int c = 0; c < 3; ++c) for (int i = 0; i < 3; ++i) A[3 * c + i] = s.v3[s.sv3 + c][i]; s.sm3++; break;
        case ADD_M3: s.sm3 -= 2; A = s.m3[s.sm3]; B = s.m3[s.sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = dadd(A[i], B[i]); s.sm3++; break;
        case SUB_M3: s.sm3 -= 2; A = s.m3[s.sm3]; B = s.m3[s.sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = dsub(A[i], B[i]); s.sm3++; break;
        case SCALE_M3: { s.sf--; s.sm3--; dual q = s.f[s.sf]; A = s.m3[s.sm3]; for (int i = 0; i < 9; ++i) A[i] = dmul(A[i], q); s.sm3++; break; }
        case MUL_M3: s.sm3 -= 2; A = s.m3[s.sm3]; B = s.m3[s.sm3 + 1];
            for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
                t[3 * c + r] = dadd(dadd(dmul(A[r], B[3 * c]), dmul(A[3 + r], B[3 * c + 1])), dmul(A[6 + r], B[3 * c + 2]));
            memcpy(A, t, 9 * sizeof(dual)); s.sm3++; break;
        case MUL_M3V3: s.sm3--; s.sv3--; A = s.m3[s.sm3]; B = s.v3[s.sv3];
            for (int r = 0; r < 3; ++r) t[r] = dadd(dadd(dmul(A[r], B[0]), dmul(A[3 + r], B[1])), dmul(A[6 + r], B[2]));
            memcpy(B, t, 3 * sizeof(dual)); s.sv3++; break;
        case DET_M3: s.sm3--; s.f[s.sf++] = det_m3_dual(s.m3[s.sm3]); break;
        case TRACE_M3: s.sm3--; A = s.m3[s.sm3]; s.f[s.sf++] = dadd(dadd(A[0], A[4]), A[8]); break;
        case TRANSPOSE_M3: A = s.m3[s.sm3 - 1];
            t[0] = A[0]; t[1] = A[3]; t[2] = A[6]; t[3] = A[1]; t[4] = A[4]; t[5] = A[7]; t[6] = A[2]; t[7] = A[5]; t[8] = A[8];
            memcpy(A, t, 9 * sizeof(dual)); break;
        default: break;
        }
    }
    return s.f[0];
}

/* compute_mse_with_gradient (evaluator.rs:177-224), restated per lane.
 * grad has 32 entries; entries >= min(P, 32) are zero.  Returns the MSE. */
ORC_API float orc_mse_grad_dual(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                                const float *params, uint32_t np, const float *feature_flat, const float *target,
                                uint32_t nf, uint64_t nbatch, uint64_t nsamples, float *grad) {
    prog_t p = mkprog(code, len, kinds, nk, params, np);
    uint32_t P = np < 32 ? np : 32;
    for (int k = 0; k < 32; ++k) grad[k] = 0.0f;
    if (P == 0) return orc_mse_ref32(code, len, kinds, nk, params, np, feature_flat, target, nf, nbatch, nsamples);
    float sse[8] = {0}, gs[32][8];
    memset(gs, 0, sizeof(gs));
    float feat[256];
    for (uint64_t b = 0; b < nbatch; ++b)
        for (int l = 0; l < 8; ++l) {
            for (uint32_t f = 0; f < nf; ++f) feat[f] = feature_flat[(b * nf + f) * 8 + l];
            float diff = 0.0f;
            for (uint32_t k = 0; k < P; ++k) {
                dual r = eval_point_dual(&p, feat, k);
                if (k == 0) { diff = r.v - target[b * 8 + l]; sse[l] = sse[l] + diff * diff; }
                gs[k][l] = gs[k][l] + (2.0f * diff) * r.g;
            }
        }
    float n = (float)nsamples;
    float mse = reduce8(sse) / n;
    if (!isfinite(mse)) return FLT_MAX;
    for (uint32_t k = 0; k < P; ++k) grad[k] = reduce8(gs[k]) / n;
    return mse;
}

/* Central finite differences of the FP64-oracle MSE with respect to each
 * flat parameter: (mse(p + h e_k) - mse(p - h e_k)) / (2h), with the
 * perturbed parameter rounded to f32 and the actual step used. */
ORC_API void orc_grad_fd(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                         const float *params, uint32_t np, const float *feature_flat, const float *target,
                         uint32_t nf, uint64_t nbatch, uint64_t nsamples, double h, double *grad) {
    float *q = (float *)malloc(sizeof(float) * (np ? np : 1));
    for (uint32_t k = 0; k < np; ++k) {
        memcpy(q, params, sizeof(float) * np);
        float hi = (float)((double)params[k] + h), lo = (float)((double)params[k] - h);
        q[k] = hi;
        double fp = orc_mse_f64(code, len, kinds, nk, q, np, feature_flat, target, nf, nbatch, nsamples);
        q[k] = lo;
        double fm = orc_mse_f64(code, len, kinds, nk, q, np, feature_flat, target, nf, nbatch, nsamples);
        grad[k] = (fp - fm) / ((double)hi - (double)lo);
    }
    free(q);
}

/* The dual-number gradient of orc_mse_grad_dual (the reference's per-point
 * rules, evaluator.rs:228-388, in f32) with the sums over points taken in
 * f64 instead of per-lane f32, for datasets of a million points where the
 * reference's f32 accumulation would add noise of its own.  Also returns,
 * per flat parameter k, the L1 scale of the sum: l1[k] = sum |2 diff_i
 * dpred_i/dtheta_k| / num_samples.  A component whose value is small
 * against its L1 scale is a cancellation of large per-point terms, and an
 * f32 evaluation of it cannot be resolved below that scale times the
 * per-point rounding.  Returns the f64 MSE. */
ORC_API double orc_grad_dual_f64(const uint32_t *code, uint32_t len, const uint8_t *kinds, uint32_t nk,
                                 const float *params, uint32_t np, const float *feature_flat, const float *target,
                                 uint32_t nf, uint64_t nbatch, uint64_t nsamples, double *grad, double *l1) {
    prog_t p = mkprog(code, len, kinds, nk, params, np);
    uint32_t P = np < 32 ? np : 32;
    for (int k = 0; k < 32; ++k) grad[k] = l1[k] = 0.0;
    double sse = 0.0;
    float feat[256];
    for (uint64_t b = 0; b < nbatch; ++b)
        for (int l = 0; l < 8; ++l) {
            for (uint32_t f = 0; f < nf; ++f) feat[f] = feature_flat[(b * nf + f) * 8 + l];
            if (P == 0) {
                double d = (double)eval_point(&p, feat) - (double)target[b * 8 + l];
                sse += d * d;
                continue;
            }
            float diff = 0.0f;
            for (uint32_t k = 0; k < P; ++k) {
                dual r = eval_point_dual(&p, feat, k);
                if (k == 0) {
                    diff = r.v - target[b * 8 + l];
                    sse += (double)diff * (double)diff;
                }
                const double t = (2.0 * (double)diff) * (double)r.g;
                grad[k] += t;
                l1[k] += fabs(t);
            }
        }
    const double n = (double)nsamples;
    for (uint32_t k = 0; k < P; ++k) {
        grad[k] /= n;
        l1[k] /= n;
    }
    return sse / n;
}

/* ---------------------------------------------- batched, multi-threaded */
/* Packed population: code/kinds/params concatenated with offset arrays of
 * n+1 entries.  Used by tests at sizes where a Python loop would be slow. */
typedef struct {
    const uint32_t *code; const uint64_t *code_off;
    const uint8_t *kinds; const uint64_t *kind_off;
    const float *params; const uint64_t *param_off;
    const float *ff; const float *tg; uint32_t nf; uint64_t nbatch, nsamples;
    double *mse64; float *mse32;
    uint32_t n, next; pthread_mutex_t mu;
} batch_job_t;

static void *batch_worker(void *arg) {
    batch_job_t *J = (batch_job_t *)arg;
    for (;;) {
        pthread_mutex_lock(&J->mu);
        uint32_t i = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (i >= J->n) break;
        const uint32_t *c = J->code + J->code_off[i];
        uint32_t len = (uint32_t)(J->code_off[i + 1] - J->code_off[i]);
        const uint8_t *k = J->kinds + J->kind_off[i];
        uint32_t nk = (uint32_t)(J->kind_off[i + 1] - J->kind_off[i]);
        const float *pp = J->params + J->param_off[i];
        uint32_t np = (uint32_t)(J->param_off[i + 1] - J->param_off[i]);
        if (J->mse64) J->mse64[i] = orc_mse_f64(c, len, k, nk, pp, np, J->ff, J->tg, J->nf, J->nbatch, J->nsamples);
        if (J->mse32) J->mse32[i] = orc_mse_ref32(c, len, k, nk, pp, np, J->ff, J->tg, J->nf, J->nbatch, J->nsamples);
    }
    return NULL;
}

ORC_API void orc_mse_batch(const uint32_t *code, const uint64_t *code_off, const uint8_t *kinds,
                           const uint64_t *kind_off, const float *params, const uint64_t *param_off, uint32_t n,
                           const float *feature_flat, const float *target, uint32_t nf, uint64_t nbatch,
                           uint64_t nsamples, int threads, double *mse64, float *mse32) {
    batch_job_t J = {code, code_off, kinds, kind_off, params, param_off, feature_flat, target, nf, nbatch, nsamples,
                     mse64, mse32, n, 0};
    pthread_mutex_init(&J.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, batch_worker, &J);
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&J.mu);
}
