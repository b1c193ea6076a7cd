/*
 * simd_baseline.c -- timed CPU baseline: an AVX2 8-lane restatement of the
 * reference's SIMD evaluator.
 *
 * TEST INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its reference
 * arm).  The reference is Rust and cannot be built in this image, so this
 * file keeps the reference's cost structure instead:
 *   - AoSoA 8-point batches (src/engine/data/dataset.rs:96-154);
 *   - a VmState of 5 typed stacks x 32 slots of f32x8, zeroed for every
 *     batch (src/engine/eval/state.rs:12-49);
 *   - one dispatch per instruction (evaluator.rs:24-146);
 *   - per-lane f32 accumulation and reduce_add (evaluator.rs:153-174);
 *   - compute_mse_with_gradient as P dual passes per batch
 *     (evaluator.rs:177-224).
 * Threads split the population, as rayon splits islands (engine.rs:52).
 * Arithmetic is unfused (no FMA), as in the reference's default build.
 */
#include <immintrin.h>
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <string.h>
#include <pthread.h>
#include <stdlib.h>

#define ORC_API __attribute__((visibility("default")))

typedef __m256 v8;
#define ADD _mm256_add_ps
#define SUB _mm256_sub_ps
#define MUL _mm256_mul_ps
#define DIV _mm256_div_ps
#define SPL _mm256_set1_ps

/* ----- vectorised Cephes transcendentals: same operation order as the
 * scalar restatement in rsr_oracle.c ----- */
static inline v8 v_pow2i(__m256i k) { return _mm256_castsi256_ps(_mm256_slli_epi32(_mm256_add_epi32(k, _mm256_set1_epi32(127)), 23)); }

static inline void v_sincos(v8 x, v8 *so, v8 *co) {
    v8 signmask = SPL(-0.0f);
    v8 xa = _mm256_andnot_ps(signmask, x);
    v8 yq = _mm256_round_ps(MUL(xa, SPL(0.636619772367581343f)), _MM_FROUND_TO_NEAREST_INT | _MM_FROUND_NO_EXC);
    __m256i q = _mm256_cvtps_epi32(yq);
    v8 r = SUB(SUB(SUB(xa, MUL(yq, SPL(1.5703125f))), MUL(yq, SPL(4.837512969970703125e-4f))),
               MUL(yq, SPL(7.54978995489188216e-8f)));
    v8 r2 = MUL(r, r);
    v8 s = ADD(MUL(SUB(MUL(ADD(MUL(SPL(-1.9515295891e-4f), r2), SPL(8.3321608736e-3f)), r2), SPL(1.6666654611e-1f)),
                   MUL(r2, r)), r);
    v8 c = ADD(MUL(ADD(MUL(SUB(MUL(SPL(2.443315711809948e-5f), r2), SPL(1.388731625493765e-3f)), r2),
                       SPL(4.166664568298827e-2f)), MUL(r2, r2)),
               SUB(SPL(1.0f), MUL(SPL(0.5f), r2)));
    __m256i q1 = _mm256_and_si256(q, _mm256_set1_epi32(1));
    v8 swap = _mm256_castsi256_ps(_mm256_cmpeq_epi32(q1, _mm256_set1_epi32(1)));
    v8 sv = _mm256_blendv_ps(s, c, swap), cv = _mm256_blendv_ps(c, s, swap);
    /* sin sign: (q & 2) xor (x < 0); cos sign: ((q + 1) & 2) */
    __m256i qs = _mm256_slli_epi32(_mm256_and_si256(q, _mm256_set1_epi32(2)), 30);
    __m256i qc = _mm256_slli_epi32(_mm256_and_si256(_mm256_add_epi32(q, _mm256_set1_epi32(1)), _mm256_set1_epi32(2)), 30);
    sv = _mm256_xor_ps(sv, _mm256_castsi256_ps(qs));
    sv = _mm256_xor_ps(sv, _mm256_and_ps(x, signmask));
    cv = _mm256_xor_ps(cv, _mm256_castsi256_ps(qc));
    v8 big = _mm256_cmp_ps(yq, SPL(16777216.0f), _CMP_GT_OQ);
    v8 bad = _mm256_cmp_ps(xa, SPL(INFINITY), _CMP_NLT_UQ); /* inf or nan */
    sv = _mm256_blendv_ps(sv, _mm256_setzero_ps(), big);
    cv = _mm256_blendv_ps(cv, SPL(1.0f), big);
    sv = _mm256_blendv_ps(sv, SPL(NAN), bad);
    cv = _mm256_blendv_ps(cv, SPL(NAN), bad);
    *so = sv; *co = cv;
}
static inline v8 v_sin(v8 x) { v8 s, c; v_sincos(x, &s, &c); return s; }
static inline v8 v_cos(v8 x) { v8 s, c; v_sincos(x, &s, &c); return c; }

static inline v8 v_exp(v8 x) {
    v8 z = _mm256_floor_ps(ADD(MUL(SPL(1.44269504088896341f), x), SPL(0.5f)));
    v8 r = SUB(SUB(x, MUL(z, SPL(0.693359375f))), MUL(z, SPL(-2.12194440e-4f)));
    v8 rr = MUL(r, r);
    v8 p = ADD(MUL(ADD(MUL(ADD(MUL(ADD(MUL(ADD(MUL(SPL(1.9875691500e-4f), r), SPL(1.3981999507e-3f)), r),
                                       SPL(8.3334519073e-3f)), r), SPL(4.1665795894e-2f)), r),
                       SPL(1.6666665459e-1f)), r), SPL(5.0000001201e-1f));
    v8 y = ADD(ADD(MUL(p, rr), r), SPL(1.0f));
    v8 zc = _mm256_max_ps(_mm256_min_ps(z, SPL(200.0f)), SPL(-200.0f));
    __m256i n = _mm256_cvtps_epi32(zc);
    __m256i n1 = _mm256_srai_epi32(n, 1), n2 = _mm256_sub_epi32(n, n1);
    n1 = _mm256_max_epi32(_mm256_min_epi32(n1, _mm256_set1_epi32(127)), _mm256_set1_epi32(-126));
    n2 = _mm256_max_epi32(_mm256_min_epi32(n2, _mm256_set1_epi32(127)), _mm256_set1_epi32(-126));
    v8 res = MUL(MUL(y, v_pow2i(n1)), v_pow2i(n2));
    res = _mm256_blendv_ps(res, SPL(INFINITY), _mm256_cmp_ps(x, SPL(88.72283905206835f), _CMP_GT_OQ));
    res = _mm256_blendv_ps(res, _mm256_setzero_ps(), _mm256_cmp_ps(x, SPL(-103.278929903431851103f), _CMP_LT_OQ));
    res = _mm256_blendv_ps(res, x, _mm256_cmp_ps(x, x, _CMP_UNORD_Q));
    return res;
}

static inline v8 v_log(v8 x) {
    v8 sub = _mm256_cmp_ps(x, SPL(1.17549435e-38f), _CMP_LT_OQ);
    v8 xs = _mm256_blendv_ps(x, MUL(x, SPL(33554432.0f)), sub);
    __m256i bits = _mm256_castps_si256(xs);
    __m256i e = _mm256_sub_epi32(_mm256_and_si256(_mm256_srli_epi32(bits, 23), _mm256_set1_epi32(0xFF)), _mm256_set1_epi32(126));
    e = _mm256_sub_epi32(e, _mm256_and_si256(_mm256_castps_si256(sub), _mm256_set1_epi32(25)));
    v8 m = _mm256_castsi256_ps(_mm256_or_si256(_mm256_and_si256(bits, _mm256_set1_epi32((int)0x807FFFFF)), _mm256_set1_epi32(126 << 23)));
    v8 lt = _mm256_cmp_ps(m, SPL(0.707106781186547524f), _CMP_LT_OQ);
    e = _mm256_sub_epi32(e, _mm256_and_si256(_mm256_castps_si256(lt), _mm256_set1_epi32(1)));
    m = _mm256_blendv_ps(SUB(m, SPL(1.0f)), SUB(ADD(m, m), SPL(1.0f)), lt);
    v8 z = MUL(m, m);
    v8 y = SPL(7.0376836292e-2f);
    y = SUB(MUL(y, m), SPL(1.1514610310e-1f));
    y = ADD(MUL(y, m), SPL(1.1676998740e-1f));
    y = SUB(MUL(y, m), SPL(1.2420140846e-1f));
    y = ADD(MUL(y, m), SPL(1.4249322787e-1f));
    y = SUB(MUL(y, m), SPL(1.6668057665e-1f));
    y = ADD(MUL(y, m), SPL(2.0000714765e-1f));
    y = SUB(MUL(y, m), SPL(2.4999993993e-1f));
    y = ADD(MUL(y, m), SPL(3.3333331174e-1f));
    y = MUL(MUL(y, m), z);
    v8 fe = _mm256_cvtepi32_ps(e);
    y = ADD(y, MUL(SPL(-2.12194440e-4f), fe));
    y = ADD(y, MUL(SPL(-0.5f), z));
    v8 r = ADD(ADD(m, y), MUL(SPL(0.693359375f), fe));
    r = _mm256_blendv_ps(r, SPL(NAN), _mm256_cmp_ps(x, _mm256_setzero_ps(), _CMP_LT_OQ));
    r = _mm256_blendv_ps(r, SPL(-INFINITY), _mm256_cmp_ps(x, _mm256_setzero_ps(), _CMP_EQ_OQ));
    r = _mm256_blendv_ps(r, x, _mm256_cmp_ps(x, SPL(INFINITY), _CMP_EQ_OQ));
    r = _mm256_blendv_ps(r, x, _mm256_cmp_ps(x, x, _CMP_UNORD_Q));
    return r;
}

/* ----- the VM (opcode numbering of compose_engine!, domain.rs:46-63) ----- */
enum { LVF = 0, LCF, LVB, LCB, LVI, LCI, LVV2, LCV2, LVV3, LCV3, LVM2, LCM2, LVM3, LCM3,
       ADDF, SUBF, MULF, DIVF, SINF, COSF, EXPF, SQRF, SQRTF, LNF,
       MKV2, MKV3, GXV2, GYV2, GXV3, GYV3, GZV3, ADDV2, SUBV2, SCV2, DOTV2, NRMV2,
       ADDV3, SUBV3, SCV3, DOTV3, NRMV3, CRSV3,
       MKM2, ADDM2, SUBM2, SCM2, MULM2, MULM2V2, DETM2, TRM2, TPM2, INVM2,
       MKM3, ADDM3, SUBM3, SCM3, MULM3, MULM3V3, DETM3, TRM3, TPM3, INVM3 };

typedef struct {
    v8 f[32]; v8 v2[32][2]; v8 v3[32][3]; v8 m2[32][4]; v8 m3[32][9];
    int sf, sv2, sv3, sm2, sm3;
} __attribute__((aligned(32))) vmst;

typedef struct { const uint32_t *code; uint32_t len; const uint8_t *kinds; uint32_t nk; const float *params; } sprog;
static const int kw[7] = {1, 0, 0, 2, 3, 4, 9};
static inline uint32_t fstart(const sprog *p, uint32_t c) { uint32_t s = 0; for (uint32_t i = 0; i < c; ++i) s += kw[p->kinds[i]]; return s; }

static inline v8 det3(const v8 *m) {
    return ADD(SUB(MUL(m[0], SUB(MUL(m[4], m[8]), MUL(m[5], m[7]))), MUL(m[3], SUB(MUL(m[1], m[8]), MUL(m[2], m[7])))),
               MUL(m[6], SUB(MUL(m[1], m[5]), MUL(m[2], m[4]))));
}

static v8 eval_batch(const sprog *p, const v8 *feat, vmst *s) {
    memset(s, 0, sizeof(*s)); /* VmState::new() zeroes every call (state.rs:46-47) */
    v8 t[9], *A, *B;
    for (uint32_t pc = 0; pc < p->len; ++pc) {
        uint32_t w = p->code[pc], op = w & 0xFF, a = (w >> 8) & 0xFFFF;
        switch (op) {
        case LVF: s->f[s->sf++] = feat[a]; break;
        case LCF: if (p->kinds[a] == 0) s->f[s->sf] = SPL(p->params[fstart(p, a)]); s->sf++; break;
        case LVV2: s->v2[s->sv2][0] = feat[a]; s->v2[s->sv2][1] = feat[a + 1]; s->sv2++; break;
        case LCV2: if (p->kinds[a] == 3) { uint32_t o = fstart(p, a); for (int i = 0; i < 2; ++i) s->v2[s->sv2][i] = SPL(p->params[o + i]); } s->sv2++; break;
        case LVV3: for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = feat[a + i]; s->sv3++; break;
        case LCV3: if (p->kinds[a] == 4) { uint32_t o = fstart(p, a); for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = SPL(p->params[o + i]); } s->sv3++; break;
        case LVM2: for (int i = 0; i < 4; ++i) s->m2[s->sm2][i] = feat[a + i]; s->sm2++; break;
        case LCM2: if (p->kinds[a] == 5) { uint32_t o = fstart(p, a); for (int i = 0; i < 4; ++i) s->m2[s->sm2][i] = SPL(p->params[o + i]); } s->sm2++; break;
        case LVM3: for (int i = 0; i < 9; ++i) s->m3[s->sm3][i] = feat[a + i]; s->sm3++; break;
        case LCM3: if (p->kinds[a] == 6) { uint32_t o = fstart(p, a); for (int i = 0; i < 9; ++i) s->m3[s->sm3][i] = SPL(p->params[o + i]); } s->sm3++; break;
        case ADDF: s->sf -= 2; s->f[s->sf] = ADD(s->f[s->sf], s->f[s->sf + 1]); s->sf++; break;
        case SUBF: s->sf -= 2; s->f[s->sf] = SUB(s->f[s->sf], s->f[s->sf + 1]); s->sf++; break;
        case MULF: s->sf -= 2; s->f[s->sf] = MUL(s->f[s->sf], s->f[s->sf + 1]); s->sf++; break;
        case DIVF: s->sf -= 2; s->f[s->sf] = DIV(s->f[s->sf], s->f[s->sf + 1]); s->sf++; break;
        case SINF: s->f[s->sf - 1] = v_sin(s->f[s->sf - 1]); break;
        case COSF: s->f[s->sf - 1] = v_cos(s->f[s->sf - 1]); break;
        case EXPF: s->f[s->sf - 1] = v_exp(s->f[s->sf - 1]); break;
        case SQRF: s->f[s->sf - 1] = MUL(s->f[s->sf - 1], s->f[s->sf - 1]); break;
        case SQRTF: s->f[s->sf - 1] = _mm256_sqrt_ps(s->f[s->sf - 1]); break;
        case LNF: s->f[s->sf - 1] = v_log(s->f[s->sf - 1]); break;
        case MKV2: s->sf -= 2; s->v2[s->sv2][0] = s->f[s->sf]; s->v2[s->sv2][1] = s->f[s->sf + 1]; s->sv2++; break;
        case MKV3: s->sf -= 3; for (int i = 0; i < 3; ++i) s->v3[s->sv3][i] = s->f[s->sf + i]; s->sv3++; break;
        case GXV2: s->sv2--; s->f[s->sf++] = s->v2[s->sv2][0]; break;
        case GYV2: s->sv2--; s->f[s->sf++] = s->v2[s->sv2][1]; break;
        case GXV3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][0]; break;
        case GYV3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][1]; break;
        case GZV3: s->sv3--; s->f[s->sf++] = s->v3[s->sv3][2]; break;
        case ADDV2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; A[0] = ADD(A[0], B[0]); A[1] = ADD(A[1], B[1]); s->sv2++; break;
        case SUBV2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; A[0] = SUB(A[0], B[0]); A[1] = SUB(A[1], B[1]); s->sv2++; break;
        case SCV2: { s->sf--; s->sv2--; v8 k = s->f[s->sf]; A = s->v2[s->sv2]; A[0] = MUL(A[0], k); A[1] = MUL(A[1], k); s->sv2++; break; }
        case DOTV2: s->sv2 -= 2; A = s->v2[s->sv2]; B = s->v2[s->sv2 + 1]; s->f[s->sf++] = ADD(MUL(A[0], B[0]), MUL(A[1], B[1])); break;
        case NRMV2: A = s->v2[s->sv2 - 1]; s->f[s->sf++] = _mm256_sqrt_ps(ADD(MUL(A[0], A[0]), MUL(A[1], A[1]))); s->sv2--; break;
        case ADDV3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = ADD(A[i], B[i]); s->sv3++; break;
        case SUBV3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; for (int i = 0; i < 3; ++i) A[i] = SUB(A[i], B[i]); s->sv3++; break;
        case SCV3: { s->sf--; s->sv3--; v8 k = s->f[s->sf]; A = s->v3[s->sv3]; for (int i = 0; i < 3; ++i) A[i] = MUL(A[i], k); s->sv3++; break; }
        case DOTV3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1]; s->f[s->sf++] = ADD(ADD(MUL(A[0], B[0]), MUL(A[1], B[1])), MUL(A[2], B[2])); break;
        case NRMV3: A = s->v3[s->sv3 - 1]; s->f[s->sf++] = _mm256_sqrt_ps(ADD(ADD(MUL(A[0], A[0]), MUL(A[1], A[1])), MUL(A[2], A[2]))); s->sv3--; break;
        case CRSV3: s->sv3 -= 2; A = s->v3[s->sv3]; B = s->v3[s->sv3 + 1];
            t[0] = SUB(MUL(A[1], B[2]), MUL(A[2], B[1])); t[1] = SUB(MUL(A[2], B[0]), MUL(A[0], B[2])); t[2] = SUB(MUL(A[0], B[1]), MUL(A[1], B[0]));
            A[0] = t[0]; A[1] = t[1]; A[2] = t[2]; s->sv3++; break;
        case MKM2: s->sv2 -= 2; A = s->m2[s->sm2]; A[0] = s->v2[s->sv2][0]; A[1] = s->v2[s->sv2][1]; A[2] = s->v2[s->sv2 + 1][0]; A[3] = s->v2[s->sv2 + 1][1]; s->sm2++; break;
        case ADDM2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = ADD(A[i], B[i]); s->sm2++; break;
        case SUBM2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1]; for (int i = 0; i < 4; ++i) A[i] = SUB(A[i], B[i]); s->sm2++; break;
        case SCM2: { s->sf--; s->sm2--; v8 k = s->f[s->sf]; A = s->m2[s->sm2]; for (int i = 0; i < 4; ++i) A[i] = MUL(A[i], k); s->sm2++; break; }
        case MULM2: s->sm2 -= 2; A = s->m2[s->sm2]; B = s->m2[s->sm2 + 1];
            t[0] = ADD(MUL(A[0], B[0]), MUL(A[2], B[1])); t[1] = ADD(MUL(A[1], B[0]), MUL(A[3], B[1]));
            t[2] = ADD(MUL(A[0], B[2]), MUL(A[2], B[3])); t[3] = ADD(MUL(A[1], B[2]), MUL(A[3], B[3]));
            for (int i = 0; i < 4; ++i) A[i] = t[i]; s->sm2++; break;
        case MULM2V2: s->sm2--; s->sv2--; A = s->m2[s->sm2]; B = s->v2[s->sv2];
            t[0] = ADD(MUL(A[0], B[0]), MUL(A[2], B[1])); t[1] = ADD(MUL(A[1], B[0]), MUL(A[3], B[1])); B[0] = t[0]; B[1] = t[1]; s->sv2++; break;
        case DETM2: s->sm2--; A = s->m2[s->sm2]; s->f[s->sf++] = SUB(MUL(A[0], A[3]), MUL(A[1], A[2])); break;
        case TRM2: s->sm2--; A = s->m2[s->sm2]; s->f[s->sf++] = ADD(A[0], A[3]); break;
        case TPM2: A = s->m2[s->sm2 - 1]; t[0] = A[1]; A[1] = A[2]; A[2] = t[0]; break;
        case INVM2: {
            A = s->m2[s->sm2 - 1];
            v8 det = SUB(MUL(A[0], A[3]), MUL(A[1], A[2]));
            v8 sing = _mm256_cmp_ps(_mm256_andnot_ps(SPL(-0.0f), det), SPL(1e-9f), _CMP_LT_OQ);
            v8 inv = DIV(SPL(1.0f), _mm256_blendv_ps(det, SPL(1.0f), sing));
            v8 neg = SPL(-0.0f);
            t[0] = _mm256_blendv_ps(MUL(A[3], inv), SPL(1.0f), sing);
            t[1] = _mm256_blendv_ps(MUL(_mm256_xor_ps(A[1], neg), inv), _mm256_setzero_ps(), sing);
            t[2] = _mm256_blendv_ps(MUL(_mm256_xor_ps(A[2], neg), inv), _mm256_setzero_ps(), sing);
            t[3] = _mm256_blendv_ps(MUL(A[0], inv), SPL(1.0f), sing);
            for (int i = 0; i < 4; ++i) A[i] = t[i];
            break; }
        case MKM3: s->sv3 -= 3; A = s->m3[s->sm3]; for (int c = 0; c < 3; ++c) for (int i = 0; i < 3; ++i) A[3 * c + i] = s->v3[s->sv3 + c][i]; s->sm3++; break;
        case ADDM3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = ADD(A[i], B[i]); s->sm3++; break;
        case SUBM3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1]; for (int i = 0; i < 9; ++i) A[i] = SUB(A[i], B[i]); s->sm3++; break;
        case SCM3: { s->sf--; s->sm3--; v8 k = s->f[s->sf]; A = s->m3[s->sm3]; for (int i = 0; i < 9; ++i) A[i] = MUL(A[i], k); s->sm3++; break; }
        case MULM3: s->sm3 -= 2; A = s->m3[s->sm3]; B = s->m3[s->sm3 + 1];
            for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) t[3 * c + r] = ADD(ADD(MUL(A[r], B[3 * c]), MUL(A[3 + r], B[3 * c + 1])), MUL(A[6 + r], B[3 * c + 2]));
            for (int i = 0; i < 9; ++i) A[i] = t[i]; s->sm3++; break;
        case MULM3V3: s->sm3--; s->sv3--; A = s->m3[s->sm3]; B = s->v3[s->sv3];
            for (int r = 0; r < 3; ++r) t[r] = ADD(ADD(MUL(A[r], B[0]), MUL(A[3 + r], B[1])), MUL(A[6 + r], B[2]));
            B[0] = t[0]; B[1] = t[1]; B[2] = t[2]; s->sv3++; break;
        case DETM3: s->sm3--; s->f[s->sf++] = det3(s->m3[s->sm3]); break;
        case TRM3: s->sm3--; A = s->m3[s->sm3]; s->f[s->sf++] = ADD(ADD(A[0], A[4]), A[8]); break;
        case TPM3: A = s->m3[s->sm3 - 1];
            t[0] = A[3]; t[1] = A[6]; t[2] = A[7]; A[3] = A[1]; A[6] = A[2]; A[7] = A[5]; A[1] = t[0]; A[2] = t[1]; A[5] = t[2]; break;
        case INVM3: {
            v8 *m = s->m3[s->sm3 - 1];
            v8 det = det3(m);
            v8 sing = _mm256_cmp_ps(_mm256_andnot_ps(SPL(-0.0f), det), SPL(1e-9f), _CMP_LT_OQ);
            v8 inv = DIV(SPL(1.0f), _mm256_blendv_ps(det, SPL(1.0f), sing));
            v8 neg = SPL(-0.0f);
            t[0] = MUL(SUB(MUL(m[4], m[8]), MUL(m[5], m[7])), inv);
            t[1] = MUL(_mm256_xor_ps(SUB(MUL(m[1], m[8]), MUL(m[2], m[7])), neg), inv);
            t[2] = MUL(SUB(MUL(m[1], m[5]), MUL(m[2], m[4])), inv);
            t[3] = MUL(_mm256_xor_ps(SUB(MUL(m[3], m[8]), MUL(m[5], m[6])), neg), inv);
            t[4] = MUL(SUB(MUL(m[0], m[8]), MUL(m[2], m[6])), inv);
            t[5] = MUL(_mm256_xor_ps(SUB(MUL(m[0], m[5]), MUL(m[2], m[3])), neg), inv);
            t[6] = MUL(SUB(MUL(m[3], m[7]), MUL(m[4], m[6])), inv);
            t[7] = MUL(_mm256_xor_ps(SUB(MUL(m[0], m[7]), MUL(m[1], m[6])), neg), inv);
            t[8] = MUL(SUB(MUL(m[0], m[4]), MUL(m[1], m[3])), inv);
            for (int i = 0; i < 9; ++i) m[i] = _mm256_blendv_ps(t[i], (i % 4 == 0) ? SPL(1.0f) : _mm256_setzero_ps(), sing);
            break; }
        default: break;
        }
    }
    return s->f[0];
}

static float hsum(v8 v) {
    float l[8];
    _mm256_storeu_ps(l, v);
    float a0 = l[0] + l[4], a1 = l[1] + l[5], a2 = l[2] + l[6], a3 = l[3] + l[7];
    return (a0 + a2) + (a1 + a3);
}

static float mse_one(const sprog *p, const float *ff, const float *tg, uint32_t nf, uint64_t nbatch, uint64_t nsamples,
                     vmst *st) {
    v8 sse = _mm256_setzero_ps();
    for (uint64_t b = 0; b < nbatch; ++b) {
        v8 pred = eval_batch(p, (const v8 *)(ff + b * nf * 8), st);
        v8 d = SUB(pred, _mm256_loadu_ps(tg + b * 8));
        sse = ADD(sse, MUL(d, d));
    }
    float mse = hsum(sse) / (float)nsamples;
    return isfinite(mse) ? mse : FLT_MAX;
}

typedef struct {
    const uint32_t *code; const uint64_t *code_off; const uint8_t *kinds; const uint64_t *kind_off;
    const float *params; const uint64_t *param_off; uint32_t n;
    const float *ff, *tg; uint32_t nf; uint64_t nbatch, nsamples; float *out;
    volatile uint32_t next; pthread_mutex_t mu;
} sjob;

static void *sworker(void *arg) {
    sjob *J = (sjob *)arg;
    vmst *st = (vmst *)aligned_alloc(64, (sizeof(vmst) + 63) & ~(size_t)63);
    for (;;) {
        pthread_mutex_lock(&J->mu);
        uint32_t i = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (i >= J->n) break;
        sprog p = {J->code + J->code_off[i], (uint32_t)(J->code_off[i + 1] - J->code_off[i]), J->kinds + J->kind_off[i],
                   (uint32_t)(J->kind_off[i + 1] - J->kind_off[i]), J->params + J->param_off[i]};
        J->out[i] = mse_one(&p, J->ff, J->tg, J->nf, J->nbatch, J->nsamples, st);
    }
    free(st);
    return NULL;
}

/* compute_mse over a packed population on `threads` host threads.
 * feature_flat must be 32-byte aligned (AoSoA f32x8 batches). */
ORC_API void simd_mse_batch(const uint32_t *code, const uint64_t *code_off, const uint8_t *kinds,
                            const uint64_t *kind_off, const float *params, const uint64_t *param_off, uint32_t n,
                            const float *feature_flat, const float *target, uint32_t nf, uint64_t nbatch,
                            uint64_t nsamples, int threads, float *out) {
    sjob J = {code, code_off, kinds, kind_off, params, param_off, n, feature_flat, target, nf, nbatch, nsamples, out, 0};
    pthread_mutex_init(&J.mu, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, sworker, &J);
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&J.mu);
}

/* Vectorised transcendentals exposed for the tests (bit-compare against the
 * scalar restatement). */
ORC_API void simd_transcendental(int which, const float *x, float *y, uint64_t n) {
    for (uint64_t i = 0; i + 8 <= n; i += 8) {
        v8 v = _mm256_loadu_ps(x + i), r;
        switch (which) { case 0: r = v_sin(v); break; case 1: r = v_cos(v); break; case 2: r = v_exp(v); break; default: r = v_log(v); }
        _mm256_storeu_ps(y + i, r);
    }
}
