// vm_ops.cuh -- the reference's op kernels as device functions over P data
// points per thread.
//
// Every function follows the operation order of the reference
// (src/domains/basic/eval.rs:4-63, src/domains/linalg/eval.rs:4-506) with
// IEEE round-to-nearest single-precision add/sub/mul/div/sqrt and no
// contraction: this file must be compiled with -fmad=false (the build does),
// so that a*b + c stays a rounded multiply followed by a rounded add, as in
// the reference.  Results are then bit-identical to the reference for every
// op except the transcendentals.
//
// sin/cos/exp/ln: the reference gets them from the `wide` 1.1.1 crate.  They
// are restated here from the published Cephes single-precision method
// (S. L. Moshier, Cephes Math Library: sinf/cosf/expf/logf) -- Cody-Waite
// range reduction followed by the Cephes minimax polynomials, Horner order.
// Measured error against double-precision libm: below 1.5 ulp.
#pragma once
#include <stdint.h>

namespace rsr {

// ---------------------------------------------------- scalar transcendentals
__device__ __forceinline__ float pow2i(int k) { return __int_as_float((k + 127) << 23); }

struct SinCos { float s, c; };

// Reduction by pi/2 (three-part constant), quadrant from the rounded
// multiple q.  Returns sin and cos of |x|'s reduced argument mapped back.
__device__ __forceinline__ SinCos cephes_sincos(float x) {
    const float xa = fabsf(x);
    const float yq = rintf(xa * 0.636619772367581343f);
    const int q = (int)fminf(yq, 16777216.0f);
    const float r = ((xa - yq * 1.5703125f) - yq * 4.837512969970703125e-4f) - yq * 7.54978995489188216e-8f;
    const float r2 = r * r;
    const float s = ((-1.9515295891e-4f * r2 + 8.3321608736e-3f) * r2 - 1.6666654611e-1f) * (r2 * r) + r;
    const float c = ((2.443315711809948e-5f * r2 - 1.388731625493765e-3f) * r2 + 4.166664568298827e-2f) * (r2 * r2)
                    + (1.0f - 0.5f * r2);
    float sv = (q & 1) ? c : s;
    float cv = (q & 1) ? s : c;
    if (q & 2) sv = -sv;
    if ((q + 1) & 2) cv = -cv;
    if (x < 0.0f) sv = -sv;
    const bool big = yq > 16777216.0f;
    sv = big ? 0.0f : sv;
    cv = big ? 1.0f : cv;
    const bool bad = !(xa <= 3.402823466e38f);  // inf or nan
    sv = bad ? __int_as_float(0x7fc00000) : sv;
    cv = bad ? __int_as_float(0x7fc00000) : cv;
    return {sv, cv};
}
__device__ __forceinline__ float cephes_sin(float x) { return cephes_sincos(x).s; }
__device__ __forceinline__ float cephes_cos(float x) { return cephes_sincos(x).c; }

__device__ __forceinline__ float cephes_exp(float x) {
    const float z = floorf(1.44269504088896341f * x + 0.5f);
    const float r = (x - z * 0.693359375f) - z * -2.12194440e-4f;
    const int n = (int)fmaxf(fminf(z, 200.0f), -200.0f);
    const float rr = r * r;
    const float p = ((((1.9875691500e-4f * r + 1.3981999507e-3f) * r + 8.3334519073e-3f) * r + 4.1665795894e-2f) * r
                     + 1.6666665459e-1f) * r + 5.0000001201e-1f;
    const float y = (p * rr + r) + 1.0f;
    const int n1 = max(min(n >> 1, 127), -126), n2 = max(min(n - (n >> 1), 127), -126);
    float res = (y * pow2i(n1)) * pow2i(n2);
    res = x > 88.72283905206835f ? __int_as_float(0x7f800000) : res;
    res = x < -103.278929903431851103f ? 0.0f : res;
    res = (x != x) ? x : res;
    return res;
}

__device__ __forceinline__ float cephes_log(float x) {
    uint32_t bits = __float_as_uint(x);
    const bool sub = ((bits >> 23) & 0xFFu) == 0u;
    bits = sub ? __float_as_uint(x * 33554432.0f) : bits;
    int e = (int)((bits >> 23) & 0xFFu) - 126 - (sub ? 25 : 0);
    float m = __uint_as_float((bits & 0x807FFFFFu) | (126u << 23));
    const bool lo = m < 0.707106781186547524f;
    e = lo ? e - 1 : e;
    m = lo ? (m + m) - 1.0f : m - 1.0f;
    const float z = m * m;
    float y = ((((((((7.0376836292e-2f * m - 1.1514610310e-1f) * m + 1.1676998740e-1f) * m - 1.2420140846e-1f) * m
                   + 1.4249322787e-1f) * m - 1.6668057665e-1f) * m + 2.0000714765e-1f) * m - 2.4999993993e-1f) * m
               + 3.3333331174e-1f) * m * z;
    const float fe = (float)e;
    y = y + -2.12194440e-4f * fe;
    y = y + -0.5f * z;
    float res = (m + y) + 0.693359375f * fe;
    res = x < 0.0f ? __int_as_float(0x7fc00000) : res;
    res = x == 0.0f ? __int_as_float(0xff800000) : res;
    res = x == __int_as_float(0x7f800000) ? x : res;
    res = (x != x) ? x : res;
    return res;
}

// ------------------------------------------------------- P-point values
template <int P>
struct __align__(P * 4 <= 16 ? P * 4 : 16) Vf {
    float v[P];
};

#define RSR_LOOP _Pragma("unroll") for (int k = 0; k < P; ++k)

template <int P> __device__ __forceinline__ Vf<P> splat(float x) { Vf<P> r; RSR_LOOP r.v[k] = x; return r; }
template <int P> __device__ __forceinline__ Vf<P> operator+(const Vf<P> &a, const Vf<P> &b) { Vf<P> r; RSR_LOOP r.v[k] = a.v[k] + b.v[k]; return r; }
template <int P> __device__ __forceinline__ Vf<P> operator-(const Vf<P> &a, const Vf<P> &b) { Vf<P> r; RSR_LOOP r.v[k] = a.v[k] - b.v[k]; return r; }
template <int P> __device__ __forceinline__ Vf<P> operator*(const Vf<P> &a, const Vf<P> &b) { Vf<P> r; RSR_LOOP r.v[k] = a.v[k] * b.v[k]; return r; }
template <int P> __device__ __forceinline__ Vf<P> operator/(const Vf<P> &a, const Vf<P> &b) { Vf<P> r; RSR_LOOP r.v[k] = a.v[k] / b.v[k]; return r; }
template <int P> __device__ __forceinline__ Vf<P> operator-(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = -a.v[k]; return r; }
template <int P> __device__ __forceinline__ Vf<P> vsqrt(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = sqrtf(a.v[k]); return r; }
template <int P> __device__ __forceinline__ Vf<P> vsin(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = cephes_sin(a.v[k]); return r; }
template <int P> __device__ __forceinline__ Vf<P> vcos(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = cephes_cos(a.v[k]); return r; }
template <int P> __device__ __forceinline__ Vf<P> vexp(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = cephes_exp(a.v[k]); return r; }
template <int P> __device__ __forceinline__ Vf<P> vlog(const Vf<P> &a) { Vf<P> r; RSR_LOOP r.v[k] = cephes_log(a.v[k]); return r; }

// ---------------------------------------------------------- linalg ops
// Arrays are component-major: a[c] is component c (Mat: column-major).
// Outputs may alias inputs: results are formed in temporaries first.
template <int P> __device__ __forceinline__ Vf<P> dot2(const Vf<P> *a, const Vf<P> *b) {
    return (a[0] * b[0]) + (a[1] * b[1]);                                   // linalg/eval.rs:129
}
template <int P> __device__ __forceinline__ Vf<P> dot3(const Vf<P> *a, const Vf<P> *b) {
    return ((a[0] * b[0]) + (a[1] * b[1])) + (a[2] * b[2]);                 // linalg/eval.rs:186
}
template <int P> __device__ __forceinline__ Vf<P> norm2(const Vf<P> *a) {
    return vsqrt((a[0] * a[0]) + (a[1] * a[1]));                           // linalg/eval.rs:141
}
template <int P> __device__ __forceinline__ Vf<P> norm3(const Vf<P> *a) {
    return vsqrt(((a[0] * a[0]) + (a[1] * a[1])) + (a[2] * a[2]));         // linalg/eval.rs:198
}
template <int P> __device__ __forceinline__ void cross3(const Vf<P> *a, const Vf<P> *b, Vf<P> *o) {
    Vf<P> t0 = a[1] * b[2] - a[2] * b[1];                                   // linalg/eval.rs:207-211
    Vf<P> t1 = a[2] * b[0] - a[0] * b[2];
    Vf<P> t2 = a[0] * b[1] - a[1] * b[0];
    o[0] = t0; o[1] = t1; o[2] = t2;
}
template <int P> __device__ __forceinline__ void mul_m2(const Vf<P> *a, const Vf<P> *b, Vf<P> *o) {
    Vf<P> t0 = a[0] * b[0] + a[2] * b[1], t1 = a[1] * b[0] + a[3] * b[1];  // linalg/eval.rs:263-268
    Vf<P> t2 = a[0] * b[2] + a[2] * b[3], t3 = a[1] * b[2] + a[3] * b[3];
    o[0] = t0; o[1] = t1; o[2] = t2; o[3] = t3;
}
template <int P> __device__ __forceinline__ void mul_m2v2(const Vf<P> *m, const Vf<P> *v, Vf<P> *o) {
    Vf<P> t0 = m[0] * v[0] + m[2] * v[1], t1 = m[1] * v[0] + m[3] * v[1];  // linalg/eval.rs:282
    o[0] = t0; o[1] = t1;
}
template <int P> __device__ __forceinline__ Vf<P> det_m2(const Vf<P> *m) {
    return (m[0] * m[3]) - (m[1] * m[2]);                                   // linalg/eval.rs:294
}
template <int P> __device__ __forceinline__ Vf<P> trace_m2(const Vf<P> *m) { return m[0] + m[3]; }
template <int P> __device__ __forceinline__ void transpose_m2(const Vf<P> *m, Vf<P> *o) {
    Vf<P> a = m[1], b = m[2];
    o[0] = m[0]; o[1] = b; o[2] = a; o[3] = m[3];
}
template <int P> __device__ __forceinline__ void inverse_m2(const Vf<P> *m, Vf<P> *o) {
    Vf<P> det = det_m2(m), r0, r1, r2, r3;                                  // linalg/eval.rs:316-329
    RSR_LOOP {
        const bool sing = fabsf(det.v[k]) < 1e-9f;
        const float inv = 1.0f / (sing ? 1.0f : det.v[k]);
        r0.v[k] = sing ? 1.0f : m[3].v[k] * inv;
        r1.v[k] = sing ? 0.0f : (-m[1].v[k]) * inv;
        r2.v[k] = sing ? 0.0f : (-m[2].v[k]) * inv;
        r3.v[k] = sing ? 1.0f : m[0].v[k] * inv;
    }
    o[0] = r0; o[1] = r1; o[2] = r2; o[3] = r3;
}
template <int P> __device__ __forceinline__ void mul_m3(const Vf<P> *a, const Vf<P> *b, Vf<P> *o) {
    Vf<P> t[9];                                                             // linalg/eval.rs:412-422
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) t[3 * c + r] = (a[r] * b[3 * c] + a[3 + r] * b[3 * c + 1]) + a[6 + r] * b[3 * c + 2];
#pragma unroll
    for (int i = 0; i < 9; ++i) o[i] = t[i];
}
template <int P> __device__ __forceinline__ void mul_m3v3(const Vf<P> *m, const Vf<P> *v, Vf<P> *o) {
    Vf<P> t[3];                                                             // linalg/eval.rs:436-440
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r] = (m[r] * v[0] + m[3 + r] * v[1]) + m[6 + r] * v[2];
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}
template <int P> __device__ __forceinline__ Vf<P> det_m3(const Vf<P> *m) {
    return (m[0] * (m[4] * m[8] - m[5] * m[7]) - m[3] * (m[1] * m[8] - m[2] * m[7]))   // linalg/eval.rs:470-472
           + m[6] * (m[1] * m[5] - m[2] * m[4]);
}
template <int P> __device__ __forceinline__ Vf<P> trace_m3(const Vf<P> *m) { return (m[0] + m[4]) + m[8]; }
template <int P> __device__ __forceinline__ void transpose_m3(const Vf<P> *m, Vf<P> *o) {
    Vf<P> t[9] = {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]};   // linalg/eval.rs:459
#pragma unroll
    for (int i = 0; i < 9; ++i) o[i] = t[i];
}
template <int P> __device__ __forceinline__ void inverse_m3(const Vf<P> *m, Vf<P> *o) {
    Vf<P> det = det_m3(m);                                                  // linalg/eval.rs:476-506
    Vf<P> c[9] = {m[4] * m[8] - m[5] * m[7], m[1] * m[8] - m[2] * m[7], m[1] * m[5] - m[2] * m[4],
                  m[3] * m[8] - m[5] * m[6], m[0] * m[8] - m[2] * m[6], m[0] * m[5] - m[2] * m[3],
                  m[3] * m[7] - m[4] * m[6], m[0] * m[7] - m[1] * m[6], m[0] * m[4] - m[1] * m[3]};
    RSR_LOOP {
        const bool sing = fabsf(det.v[k]) < 1e-9f;
        const float inv = 1.0f / (sing ? 1.0f : det.v[k]);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            const float adj = ((i & 1) ? -c[i].v[k] : c[i].v[k]) * inv;
            c[i].v[k] = sing ? ((i % 4 == 0) ? 1.0f : 0.0f) : adj;
        }
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) o[i] = c[i];
}

}  // namespace rsr
