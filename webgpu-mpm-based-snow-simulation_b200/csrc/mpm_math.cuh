// mpm_math.cuh -- device arithmetic of the MPM step.
//
// Every helper fixes one evaluation order so the f32 results, and therefore
// the i32 fixed-point grid, are reproducible bit for bit.  The kernels are
// compiled with -fmad=false (the compiler fuses nothing on its own), IEEE
// division and square root, and without flush-to-zero; every fused
// multiply-add below is an explicit __fmaf_rn.
//
// Canonical rules (WGSL leaves fusion and the rounding of division, exp and
// pow to the implementation; division is specified to 2.5 ulp):
//   mat3 is column-major, m[c*3 + r] = M[c][r]; constructors take columns
//   dot(a,b)     = fma(a.z, b.z, fma(a.y, b.y, a.x*b.x))
//   (M*v)[r]     = fma(M[2][r], v.z, fma(M[1][r], v.y, M[0][r]*v.x))
//   (A*B)[c][r]  = fma(A[2][r], B[c][2], fma(A[1][r], B[c][1], A[0][r]*B[c][0]))
//   cross(a,b).x = fma(a.y, b.z, -(a.z*b.y)), and cyclically
//   det(M)       = fma(M20, k2, fma(-M10, k1, M00*k0)),
//                  k0 = fma(M11,M22,-(M21*M12)), k1 = fma(M01,M22,-(M21*M02)), k2 = fma(M01,M12,-(M11*M02))
//   s += a*b in the transfer sums = fma(a, b, s)
//   x / d, d constant over a substep (dt, cell size, fixed-point scale,
//     force divisor) = x * RN(1/d), the reciprocal rounded once on the host
//   momentum / cell mass = momentum * RN(1/mass)
//   other divisions and sqrt are IEEE
//   i32(f): truncation toward zero, saturating, NaN -> 0
//   exp: f64 evaluation by exp64 below, rounded once to f32
//   pow: f64 evaluation by the table-driven log_t64/exp_t64 below, rounded
//     once to f32
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

struct M3 { float m[9]; };

// cvt.rzi.s32.f32 truncates toward zero, saturates out-of-range values and
// converts NaN to 0 (checked on the device by mpm_selftest).
__device__ __forceinline__ int32_t f2i(float x) { return __float2int_rz(x); }
__device__ __forceinline__ float i2f(int32_t i) { return __int2float_rn(i); }

// xxHash32-style 3-word mix (randomNumberGenerators.wgsl:24-38).
__host__ __device__ __forceinline__ uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t p2 = 2246822519u, p3 = 3266489917u, p4 = 668265263u, p5 = 374761393u;
    uint32_t h = z + p5 + x * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h += y * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h = p2 * (h ^ (h >> 15));
    h = p3 * (h ^ (h >> 13));
    return h ^ (h >> 16);
}

// 1- and 4-word variants of the same mix (randomNumberGenerators.wgsl:3-9, 40-55)
__host__ __device__ __forceinline__ uint32_t hash1(uint32_t n) {
    uint32_t h = n + 374761393u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h = 2246822519u * (h ^ (h >> 15));
    h = 3266489917u * (h ^ (h >> 13));
    return h ^ (h >> 16);
}
__host__ __device__ __forceinline__ uint32_t hash4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    const uint32_t p2 = 2246822519u, p3 = 3266489917u, p4 = 668265263u, p5 = 374761393u;
    uint32_t h = w + p5 + x * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h += y * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h += z * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h = p2 * (h ^ (h >> 15));
    h = p3 * (h ^ (h >> 13));
    return h ^ (h >> 16);
}

// exp(x) in f64: Cody-Waite reduction x = k ln2 + r, then the degree-13
// Taylor polynomial of e^r (Horner, one fused multiply-add per step), then
// exact scaling by 2^k.
__device__ __forceinline__ double pow2i(int k) {
    return __longlong_as_double((long long)(k + 1023) << 52);
}
static __device__ __forceinline__ double exp64(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000ll);
    if (x < -745.2) return 0.0;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    const double INV_LN2 = 1.44269504088896338700e+00;
    double kf = floor(__dadd_rn(__dmul_rn(x, INV_LN2), 0.5));
    int k = (int)kf;
    double r = __dsub_rn(__dsub_rn(x, __dmul_rn(kf, LN2_HI)), __dmul_rn(kf, LN2_LO));
    double p = 1.0 / 6227020800.0;
    p = __fma_rn(p, r, 1.0 / 479001600.0);
    p = __fma_rn(p, r, 1.0 / 39916800.0);
    p = __fma_rn(p, r, 1.0 / 3628800.0);
    p = __fma_rn(p, r, 1.0 / 362880.0);
    p = __fma_rn(p, r, 1.0 / 40320.0);
    p = __fma_rn(p, r, 1.0 / 5040.0);
    p = __fma_rn(p, r, 1.0 / 720.0);
    p = __fma_rn(p, r, 1.0 / 120.0);
    p = __fma_rn(p, r, 1.0 / 24.0);
    p = __fma_rn(p, r, 1.0 / 6.0);
    p = __fma_rn(p, r, 0.5);
    p = __fma_rn(p, r, 1.0);
    p = __fma_rn(p, r, 1.0);
    int k1 = k / 2, k2 = k - k1;
    return __dmul_rn(__dmul_rn(p, pow2i(k1)), pow2i(k2));
}

__device__ __forceinline__ float expf_m(float x) { return __double2float_rn(exp64((double)x)); }
// Tables of log_t64 / exp_t64 (written by gen_pow_tables.py): reciprocals
// of the 128 slice centres of [1, 2) and minus their logs, and 2^(i/64).
// Read through the read-only data path (lanes index them divergently).
#define MPM_POW_TABLE static __device__ const
#include "mpm_pow_tables.h"
#undef MPM_POW_TABLE

// log(x) in f64 for an f32 x > 0 (NaN for x < 0 or NaN, +inf for +inf):
// x = m 2^e from the f32 fields (subnormals scaled by 2^24 first), j = the
// top 7 mantissa bits, r = m * INVC[j] - 1 (one fused multiply-add, |r| <
// 2^-7.9), log x = e ln2 + NLOGC[j] + log1p(r), log1p by its Taylor series
// to r^7 (truncation < 2^-66).
static __device__ __forceinline__ double log_t64(float x) {
    if (!(x > 0.0f)) return __longlong_as_double(0x7ff8000000000000ll);
    uint32_t u = __float_as_uint(x);
    if (u == 0x7f800000u) return (double)x;
    int e = -127;
    if ((u >> 23) == 0) {
        u = __float_as_uint(__fmul_rn(x, 0x1p24f));
        e -= 24;
    }
    e += (int)(u >> 23);
    const int j = (int)((u >> 16) & 127u);
    const double m = (double)__uint_as_float((u & 0x7fffffu) | 0x3f800000u);
    const double r = __fma_rn(m, __ldg(&POW_INVC[j]), -1.0);
    double q = __fma_rn(1.0 / 7.0, r, -1.0 / 6.0);
    q = __fma_rn(q, r, 1.0 / 5.0);
    q = __fma_rn(q, r, -0.25);
    q = __fma_rn(q, r, 1.0 / 3.0);
    q = __fma_rn(q, r, -0.5);
    const double l1 = __fma_rn(q, __dmul_rn(r, r), r);
    const double LN2 = 6.93147180559945309417e-01;
    return __fma_rn((double)e, LN2, __dadd_rn(__ldg(&POW_NLOGC[j]), l1));
}

// exp(z) in f64 where only its f32 rounding is used: +inf above 89 and 0
// below -104 (both round to the same f32 as the exact value); otherwise
// z = k ln2/64 + r (Cody-Waite, k = RN(64 z / ln2), |r| <= ln2/128), e^r by
// its Taylor series to r^7 (truncation < 2^-73), times EXP2[k mod 64] and
// the exact power 2^floor(k/64).
static __device__ __forceinline__ double exp_t64(double z) {
    if (z != z) return z;
    if (z > 89.0) return __longlong_as_double(0x7ff0000000000000ll);
    if (z < -104.0) return 0.0;
    const double K = 0x1.71547652b82fep+6;   // 64 / ln2
    const double L_HI = 6.93147180369123816490e-01 / 64.0, L_LO = 1.90821492927058770002e-10 / 64.0;
    const double kf = rint(__dmul_rn(z, K));
    const int k = (int)kf;
    const double r = __dsub_rn(__dsub_rn(z, __dmul_rn(kf, L_HI)), __dmul_rn(kf, L_LO));
    double p = __fma_rn(1.0 / 5040.0, r, 1.0 / 720.0);
    p = __fma_rn(p, r, 1.0 / 120.0);
    p = __fma_rn(p, r, 1.0 / 24.0);
    p = __fma_rn(p, r, 1.0 / 6.0);
    p = __fma_rn(p, r, 0.5);
    p = __fma_rn(p, r, 1.0);
    p = __fma_rn(p, r, 1.0);
    return __dmul_rn(__dmul_rn(p, __ldg(&POW_EXP2[k & 63])), pow2i(k >> 6));
}

// pow(x, y) = exp(y log x) in f64, rounded once to f32; pow(0, y) = +inf,
// 1 or 0 for y < 0, y == 0, y > 0.
__device__ __forceinline__ float powf_m(float x, float y) {
    if (x == 0.0f) return y < 0.0f ? __int_as_float(0x7f800000) : (y == 0.0f ? 1.0f : 0.0f);
    return __double2float_rn(exp_t64(__dmul_rn((double)y, log_t64(x))));
}

// ---- scalar f32 ops with explicit rounding (no contraction) ----------
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ float ff(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Paired f32 operations (one FFMA2 / FMUL2 / FADD2 instruction on sm_100 for
// two lanes); each component rounds exactly as the scalar op above.
__device__ __forceinline__ float2 ff2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fm2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fa2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

__device__ __forceinline__ float dot3(const float* a, const float* b) {
    return ff(a[2], b[2], ff(a[1], b[1], fm(a[0], b[0])));
}
__device__ __forceinline__ void cross3(const float* a, const float* b, float* o) {
    float x = ff(a[1], b[2], -fm(a[2], b[1]));
    float y = ff(a[2], b[0], -fm(a[0], b[2]));
    float z = ff(a[0], b[1], -fm(a[1], b[0]));
    o[0] = x; o[1] = y; o[2] = z;
}
__device__ __forceinline__ float len3(const float* a) { return __fsqrt_rn(dot3(a, a)); }

__device__ __forceinline__ float det3(const float* m) {
    float k0 = ff(m[4], m[8], -fm(m[7], m[5]));
    float k1 = ff(m[1], m[8], -fm(m[7], m[2]));
    float k2 = ff(m[1], m[5], -fm(m[4], m[2]));
    return ff(m[6], k2, ff(-m[3], k1, fm(m[0], k0)));
}

// mat3x3Inverse (matrixOps.wgsl:8-27): adjugate * (1/det); identity if det == 0.
// The cofactors are formed in pairs (FFMA2/FMUL2); cofactors 0 and 2 equal
// the determinant's k0 and k2 (the same products), so det3's value is
// reproduced from them.
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ void inv3(const float* m, float* o) {
    const float2 a01 = ff2(make_float2(m[4], m[2]), make_float2(m[8], m[7]),
                           neg2(fm2(make_float2(m[5], m[1]), make_float2(m[7], m[8]))));
    const float2 a23 = ff2(make_float2(m[1], m[5]), make_float2(m[5], m[6]),
                           neg2(fm2(make_float2(m[2], m[3]), make_float2(m[4], m[8]))));
    const float k1 = ff(m[1], m[8], -fm(m[7], m[2]));
    const float det = ff(m[6], a23.x, ff(-m[3], k1, fm(m[0], a01.x)));
    if (det == 0.0f) {
        o[0] = 1.f; o[1] = 0.f; o[2] = 0.f; o[3] = 0.f; o[4] = 1.f; o[5] = 0.f; o[6] = 0.f; o[7] = 0.f; o[8] = 1.f;
        return;
    }
    const float2 a45 = ff2(make_float2(m[0], m[2]), make_float2(m[8], m[3]),
                           neg2(fm2(make_float2(m[2], m[0]), make_float2(m[6], m[5]))));
    const float2 a67 = ff2(make_float2(m[3], m[1]), make_float2(m[7], m[6]),
                           neg2(fm2(make_float2(m[4], m[0]), make_float2(m[6], m[7]))));
    const float a8 = ff(m[0], m[4], -fm(m[1], m[3]));
    const float s = __frcp_rn(det);   // RN(1/det), the IEEE quotient 1/det
    const float2 s2 = dup2(s);
    const float2 o01 = fm2(a01, s2), o23 = fm2(a23, s2), o45 = fm2(a45, s2), o67 = fm2(a67, s2);
    o[0] = o01.x; o[1] = o01.y; o[2] = o23.x; o[3] = o23.y;
    o[4] = o45.x; o[5] = o45.y; o[6] = o67.x; o[7] = o67.y;
    o[8] = fm(a8, s);
}

__device__ __forceinline__ void tr3(const float* m, float* o) {
    float t[9] = {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]};
#pragma unroll
    for (int i = 0; i < 9; i++) o[i] = t[i];
}

// A * B, column-major: column c, row r = A[6+r] B[3c+2] + (A[3+r] B[3c+1] + A[r] B[3c])
// with rows 0 and 1 of each column in paired form
__device__ __forceinline__ void mul3(const float* A, const float* B, float* o) {
    float t[9];
    const float2 A01 = make_float2(A[0], A[1]), A34 = make_float2(A[3], A[4]), A67 = make_float2(A[6], A[7]);
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float2 t01 = ff2(A67, dup2(B[c * 3 + 2]), ff2(A34, dup2(B[c * 3 + 1]), fm2(A01, dup2(B[c * 3 + 0]))));
        t[c * 3 + 0] = t01.x;
        t[c * 3 + 1] = t01.y;
        t[c * 3 + 2] = ff(A[8], B[c * 3 + 2], ff(A[5], B[c * 3 + 1], fm(A[2], B[c * 3 + 0])));
    }
#pragma unroll
    for (int i = 0; i < 9; i++) o[i] = t[i];
}

__device__ __forceinline__ void mv3(const float* M, const float* v, float* o) {
    float t0 = ff(M[6], v[2], ff(M[3], v[1], fm(M[0], v[0])));
    float t1 = ff(M[7], v[2], ff(M[4], v[1], fm(M[1], v[0])));
    float t2 = ff(M[8], v[2], ff(M[5], v[1], fm(M[2], v[0])));
    o[0] = t0; o[1] = t1; o[2] = t2;
}

// calculatePolarDecompositionRotation (matrixOps.wgsl:33-45): 4 averaging
// steps R <- 0.5 (R + R^-T).
__device__ __forceinline__ void polar3(const float* F, float* R) {
    float g[9];
#pragma unroll
    for (int i = 0; i < 9; i++) g[i] = F[i];
#pragma unroll 1
    for (int it = 0; it < 4; it++) {
        float iv[9];
        inv3(g, iv);
        // g <- 0.5 (g + transpose(iv)), transpose(iv)[c*3+r] = iv[r*3+c], in pairs
        const float t[9] = {iv[0], iv[3], iv[6], iv[1], iv[4], iv[7], iv[2], iv[5], iv[8]};
        const float2 h = dup2(0.5f);
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
            const float2 v = fm2(h, fa2(make_float2(g[i], g[i + 1]), make_float2(t[i], t[i + 1])));
            g[i] = v.x;
            g[i + 1] = v.y;
        }
        g[8] = fm(0.5f, fa(g[8], t[8]));
    }
#pragma unroll
    for (int i = 0; i < 9; i++) R[i] = g[i];
}

// mat4 (column-major) * vec4(v, 1), .xyz
__device__ __forceinline__ void xform_point(const float* M, const float* v, float* o) {
    float t[3];
#pragma unroll
    for (int r = 0; r < 3; r++)
        t[r] = fa(ff(M[8 + r], v[2], ff(M[4 + r], v[1], fm(M[r], v[0]))), M[12 + r]);
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}

}  // namespace mpm
