/*
 * mpm_oracle.c -- TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference
 * MPM step; see mpm_oracle.h for the scope and the parity status (UNPINNED).
 *
 * Compiled twice: -DOR_FP64=0 gives the orf_* (f32, fixed-point grid) symbols,
 * -DOR_FP64=1 the ord_* (f64) symbols.  Build with -ffp-contract=off (every
 * fused multiply-add is written out as fmaf) and without -ffast-math: the f32
 * instantiation defines, operation by operation, the canonical evaluation
 * order the CUDA path must reproduce bit for bit.
 *
 * Canonical evaluation rules.  WGSL leaves operation fusion and the exact
 * rounding of division, exp and pow to the implementation (division is
 * specified to 2.5 ulp); the oracle fixes one choice within those bounds:
 *   fma(a,b,c) = a*b+c rounded once (C fmaf); M[c][r] is column-major
 *   dot(a,b)     = fma(a.z, b.z, fma(a.y, b.y, a.x*b.x))
 *   (M*v)[r]     = fma(M[2][r], v.z, fma(M[1][r], v.y, M[0][r]*v.x))
 *   (A*B)[c][r]  = fma(A[2][r], B[c][2], fma(A[1][r], B[c][1], A[0][r]*B[c][0]))
 *   cross(a,b).x = fma(a.y, b.z, -(a.z*b.y)), and cyclically
 *   det(M)       = fma(M20, k2, fma(-M10, k1, M00*k0)), k0 = fma(M11, M22, -(M21*M12)),
 *                  k1 = fma(M01, M22, -(M21*M02)), k2 = fma(M01, M12, -(M11*M02))
 *   s += a*b     = fma(a, b, s) in the transfer sums (velocity, B, velocity gradient)
 *   x / d for d constant over the substep (dt, cell size, fixed-point scale,
 *                  force divisor) = x * RN(1/d), error <= 1.5 ulp
 *   momentum / cell mass = momentum * RN(1/mass)
 *   every other division, and sqrt, are IEEE; length(v) = sqrt(dot(v,v))
 *   i32(f) = truncation toward zero, saturating, NaN -> 0
 *   exp evaluated in f64 by or_exp64 below, rounded once to f32
 *   pow evaluated in f64 by the table-driven or_log_t64/or_exp_t64 below,
 *                  rounded once to f32
 * Every other expression follows the WGSL source's own left-to-right order;
 * the f64 instantiation uses the same formulas with IEEE f64 division.
 */
#include "mpm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef OR_FP64
#define OR_FP64 0
#endif

#if OR_FP64
typedef double real;
typedef OrParticleD PART;
#define PFX(n) ord_##n
#else
typedef float real;
typedef OrParticle PART;
#define PFX(n) orf_##n
#endif

/* ------------------------------------------------------------------ */
/* shared scalar helpers (emitted once, by the f32 instantiation)       */
/* ------------------------------------------------------------------ */
uint32_t or_hash3(uint32_t x, uint32_t y, uint32_t z);
double or_exp64(double x);

#if !OR_FP64
/* xxHash32-style 3-word mix (randomNumberGenerators.wgsl:24-38). */
uint32_t or_hash3(uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t p2 = 2246822519u, p3 = 3266489917u, p4 = 668265263u, p5 = 374761393u;
    uint32_t h = z + p5 + x * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h += y * p3;
    h = p4 * ((h << 17) | (h >> 15));
    h = p2 * (h ^ (h >> 15));
    h = p3 * (h ^ (h >> 13));
    return h ^ (h >> 16);
}

static inline uint64_t d2u(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
static inline double u2d(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }

/* 2^k for integer k in [-1022, 1023], built from the bit pattern. */
static inline double pow2i(int k) { return u2d((uint64_t)(k + 1023) << 52); }

/* exp(x) in f64: Cody-Waite reduction x = k*ln2 + r, |r| <= ln2/2, then the
 * Taylor series of e^r to degree 13 by Horner with fused multiply-adds
 * (truncation error < 1e-17 relative), then scaling by 2^k in two exact steps. */
double or_exp64(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.2) return 0.0;
    const double LN2_HI = 6.93147180369123816490e-01; /* 0x3FE62E42FEE00000 */
    const double LN2_LO = 1.90821492927058770002e-10; /* ln2 - LN2_HI */
    const double INV_LN2 = 1.44269504088896338700e+00;
    double kf = floor(x * INV_LN2 + 0.5);
    int k = (int)kf;
    double r = (x - kf * LN2_HI) - kf * LN2_LO;
    double p = 1.0 / 6227020800.0;               /* 1/13! */
    p = fma(p, r, 1.0 / 479001600.0);               /* 1/12! */
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int k1 = k / 2, k2 = k - k1;
    return (p * pow2i(k1)) * pow2i(k2);
}

float or_expf(float x) { return (float)or_exp64((double)x); }

/* The pow tables: the CUDA path reads the same generated file
 * (webgpu-mpm-based-snow-simulation_b200/csrc/gen_pow_tables.py), so both
 * sides hold identical constants: POW_INVC[j] = RN(1/c_j) for the slice
 * centres c_j = 1 + (j + 1/2)/128 of [1, 2), POW_NLOGC[j] = RN(-log
 * POW_INVC[j]), POW_EXP2[i] = RN(2^(i/64)). */
#define MPM_POW_TABLE static const
#include "../webgpu-mpm-based-snow-simulation_b200/csrc/mpm_pow_tables.h"
#undef MPM_POW_TABLE

static inline uint32_t f2u(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
static inline float u2f(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }

/* log(x) in f64 for an f32 x > 0 (NaN for x < 0 or NaN, +inf for +inf):
 * x = m * 2^e from the f32 fields (subnormals scaled by 2^24 first), j = the
 * top 7 mantissa bits, r = m * POW_INVC[j] - 1 by one fma (|r| < 2^-7.9),
 * log x = e*ln2 + POW_NLOGC[j] + log1p(r), log1p by its Taylor series to r^7
 * (truncation < 2^-66). */
static double or_log_t64(float x) {
    if (!(x > 0.0f)) return NAN;
    uint32_t u = f2u(x);
    if (u == 0x7f800000u) return (double)x;
    int e = -127;
    if ((u >> 23) == 0) {
        u = f2u(x * 0x1p24f);
        e -= 24;
    }
    e += (int)(u >> 23);
    const int j = (int)((u >> 16) & 127u);
    const double m = (double)u2f((u & 0x7fffffu) | 0x3f800000u);
    const double r = fma(m, POW_INVC[j], -1.0);
    double q = fma(1.0 / 7.0, r, -1.0 / 6.0);
    q = fma(q, r, 1.0 / 5.0);
    q = fma(q, r, -0.25);
    q = fma(q, r, 1.0 / 3.0);
    q = fma(q, r, -0.5);
    const double l1 = fma(q, r * r, r);
    const double LN2 = 6.93147180559945309417e-01;
    return fma((double)e, LN2, POW_NLOGC[j] + l1);
}

/* exp(z) in f64 where only its f32 rounding is used: +inf above 89 and 0
 * below -104 (both round to the same f32 as the exact value); otherwise
 * z = k*ln2/64 + r (Cody-Waite, k = RN(64 z / ln2), |r| <= ln2/128), e^r by
 * its Taylor series to r^7 (truncation < 2^-73), times POW_EXP2[k mod 64]
 * and the exact power 2^floor(k/64). */
static double or_exp_t64(double z) {
    if (z != z) return z;
    if (z > 89.0) return INFINITY;
    if (z < -104.0) return 0.0;
    const double K = 0x1.71547652b82fep+6; /* 64 / ln2 */
    const double L_HI = 6.93147180369123816490e-01 / 64.0, L_LO = 1.90821492927058770002e-10 / 64.0;
    const double kf = rint(z * K);
    const int k = (int)kf;
    const double r = (z - kf * L_HI) - kf * L_LO;
    double p = fma(1.0 / 5040.0, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return (p * POW_EXP2[k & 63]) * pow2i(k >> 6);
}

/* pow(x, y) = exp(y*log(x)) in f64, rounded once to f32; pow(0, y) = +inf,
 * 1 or 0 for y < 0, y == 0, y > 0. */
float or_powf(float x, float y) {
    if (x == 0.0f) return y < 0.0f ? INFINITY : (y == 0.0f ? 1.0f : 0.0f);
    return (float)or_exp_t64((double)y * or_log_t64(x));
}

int32_t or_f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}

void or_default_ext(OrExt* e) {
    memset(e, 0, sizeof(*e));
    e->gravity[0] = 0.0f; e->gravity[1] = 0.0f; e->gravity[2] = -9.81f;
    e->youngs_modulus = 1.4e5f;
    e->poissons_ratio = 0.2f;
    e->hardening_explicit = 5.0f;
    e->hardening_pbmpm = 20.0f;
    e->theta_c = 2.5e-2f;
    e->theta_s = 7.5e-3f;
    e->density = 400.0f;
    e->n_iter = 3;
    e->force_divisor = 3.0f;
    e->boundary_mode = 0;
    e->restitution = -0.5f;
    e->bc_cells = 2;
    e->ground_axis = 2;
    e->collider_margin = 0.05f;
    e->collider_surface_margin = 0.05f;
    e->collider_threshold = 0.05f;
    e->collider_friction = 0.1f;
    e->collider_vel_scale = 0.2f;
    e->pbmpm_blend = 0.95f;
    e->pbmpm_volume_exponent = -0.3333333f;
}
#endif /* !OR_FP64 */

/* ------------------------------------------------------------------ */
/* precision-dependent scalar ops                                      */
/* ------------------------------------------------------------------ */
#if OR_FP64
#define FMA(a, b, c) fma((a), (b), (c))
/* x / d for a divisor constant over the substep; rd = RN(1/d) in f32 */
#define KDIV(x, d, rd) ((x) / (d))
static inline real r_exp(real x) { return exp(x); }
static inline real r_pow(real x, real y) { return pow(x, y); }
static inline real r_sqrt(real x) { return sqrt(x); }
static inline real r_min(real a, real b) { return fmin(a, b); }
static inline real r_max(real a, real b) { return fmax(a, b); }
static inline real r_abs(real a) { return fabs(a); }
#else
#define FMA(a, b, c) fmaf((a), (b), (c))
#define KDIV(x, d, rd) ((x) * (rd))
static inline real r_exp(real x) { return (float)or_exp64((double)x); }
static inline real r_pow(real x, real y) { return or_powf(x, y); }
static inline real r_sqrt(real x) { return sqrtf(x); }
static inline real r_min(real a, real b) { return fminf(a, b); }
static inline real r_max(real a, real b) { return fmaxf(a, b); }
static inline real r_abs(real a) { return fabsf(a); }
#endif

static inline int32_t to_i32(real x) {
    if (x != x) return 0;
    if (x >= (real)2147483648.0) return 2147483647;
    if (x <= (real)-2147483648.0) return (int32_t)0x80000000u;
    return (int32_t)x;
}

static inline real sgn(real x) { return x > 0 ? (real)1 : (x < 0 ? (real)-1 : (real)0); }

/* ------------------------------------------------------------------ */
/* vector / matrix helpers (matrixOps.wgsl; WGSL builtins)             */
/* ------------------------------------------------------------------ */
static inline real dot3(const real* a, const real* b) { return FMA(a[2], b[2], FMA(a[1], b[1], a[0] * b[0])); }
static inline void cross3(const real* a, const real* b, real* o) {
    real x = FMA(a[1], b[2], -(a[2] * b[1]));
    real y = FMA(a[2], b[0], -(a[0] * b[2]));
    real z = FMA(a[0], b[1], -(a[1] * b[0]));
    o[0] = x; o[1] = y; o[2] = z;
}
static inline real len3(const real* a) { return r_sqrt(dot3(a, a)); }

static inline real det3(const real* m) {
    real k0 = FMA(m[4], m[8], -(m[7] * m[5]));
    real k1 = FMA(m[1], m[8], -(m[7] * m[2]));
    real k2 = FMA(m[1], m[5], -(m[4] * m[2]));
    return FMA(m[6], k2, FMA(-m[3], k1, m[0] * k0));
}

static const real IDENT[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

/* mat3x3Inverse (matrixOps.wgsl:8-27): adjugate * (1/det), identity if det == 0. */
static inline void inv3(const real* m, real* o) {
    real det = det3(m);
    if (det == 0) { memcpy(o, IDENT, sizeof(IDENT)); return; }
    real a[9];
    a[0] = FMA(m[4], m[8], -(m[5] * m[7]));
    a[1] = FMA(m[2], m[7], -(m[1] * m[8]));
    a[2] = FMA(m[1], m[5], -(m[2] * m[4]));
    a[3] = FMA(m[5], m[6], -(m[3] * m[8]));
    a[4] = FMA(m[0], m[8], -(m[2] * m[6]));
    a[5] = FMA(m[2], m[3], -(m[0] * m[5]));
    a[6] = FMA(m[3], m[7], -(m[4] * m[6]));
    a[7] = FMA(m[1], m[6], -(m[0] * m[7]));
    a[8] = FMA(m[0], m[4], -(m[1] * m[3]));
    real s = (real)1 / det;
    for (int i = 0; i < 9; i++) o[i] = a[i] * s;
}

static inline void tr3(const real* m, real* o) {
    real t[9] = {m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8]};
    memcpy(o, t, sizeof(t));
}

/* (A*B)[c][r] = sum_k A[k][r] * B[c][k] */
static inline void mul3(const real* A, const real* B, real* o) {
    real t[9];
    for (int c = 0; c < 3; c++)
        for (int r = 0; r < 3; r++)
            t[c * 3 + r] = FMA(A[2 * 3 + r], B[c * 3 + 2], FMA(A[1 * 3 + r], B[c * 3 + 1], A[0 * 3 + r] * B[c * 3 + 0]));
    memcpy(o, t, sizeof(t));
}

static inline void mv3(const real* M, const real* v, real* o) {
    real t[3];
    for (int r = 0; r < 3; r++) t[r] = FMA(M[2 * 3 + r], v[2], FMA(M[1 * 3 + r], v[1], M[0 * 3 + r] * v[0]));
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}

/* calculatePolarDecompositionRotation (matrixOps.wgsl:33-45). */
static inline void polar3(const real* F, real* R) {
    real g[9];
    memcpy(g, F, sizeof(g));
    for (int it = 0; it < 4; it++) {
        real iv[9], it_[9];
        inv3(g, iv);
        tr3(iv, it_);
        for (int i = 0; i < 9; i++) g[i] = (real)0.5 * (g[i] + it_[i]);
    }
    memcpy(R, g, sizeof(g));
}

/* mat4 (column-major 16) * vec4(v, 1).xyz */
static inline void xform_point(const real* M, const real* v, real* o) {
    real t[3];
    for (int r = 0; r < 3; r++)
        t[r] = FMA(M[2 * 4 + r], v[2], FMA(M[1 * 4 + r], v[1], M[0 * 4 + r] * v[0])) + M[3 * 4 + r];
    o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
}

/* ------------------------------------------------------------------ */
/* scene: uniform block (uniforms.wgsl:8-56) + extension parameters     */
/* ------------------------------------------------------------------ */
typedef struct Scene {
    real dt, scale;
    real gmin[3], gmax[3], cd[3];
    int32_t res[3];
    real cmin[3], cmax[3], xf[16], xfi[16], cvel[3];
    uint32_t c_nidx, c_nobj;
    real ipos[3], istr, irad;
    uint32_t iact, imode;
    real g[3], mu0, la0, xi_e, xi_p, smin, smax, inv_rho;
    uint32_t n_iter;
    real fdiv;
    uint32_t bmode;
    real rest;
    int32_t bc;
    uint32_t gaxis;
    real cmargin, csurf, cthr, cfric, cvs, blend, vexp;
    uint32_t rmap;   /* return map: 0 applyPlasticity, 1 SVD clamp (library option) */
    /* RN(1/d) of the substep-constant divisors (f32 instantiation), and
     * g*dt rounded once (gridUpdate.cs.wgsl:44) */
    real rdt, rcd[3], rscale, rfdiv, gdt[3];
} Scene;

static inline float rdf(const uint8_t* u, size_t off) { float f; memcpy(&f, u + off, 4); return f; }
static inline uint32_t rdu(const uint8_t* u, size_t off) { uint32_t v; memcpy(&v, u + off, 4); return v; }

static void load_scene(Scene* s, const uint8_t* u, const OrExt* e) {
    s->dt = rdf(u, 0);
    s->scale = rdf(u, 4);
    for (int i = 0; i < 3; i++) {
        s->gmin[i] = rdf(u, 16 + 4 * i);
        s->gmax[i] = rdf(u, 32 + 4 * i);
        s->res[i] = (int32_t)rdu(u, 208 + 4 * i);
        s->cmin[i] = rdf(u, 224 + 4 * i);
        s->cmax[i] = rdf(u, 240 + 4 * i);
        s->cvel[i] = rdf(u, 320 + 4 * i);
        s->cd[i] = rdf(u, 352 + 4 * i);
        s->ipos[i] = rdf(u, 496 + 4 * i);
    }
    for (int i = 0; i < 16; i++) {
        s->xf[i] = rdf(u, 256 + 4 * i);
        s->xfi[i] = rdf(u, 432 + 4 * i);
    }
    s->c_nidx = rdu(u, 348);
    s->c_nobj = rdu(u, 364);
    s->istr = rdf(u, 508);
    s->irad = rdf(u, 512);
    s->iact = rdu(u, 516);
    s->imode = rdu(u, 520);
    for (int i = 0; i < 3; i++) s->g[i] = e->gravity[i];
    /* WGSL evaluates these constant expressions at shader compile time in
     * abstract (f64) precision and rounds once: stressTensorOps.wgsl:5-6,
     * plasticityOps.wgsl:18-19, particleToGrid.cs.wgsl:37. */
    double E = e->youngs_modulus, nu = e->poissons_ratio;
    s->mu0 = (real)(E / (2.0 * (1.0 + nu)));
    s->la0 = (real)(E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    s->xi_e = e->hardening_explicit;
    s->xi_p = e->hardening_pbmpm;
    s->smin = (real)(1.0 - (double)e->theta_c);
    s->smax = (real)(1.0 + (double)e->theta_s);
    s->inv_rho = (real)(1.0 / (double)e->density);
    s->n_iter = e->n_iter;
    s->fdiv = e->force_divisor;
    s->bmode = e->boundary_mode;
    s->rest = e->restitution;
    s->bc = (int32_t)e->bc_cells;
    s->gaxis = e->ground_axis;
    s->cmargin = e->collider_margin;
    s->csurf = e->collider_surface_margin;
    s->cthr = e->collider_threshold;
    s->cfric = e->collider_friction;
    s->cvs = e->collider_vel_scale;
    s->blend = e->pbmpm_blend;
    s->vexp = e->pbmpm_volume_exponent;
    s->rmap = e->return_map;
    s->rdt = (real)1 / s->dt;
    for (int i = 0; i < 3; i++) s->rcd[i] = (real)1 / s->cd[i];
    s->rscale = (real)1 / s->scale;
    s->rfdiv = (real)1 / s->fdiv;
    for (int i = 0; i < 3; i++) s->gdt[i] = s->g[i] * s->dt;
}

/* ------------------------------------------------------------------ */
/* particle state                                                      */
/* ------------------------------------------------------------------ */
typedef struct PS {
    real pos[3], vel[3], mass, Fe[9], Fp[9], dxp[3], D[9];
} PS;

#if OR_FP64
static inline void p_load(const PART* p, PS* s) {
    memcpy(s->pos, p->pos, sizeof(s->pos)); memcpy(s->vel, p->vel, sizeof(s->vel));
    s->mass = p->mass;
    memcpy(s->Fe, p->Fe, sizeof(s->Fe)); memcpy(s->Fp, p->Fp, sizeof(s->Fp));
    memcpy(s->dxp, p->dxp, sizeof(s->dxp)); memcpy(s->D, p->D, sizeof(s->D));
}
static inline void p_store(PART* p, const PS* s) {
    memcpy(p->pos, s->pos, sizeof(s->pos)); memcpy(p->vel, s->vel, sizeof(s->vel));
    p->mass = s->mass;
    memcpy(p->Fe, s->Fe, sizeof(s->Fe)); memcpy(p->Fp, s->Fp, sizeof(s->Fp));
    memcpy(p->dxp, s->dxp, sizeof(s->dxp)); memcpy(p->D, s->D, sizeof(s->D));
}
#else
static inline void m_unpack(const float* pad12, float* m9) {
    for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) m9[c * 3 + r] = pad12[c * 4 + r];
}
static inline void m_pack(const float* m9, float* pad12) {
    for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) pad12[c * 4 + r] = m9[c * 3 + r];
}
static inline void p_load(const PART* p, PS* s) {
    memcpy(s->pos, p->pos, 12); memcpy(s->vel, p->vel, 12);
    s->mass = p->mass;
    m_unpack(p->Fe, s->Fe); m_unpack(p->Fp, s->Fp);
    memcpy(s->dxp, p->dxp, 12); m_unpack(p->D, s->D);
}
static inline void p_store(PART* p, const PS* s) {
    memcpy(p->pos, s->pos, 12); memcpy(p->vel, s->vel, 12);
    p->mass = s->mass;
    m_pack(s->Fe, p->Fe); m_pack(s->Fp, p->Fp);
    memcpy(p->dxp, s->dxp, 12); m_pack(s->D, p->D);
}
#endif

/* ------------------------------------------------------------------ */
/* grid geometry (mpmOps.wgsl:14-53)                                    */
/* ------------------------------------------------------------------ */
static inline void cell_number(const Scene* s, const real* pos, int32_t* c) {
    for (int i = 0; i < 3; i++) c[i] = to_i32(KDIV(pos[i] - s->gmin[i], s->cd[i], s->rcd[i]));
}
static inline int in_range(const Scene* s, const int32_t* c) {
    return 0 <= c[0] && 0 <= c[1] && 0 <= c[2] && c[0] < s->res[0] && c[1] < s->res[1] && c[2] < s->res[2];
}
static inline void frac_pos(const Scene* s, const real* pos, const int32_t* c, real* f) {
    for (int i = 0; i < 3; i++) {
        real mn = FMA(s->cd[i], (real)c[i], s->gmin[i]);
        f[i] = KDIV(pos[i] - mn, s->cd[i], s->rcd[i]);
    }
}
/* w[k][axis], k = offset + 1 */
static inline void bspline_w(const real* f, real w[3][3]) {
    for (int i = 0; i < 3; i++) {
        w[0][i] = ((real)0.5 * ((real)1 - f[i])) * ((real)1 - f[i]);
        w[1][i] = FMA(-(f[i] - (real)0.5), f[i] - (real)0.5, (real)0.75);
        w[2][i] = ((real)0.5 * f[i]) * f[i];
    }
}
static inline void bspline_dw(const real* f, real d[3][3]) {
    for (int i = 0; i < 3; i++) {
        d[0][i] = f[i] - (real)1;
        d[1][i] = (real)-2 * (f[i] - (real)0.5);
        d[2][i] = f[i];
    }
}

/* ------------------------------------------------------------------ */
/* context: block hash map (sparseGridPrelude.wgsl:1-24) and grid      */
/* ------------------------------------------------------------------ */
#define EMPTY_IDX 0xFFFFFFFFu
#define RESERVED_IDX 0xFFFFFFFEu
#define N_PROBES 100u

struct OrCtx {
    uint32_t hash_size, max_blocks, max_particles;
    int32_t* coord;          /* hash_size * 3 */
    uint32_t* index;         /* hash_size */
    uint32_t n_blocks;
    uint32_t* mapped;        /* max_blocks */
    uint32_t* counts;
    uint32_t* offsets;
    uint32_t* sorted;        /* max_particles */
#if OR_FP64
    double* grid;            /* max_blocks * 64 * 4 */
#else
    uint32_t* grid;          /* i32 fixed point stored as u32 for wrapping adds */
#endif
    uint32_t status;
};

OrCtx* PFX(create)(uint32_t hash_size, uint32_t max_blocks, uint32_t max_particles) {
    OrCtx* c = (OrCtx*)calloc(1, sizeof(OrCtx));
    if (!c) return NULL;
    c->hash_size = hash_size;
    c->max_blocks = max_blocks;
    c->max_particles = max_particles;
    c->coord = (int32_t*)calloc((size_t)hash_size * 3, sizeof(int32_t));
    c->index = (uint32_t*)calloc(hash_size, sizeof(uint32_t));
    c->mapped = (uint32_t*)calloc(max_blocks, sizeof(uint32_t));
    c->counts = (uint32_t*)calloc(max_blocks, sizeof(uint32_t));
    c->offsets = (uint32_t*)calloc(max_blocks, sizeof(uint32_t));
    c->sorted = (uint32_t*)calloc(max_particles ? max_particles : 1, sizeof(uint32_t));
    c->grid = calloc((size_t)max_blocks * 256, sizeof(*c->grid));
    if (!c->coord || !c->index || !c->mapped || !c->counts || !c->offsets || !c->sorted || !c->grid) {
        PFX(destroy)(c);
        return NULL;
    }
    return c;
}

void PFX(destroy)(OrCtx* c) {
    if (!c) return;
    free(c->coord); free(c->index); free(c->mapped); free(c->counts);
    free(c->offsets); free(c->sorted); free(c->grid); free(c);
}

uint32_t PFX(status)(const OrCtx* c) { return c->status; }

#if !OR_FP64
uint32_t orf_n_blocks(const OrCtx* c) { return c->n_blocks; }
void orf_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
#endif

static inline uint32_t ld_idx(uint32_t* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }

/* clearHashMap (clearHashMap.wgsl:7-19) */
static void clear_hash(OrCtx* c) {
    c->n_blocks = 0;
    for (uint32_t i = 0; i < c->hash_size; i++) c->index[i] = EMPTY_IDX;
}

/* allocateBlock (mapAffectedBlocks.wgsl:7-62).  The reference gives up on a
 * reserved slot after 32 polls and re-probes it; here the poll waits until
 * the reserving thread has published (it always makes progress on a CPU), so
 * the result does not depend on thread timing. */
static void allocate_block(OrCtx* c, const int32_t* b) {
    uint32_t h = or_hash3((uint32_t)b[0], (uint32_t)b[1], (uint32_t)b[2]);
    uint32_t cand = h % c->hash_size;
    for (uint32_t i = 0; i < N_PROBES; i++) {
        uint32_t cur = ld_idx(&c->index[cand]);
        if (cur == EMPTY_IDX) {
            uint32_t expect = EMPTY_IDX;
            if (__atomic_compare_exchange_n(&c->index[cand], &expect, RESERVED_IDX, 0,
                                            __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE)) {
                uint32_t next = __atomic_fetch_add(&c->n_blocks, 1u, __ATOMIC_ACQ_REL);
                if (next >= c->max_blocks) {
                    __atomic_or_fetch(&c->status, OR_STATUS_BLOCK_OVERFLOW, __ATOMIC_RELAXED);
                    __atomic_store_n(&c->index[cand], EMPTY_IDX, __ATOMIC_RELEASE);
                    return;
                }
                c->coord[cand * 3 + 0] = b[0];
                c->coord[cand * 3 + 1] = b[1];
                c->coord[cand * 3 + 2] = b[2];
                c->mapped[next] = cand;
                __atomic_store_n(&c->index[cand], next, __ATOMIC_RELEASE);
                return;
            }
            cur = ld_idx(&c->index[cand]);
        }
        while (cur == RESERVED_IDX) cur = ld_idx(&c->index[cand]);
        if (cur == EMPTY_IDX) continue;
        if (c->coord[cand * 3 + 0] == b[0] && c->coord[cand * 3 + 1] == b[1] && c->coord[cand * 3 + 2] == b[2]) return;
        cand = (cand + 1 >= c->hash_size) ? 0 : cand + 1;
    }
    __atomic_or_fetch(&c->status, OR_STATUS_HASH_PROBE_FAIL, __ATOMIC_RELAXED);
}

/* retrieveBlockIndexFromHashMap (sparseGridPrelude.wgsl:35-52).  Note the u32
 * wrap of (hash + i) before the modulo, kept as the reference has it. */
static inline uint32_t lookup_block(const OrCtx* c, const int32_t* b) {
    uint32_t h = or_hash3((uint32_t)b[0], (uint32_t)b[1], (uint32_t)b[2]);
    for (uint32_t i = 0; i < N_PROBES; i++) {
        uint32_t cand = (uint32_t)(h + i) % c->hash_size;
        uint32_t bi = c->index[cand];
        if (bi == EMPTY_IDX) return EMPTY_IDX;
        if (c->coord[cand * 3 + 0] == b[0] && c->coord[cand * 3 + 1] == b[1] && c->coord[cand * 3 + 2] == b[2]) return bi;
    }
    return EMPTY_IDX;
}

/* calculateCellIndexFromCellNumber (sparseGridPrelude.wgsl:54-65) */
static inline uint32_t cell_index(const OrCtx* c, const int32_t* cell) {
    int32_t b[3] = {cell[0] >> 2, cell[1] >> 2, cell[2] >> 2};
    uint32_t bi = lookup_block(c, b);
    if (bi == EMPTY_IDX) return EMPTY_IDX;
    uint32_t w = (uint32_t)((cell[0] & 3) + (cell[1] & 3) * 4 + (cell[2] & 3) * 16);
    return bi * 64u + w;
}

/* ------------------------------------------------------------------ */
/* grid accumulation                                                   */
/* ------------------------------------------------------------------ */
#if OR_FP64
static inline void grid_add(OrCtx* c, uint32_t ci, int comp, real v) {
    double* p = &c->grid[(size_t)ci * 4 + comp];
#pragma omp atomic
    *p += v;
}
#else
static inline void grid_add(OrCtx* c, uint32_t ci, int comp, real v) {
    __atomic_fetch_add(&c->grid[(size_t)ci * 4 + comp], (uint32_t)to_i32(v), __ATOMIC_RELAXED);
}
#endif

/* the value the reference adds for one component: i32(x * fixedPointScale) */
#if OR_FP64
#define ENC(x, s) (x)
#else
#define ENC(x, s) ((x) * (s))
#endif

/* ------------------------------------------------------------------ */
/* hardening + stress (stressTensorOps.wgsl:9-22, 39-56)                */
/* ------------------------------------------------------------------ */
static void stress_pk1(const Scene* s, const PS* p, real* P) {
    real mu = s->mu0, la = s->la0;
    real Jp = det3(p->Fp);
    real ef = r_exp(s->xi_e * ((real)1 - Jp));
    mu *= ef;
    la *= ef;
    real J = det3(p->Fe);
    real R[9], Fi[9], FiT[9];
    polar3(p->Fe, R);
    inv3(p->Fe, Fi);
    tr3(Fi, FiT);
    real a = (real)2 * mu;
    real b = (la * (J - (real)1)) * J;
    for (int i = 0; i < 9; i++) P[i] = FMA(b, FiT[i], a * (p->Fe[i] - R[i]));
}

/* ------------------------------------------------------------------ */
/* P2G                                                                  */
/* ------------------------------------------------------------------ */
/* explicit branch of doParticleToGrid (particleToGrid.cs.wgsl:27-79) */
static void p2g_explicit(OrCtx* c, const Scene* s, const PS* p) {
    int32_t cell[3];
    real f[3], w[3][3], dw[3][3];
    cell_number(s, p->pos, cell);
    frac_pos(s, p->pos, cell, f);
    bspline_w(f, w);
    bspline_dw(f, dw);
    real P[9], Pt[9], M[9];
    stress_pk1(s, p, P);
    tr3(P, Pt);
    real V = p->mass * s->inv_rho;
    for (int i = 0; i < 9; i++) M[i] = (-V) * Pt[i];
    real pm[3] = {p->mass * p->vel[0], p->mass * p->vel[1], p->mass * p->vel[2]};
    for (int oz = -1; oz <= 1; oz++)
        for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++) {
                int32_t cc[3] = {cell[0] + ox, cell[1] + oy, cell[2] + oz};
                if (!in_range(s, cc)) continue;
                uint32_t ci = cell_index(c, cc);
                if (ci == EMPTY_IDX) continue;
                real wgt = (w[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2];
                real g[3];
                g[0] = KDIV((dw[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2], s->cd[0], s->rcd[0]);
                g[1] = KDIV((w[ox + 1][0] * dw[oy + 1][1]) * w[oz + 1][2], s->cd[1], s->rcd[1]);
                g[2] = KDIV((w[ox + 1][0] * w[oy + 1][1]) * dw[oz + 1][2], s->cd[2], s->rcd[2]);
                real sf[3];
                mv3(M, g, sf);
                real mom[3];
                for (int k = 0; k < 3; k++) mom[k] = FMA(wgt, pm[k], sf[k] * s->dt);
                grid_add(c, ci, 1, ENC(mom[0], s->scale));
                grid_add(c, ci, 2, ENC(mom[1], s->scale));
                grid_add(c, ci, 3, ENC(mom[2], s->scale));
                grid_add(c, ci, 0, ENC(wgt * p->mass, s->scale));
            }
}

/* solveParticleConstraints (pbmpm.wgsl:16-39) */
static void pbmpm_constraints(const Scene* s, PS* p) {
    real IpD[9], Ft[9], Rt[9];
    for (int i = 0; i < 9; i++) IpD[i] = IDENT[i] + p->D[i];
    mul3(IpD, p->Fe, Ft);
    polar3(Ft, Rt);
    real tv = det3(Ft);
    real vs = r_pow(r_abs(tv), s->vexp);
    real tb[9], Fei[9], Dc[9];
    real ob = (real)1 - s->blend;
    for (int i = 0; i < 9; i++) {
        real ts = Rt[i] * vs;
        tb[i] = FMA(s->blend, ts, ob * Rt[i]);
    }
    inv3(p->Fe, Fei);
    mul3(tb, Fei, Dc);
    for (int i = 0; i < 9; i++) Dc[i] = Dc[i] - IDENT[i];
    real J = det3(p->Fp);
    real relax = FMA((real)0.5, (real)1 - r_exp((-s->xi_p) / J), (real)0.5);
    for (int i = 0; i < 9; i++) {
        real diff = Dc[i] - p->D[i];
        p->D[i] = FMA(relax, diff, p->D[i]);
    }
}

/* transferParticlesToGrid + updateGrid (pbmpm.wgsl:41-147); the affine branch
 * of doParticleToGrid (particleToGrid.cs.wgsl:81-114) is the same transfer. */
static void p2g_pbmpm(OrCtx* c, const Scene* s, const PS* p, int with_forces) {
    int32_t cell[3];
    real f[3], w[3][3];
    cell_number(s, p->pos, cell);
    frac_pos(s, p->pos, cell, f);
    bspline_w(f, w);
    real pcp[3];
    for (int i = 0; i < 3; i++) pcp[i] = ((real)cell[i] + f[i]) - (real)0.5;
    for (int oz = -1; oz <= 1; oz++)
        for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++) {
                int32_t cc[3] = {cell[0] + ox, cell[1] + oy, cell[2] + oz};
                if (!in_range(s, cc)) continue;
                uint32_t ci = cell_index(c, cc);
                if (ci == EMPTY_IDX) continue;
                real wgt = (w[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2];
                real wm = wgt * p->mass;
                real off[3], aff[3], mom[3];
                for (int k = 0; k < 3; k++) off[k] = (real)cc[k] - pcp[k];
                mv3(p->D, off, aff);
                for (int k = 0; k < 3; k++) mom[k] = KDIV(wm * (p->dxp[k] + aff[k]), s->dt, s->rdt);
                grid_add(c, ci, 1, ENC(mom[0], s->scale));
                grid_add(c, ci, 2, ENC(mom[1], s->scale));
                grid_add(c, ci, 3, ENC(mom[2], s->scale));
                grid_add(c, ci, 0, ENC(wm, s->scale));
            }
    if (!with_forces) return;
    /* updateGrid: second 27-cell loop, momentum only */
    for (int oz = -1; oz <= 1; oz++)
        for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++) {
                int32_t cc[3] = {cell[0] + ox, cell[1] + oy, cell[2] + oz};
                if (!in_range(s, cc)) continue;
                uint32_t ci = cell_index(c, cc);
                if (ci == EMPTY_IDX) continue;
                real wgt = (w[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2];
                real wm = wgt * p->mass;
                real fo[3] = {s->g[0], s->g[1], s->g[2]};
                if (s->iact != 0u) {
                    real gnp[3] = {(real)cc[0], (real)cc[1], (real)cc[2]};
                    real dv[3] = {gnp[0] - s->ipos[0], gnp[1] - s->ipos[1], gnp[2] - s->ipos[2]};
                    real dist = len3(dv);
                    if (dist < s->irad) {
                        real offv[3] = {gnp[0] - s->ipos[0], gnp[1] - s->ipos[1], gnp[2] - s->ipos[2]};
                        real pd[3] = {0, 0, 1};
                        if (len3(offv) > (real)0.001) {
                            real l = len3(offv);
                            for (int k = 0; k < 3; k++) pd[k] = offv[k] / l;
                        }
                        real fl = dist / s->irad;
                        real falloff = (real)1 - fl * fl;
                        real af[3];
                        if (s->imode == 0u) {
                            for (int k = 0; k < 3; k++) af[k] = (pd[k] * s->istr) * falloff;
                        } else {
                            for (int k = 0; k < 3; k++) af[k] = (((-pd[k]) * s->istr) * falloff) * ((real)1 - falloff);
                        }
                        for (int k = 0; k < 3; k++) fo[k] = fo[k] + af[k];
                    }
                }
                for (int k = 0; k < 3; k++) fo[k] = KDIV(fo[k], s->fdiv, s->rfdiv);
                real mc[3];
                for (int k = 0; k < 3; k++) mc[k] = (fo[k] * wm) * s->dt;
                grid_add(c, ci, 1, ENC(mc[0], s->scale));
                grid_add(c, ci, 2, ENC(mc[1], s->scale));
                grid_add(c, ci, 3, ENC(mc[2], s->scale));
            }
}

/* ------------------------------------------------------------------ */
/* grid cell decode                                                    */
/* ------------------------------------------------------------------ */
#if OR_FP64
static inline real cell_mass(const OrCtx* c, const Scene* s, uint32_t ci) { (void)s; return c->grid[(size_t)ci * 4]; }
static inline real cell_mom(const OrCtx* c, const Scene* s, uint32_t ci, int k) { (void)s; return c->grid[(size_t)ci * 4 + 1 + k]; }
#else
static inline real cell_mass(const OrCtx* c, const Scene* s, uint32_t ci) {
    return KDIV((real)(int32_t)c->grid[(size_t)ci * 4], s->scale, s->rscale);
}
static inline real cell_mom(const OrCtx* c, const Scene* s, uint32_t ci, int k) {
    return KDIV((real)(int32_t)c->grid[(size_t)ci * 4 + 1 + k], s->scale, s->rscale);
}
#endif

/* momentum / cell mass: momentum * RN(1/mass) in f32, IEEE division in f64 */
static inline void div_mass(real* v, real m) {
#if OR_FP64
    for (int k = 0; k < 3; k++) v[k] = v[k] / m;
#else
    real rm = (real)1 / m;
    for (int k = 0; k < 3; k++) v[k] = v[k] * rm;
#endif
}

/* Grid-side boundary of boundary_mode 1 (an extension: sticky ground plane at
 * the grid minimum of `ground_axis`, slip walls elsewhere). */
static inline void grid_bc(const Scene* s, const int32_t* cc, real* v) {
    if (s->bmode != 1u) return;
    if (cc[s->gaxis] < s->bc) { v[0] = 0; v[1] = 0; v[2] = 0; return; }
    for (int a = 0; a < 3; a++) {
        if (cc[a] < s->bc && v[a] < 0) v[a] = 0;
        if (cc[a] >= s->res[a] - s->bc && v[a] > 0) v[a] = 0;
    }
}

/* doGridUpdate explicit branch (gridUpdate.cs.wgsl:15-53) */
static void grid_update_explicit(OrCtx* c, const Scene* s) {
    uint32_t nb = c->n_blocks < c->max_blocks ? c->n_blocks : c->max_blocks;
#pragma omp parallel for schedule(static)
    for (uint32_t b = 0; b < nb; b++) {
        uint32_t slot = c->mapped[b];
        int32_t bn[3] = {c->coord[slot * 3], c->coord[slot * 3 + 1], c->coord[slot * 3 + 2]};
        for (uint32_t l = 0; l < 64; l++) {
            uint32_t ci = b * 64u + l;
            real m = cell_mass(c, s, ci);
            if (m <= 0) continue;
            real v[3];
            for (int k = 0; k < 3; k++) v[k] = cell_mom(c, s, ci, k);
            div_mass(v, m);
            for (int k = 0; k < 3; k++) v[k] = v[k] + s->gdt[k];
            int32_t cc[3] = {bn[0] * 4 + (int32_t)(l & 3), bn[1] * 4 + (int32_t)((l >> 2) & 3), bn[2] * 4 + (int32_t)(l >> 4)};
            grid_bc(s, cc, v);
#if OR_FP64
            for (int k = 0; k < 3; k++) c->grid[(size_t)ci * 4 + 1 + k] = v[k] * m;
#else
            for (int k = 0; k < 3; k++) c->grid[(size_t)ci * 4 + 1 + k] = (uint32_t)to_i32((v[k] * m) * s->scale);
#endif
        }
    }
}

/* velocity the G2P kernels read from one cell; returns 0 when the cell is skipped */
static inline int cell_velocity(const OrCtx* c, const Scene* s, const int32_t* cc, int pbmpm, real* v) {
    if (!in_range(s, cc)) return 0;
    uint32_t ci = cell_index(c, cc);
    if (ci == EMPTY_IDX) return 0;
    real m = cell_mass(c, s, ci);
    if (m <= 0) return 0;
    for (int k = 0; k < 3; k++) v[k] = cell_mom(c, s, ci, k);
    div_mass(v, m);
    if (pbmpm) grid_bc(s, cc, v);
    return 1;
}

/* doGridToParticle (gridToParticle.cs.wgsl:14-131) */
static void g2p(const OrCtx* c, const Scene* s, PS* p, int pbmpm) {
    int32_t cell[3];
    real f[3], w[3][3], dw[3][3];
    cell_number(s, p->pos, cell);
    frac_pos(s, p->pos, cell, f);
    bspline_w(f, w);
    bspline_dw(f, dw);
    real nv[3] = {0, 0, 0};
    real G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    real pcp[3];
    for (int i = 0; i < 3; i++) pcp[i] = ((real)cell[i] + f[i]) - (real)0.5;
    for (int oz = -1; oz <= 1; oz++)
        for (int oy = -1; oy <= 1; oy++)
            for (int ox = -1; ox <= 1; ox++) {
                int32_t cc[3] = {cell[0] + ox, cell[1] + oy, cell[2] + oz};
                real cv[3];
                if (!cell_velocity(c, s, cc, pbmpm, cv)) continue;
                real wgt = (w[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2];
                if (!pbmpm) {
                    for (int k = 0; k < 3; k++) nv[k] = FMA(wgt, cv[k], nv[k]);
                    real g[3];
                    g[0] = (dw[ox + 1][0] * w[oy + 1][1]) * w[oz + 1][2];
                    g[1] = (w[ox + 1][0] * dw[oy + 1][1]) * w[oz + 1][2];
                    g[2] = (w[ox + 1][0] * w[oy + 1][1]) * dw[oz + 1][2];
                    for (int col = 0; col < 3; col++)
                        for (int r = 0; r < 3; r++) G[col * 3 + r] = FMA(g[col], cv[r], G[col * 3 + r]);
                } else {
                    for (int k = 0; k < 3; k++) nv[k] = FMA(wgt, cv[k], nv[k]);
                    real wv[3] = {wgt * cv[0], wgt * cv[1], wgt * cv[2]};
                    real dist[3];
                    for (int k = 0; k < 3; k++) dist[k] = (real)cc[k] - pcp[k];
                    for (int col = 0; col < 3; col++)
                        for (int r = 0; r < 3; r++) G[col * 3 + r] = FMA(wv[r], dist[col], G[col * 3 + r]);
                }
            }
    for (int k = 0; k < 3; k++) p->vel[k] = nv[k];
    for (int k = 0; k < 3; k++) p->dxp[k] = nv[k] * s->dt;
    if (!pbmpm) {
        for (int i = 0; i < 9; i++) p->D[i] = G[i] * s->dt;
    } else {
        for (int i = 0; i < 9; i++) p->D[i] = (G[i] * s->dt) * (real)4;
    }
}

/* ------------------------------------------------------------------ */
/* plasticity (plasticityOps.wgsl:7-48)                                */
/* ------------------------------------------------------------------ */
static void plasticity_svd(const Scene* s, real* Fe, real* Fp);

static void plasticity(const Scene* s, real* Fe, real* Fp) {
    if (s->rmap == 1u) {
        plasticity_svd(s, Fe, Fp);
        return;
    }
    real R[9], Rt[9], S[9];
    polar3(Fe, R);
    tr3(R, Rt);
    mul3(Rt, Fe, S);
    real sg[3] = {S[0], S[4], S[8]};
    if (s->smin <= sg[0] && s->smin <= sg[1] && s->smin <= sg[2] &&
        sg[0] <= s->smax && sg[1] <= s->smax && sg[2] <= s->smax) return;
    real sc[3];
    for (int k = 0; k < 3; k++) sc[k] = r_min(r_max(sg[k], s->smin), s->smax);
    real Dg[9] = {sc[0], 0, 0, 0, sc[1], 0, 0, 0, sc[2]};
    real Fn[9], Fni[9], F[9], Fpn[9];
    mul3(R, Dg, Fn);
    inv3(Fn, Fni);
    mul3(Fe, Fp, F);
    mul3(Fni, F, Fpn);
    memcpy(Fe, Fn, sizeof(Fn));
    memcpy(Fp, Fpn, sizeof(Fpn));
}

/* ------------------------------------------------------------------ */
/* SVD return map (return_map 1): an option of this library, not the      */
/* reference's map.  One-sided Jacobi SVD (M. R. Hestenes, "Inversion of  */
/* matrices by biorthogonalization and related results", J. SIAM 6, 1958): */
/* the column pairs (0,1), (0,2), (1,2) of A = Fe are rotated in 4 sweeps */
/* until A V = U diag(sigma), sigma_k = |a_k|.  Every sigma in            */
/* [smin, smax]: unchanged; else Fe' = sum_k (clamp(sigma_k) / sigma_k)    */
/* a_k v_k^T and Fp' = Fe'^-1 (Fe Fp).  Same operations as plasticity_svd */
/* in mpm_plast.cuh.                                                     */
/* ------------------------------------------------------------------ */
#define SVD_SWEEPS 4
static inline void jrot(real* x, real* y, real c, real sn) {
    for (int r = 0; r < 3; r++) {
        real xr = x[r], yr = y[r];
        x[r] = c * xr - sn * yr;
        y[r] = sn * xr + c * yr;
    }
}
static void plasticity_svd(const Scene* s, real* Fe, real* Fp) {
    real a[9], v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    memcpy(a, Fe, sizeof(a));
    static const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
    for (int sw = 0; sw < SVD_SWEEPS; sw++)
        for (int k = 0; k < 3; k++) {
            real* ap = a + 3 * P[k];
            real* aq = a + 3 * Q[k];
            real al = dot3(ap, ap), be = dot3(aq, aq), ga = dot3(ap, aq);
            if (ga == (real)0) continue;
            real ze = (be - al) / ((real)2 * ga);
            real t = (signbit(ze) ? (real)-1 : (real)1) / (r_abs(ze) + r_sqrt(FMA(ze, ze, (real)1)));
            real c = (real)1 / r_sqrt(FMA(t, t, (real)1));
            real sn = c * t;
            jrot(ap, aq, c, sn);
            jrot(v + 3 * P[k], v + 3 * Q[k], c, sn);
        }
    real sg[3];
    for (int k = 0; k < 3; k++) sg[k] = r_sqrt(dot3(a + 3 * k, a + 3 * k));
    if (s->smin <= sg[0] && s->smin <= sg[1] && s->smin <= sg[2] &&
        sg[0] <= s->smax && sg[1] <= s->smax && sg[2] <= s->smax) return;
    real w[3];
    for (int k = 0; k < 3; k++) w[k] = sg[k] > (real)0 ? r_min(r_max(sg[k], s->smin), s->smax) / sg[k] : (real)1;
    real Fn[9], Fni[9], F[9], Fpn[9];
    for (int j = 0; j < 3; j++)
        for (int r = 0; r < 3; r++)
            Fn[3 * j + r] = FMA((w[2] * a[6 + r]), v[6 + j], FMA((w[1] * a[3 + r]), v[3 + j], (w[0] * a[r]) * v[j]));
    inv3(Fn, Fni);
    mul3(Fe, Fp, F);
    mul3(Fni, F, Fpn);
    memcpy(Fe, Fn, sizeof(Fn));
    memcpy(Fp, Fpn, sizeof(Fpn));
}

/* ------------------------------------------------------------------ */
/* collider (colliderPrelude.wgsl:1-356)                                */
/* ------------------------------------------------------------------ */
static inline void col_vertex(const OrCollider* col, const Scene* s, uint32_t idx, real* v) {
    uint32_t base = s->c_nidx + idx * 3u;
    for (int k = 0; k < 3; k++) {
        float f;
        uint32_t w = base + (uint32_t)k < col->data_words ? col->data[base + k] : 0u;
        memcpy(&f, &w, 4);
        v[k] = f;
    }
}

static void closest_point_tri(const real* p, const real* a, const real* b, const real* c, real* o) {
    real ab[3], ac[3], ap[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = p[k] - a[k]; }
    real d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) { memcpy(o, a, 3 * sizeof(real)); return; }
    real bp[3];
    for (int k = 0; k < 3; k++) bp[k] = p[k] - b[k];
    real d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) { memcpy(o, b, 3 * sizeof(real)); return; }
    real vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        real v = d1 / (d1 - d3);
        for (int k = 0; k < 3; k++) o[k] = a[k] + v * ab[k];
        return;
    }
    real cp[3];
    for (int k = 0; k < 3; k++) cp[k] = p[k] - c[k];
    real d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) { memcpy(o, c, 3 * sizeof(real)); return; }
    real vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        real w = d2 / (d2 - d6);
        for (int k = 0; k < 3; k++) o[k] = a[k] + w * ac[k];
        return;
    }
    real va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        real w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; k++) o[k] = b[k] + w * (c[k] - b[k]);
        return;
    }
    real denom = (real)1 / ((va + vb) + vc);
    real v = vb * denom, w = vc * denom;
    for (int k = 0; k < 3; k++) o[k] = (a[k] + v * ab[k]) + w * ac[k];
}

static real ray_tri(const real* org, const real* dir, const real* a, const real* b, const real* c) {
    const real EPS = (real)1e-6f;
    real e1[3], e2[3], h[3], sv[3], q[3];
    for (int k = 0; k < 3; k++) { e1[k] = b[k] - a[k]; e2[k] = c[k] - a[k]; }
    cross3(dir, e2, h);
    real aa = dot3(e1, h);
    if (aa > -EPS && aa < EPS) return -1;
    real f = (real)1 / aa;
    for (int k = 0; k < 3; k++) sv[k] = org[k] - a[k];
    real u = f * dot3(sv, h);
    if (u < 0 || u > 1) return -1;
    cross3(sv, e1, q);
    real v = f * dot3(dir, q);
    if (v < 0 || u + v > 1) return -1;
    real t = f * dot3(e2, q);
    if (t > EPS) return t;
    return -1;
}

static void collide(OrCtx* ctx, const Scene* s, const OrCollider* col, PS* p) {
    if (!col || col->n_nodes == 0) return;
    real mnb[3], mxb[3];
    xform_point(s->xf, s->cmin, mnb);
    xform_point(s->xf, s->cmax, mxb);
    const real margin = s->cmargin;
    real smin[3], smax[3];
    for (int k = 0; k < 3; k++) {
        smin[k] = r_min(mnb[k], mxb[k]) - margin;
        smax[k] = r_max(mnb[k], mxb[k]) + margin;
    }
    real cur[3], prev[3], minp[3], maxp[3];
    for (int k = 0; k < 3; k++) {
        cur[k] = p->pos[k];
        prev[k] = cur[k] - p->dxp[k];
        minp[k] = r_min(cur[k], prev[k]);
        maxp[k] = r_max(cur[k], prev[k]);
    }
    for (int k = 0; k < 3; k++)
        if (minp[k] > smax[k] || maxp[k] < smin[k]) return;
    if (s->c_nobj == 0u) return;

    real min_d2 = (real)1e20f;
    real cnorm[3] = {0, 0, 1}, cpos[3] = {cur[0], cur[1], cur[2]};
    real min_t = 1;
    real hnorm[3] = {0, 0, 1}, hpos[3] = {cur[0], cur[1], cur[2]};
    int has_hit = 0;
    real rd[3] = {p->dxp[0], p->dxp[1], p->dxp[2]};
    real rlen = len3(rd);
    int do_ccd = rlen > (real)1e-4f;
    real curl[3], prevl[3];
    xform_point(s->xfi, cur, curl);
    xform_point(s->xfi, prev, prevl);
    real pminl[3], pmaxl[3];
    for (int k = 0; k < 3; k++) {
        pminl[k] = r_min(curl[k], prevl[k]);
        pmaxl[k] = r_max(curl[k], prevl[k]);
    }
    uint32_t stack[32];
    uint32_t sp = 0;
    stack[sp++] = 0;
    uint32_t visits = 0, max_visits = 2u * col->n_nodes + 64u;
    while (sp > 0) {
        if (++visits > max_visits) { __atomic_or_fetch(&ctx->status, OR_STATUS_BVH_STACK, __ATOMIC_RELAXED); break; }
        uint32_t ni = stack[--sp];
        if (ni >= col->n_nodes) continue;
        const uint32_t* nd = col->nodes + (size_t)ni * 8;
        float nf[8];
        memcpy(nf, nd, 32);
        real bmin[3] = {(real)nf[0] - margin, (real)nf[1] - margin, (real)nf[2] - margin};
        real bmax[3] = {(real)nf[4] + margin, (real)nf[5] + margin, (real)nf[6] + margin};
        if (pminl[0] > bmax[0] || pminl[1] > bmax[1] || pminl[2] > bmax[2] ||
            pmaxl[0] < bmin[0] || pmaxl[1] < bmin[1] || pmaxl[2] < bmin[2]) continue;
        if (nd[7] & 0x80000000u) {
            uint32_t start = nd[3], cnt = nd[7] & 0x7FFFFFFFu, end = start + cnt;
            for (uint32_t i = start; i < end; i++) {
                uint32_t tb = i * 3u;
                if (tb + 2 >= col->data_words) break;
                real v0l[3], v1l[3], v2l[3], v0[3], v1[3], v2[3];
                col_vertex(col, s, col->data[tb], v0l);
                col_vertex(col, s, col->data[tb + 1], v1l);
                col_vertex(col, s, col->data[tb + 2], v2l);
                xform_point(s->xf, v0l, v0);
                xform_point(s->xf, v1l, v1);
                xform_point(s->xf, v2l, v2);
                real cp[3], df[3];
                closest_point_tri(cur, v0, v1, v2, cp);
                for (int k = 0; k < 3; k++) df[k] = cur[k] - cp[k];
                real d2 = dot3(df, df);
                if (d2 < min_d2) {
                    min_d2 = d2;
                    memcpy(cpos, cp, sizeof(cp));
                    real e1[3], e2[3], n[3];
                    for (int k = 0; k < 3; k++) { e1[k] = v1[k] - v0[k]; e2[k] = v2[k] - v0[k]; }
                    cross3(e1, e2, n);
                    real ln = len3(n);
                    if (ln > (real)1e-6f)
                        for (int k = 0; k < 3; k++) cnorm[k] = n[k] / ln;
                }
                if (do_ccd) {
                    real t = ray_tri(prev, rd, v0, v1, v2);
                    if (t > 0 && t < min_t) {
                        min_t = t;
                        has_hit = 1;
                        for (int k = 0; k < 3; k++) hpos[k] = prev[k] + rd[k] * t;
                        real e1[3], e2[3], n[3];
                        for (int k = 0; k < 3; k++) { e1[k] = v1[k] - v0[k]; e2[k] = v2[k] - v0[k]; }
                        cross3(e1, e2, n);
                        real ln = len3(n);
                        real fn[3] = {n[0] / ln, n[1] / ln, n[2] / ln};
                        real sg = sgn(dot3(rd, fn));
                        for (int k = 0; k < 3; k++) hnorm[k] = fn[k] * sg;
                    }
                }
            }
        } else {
            if (sp < 31u) {
                stack[sp++] = nd[3];
                stack[sp++] = nd[7];
            } else {
                __atomic_or_fetch(&ctx->status, OR_STATUS_BVH_STACK, __ATOMIC_RELAXED);
            }
        }
    }
    real vsf = KDIV(s->cvs, s->dt, s->rdt);
    if (has_hit) {
        real sm = s->csurf;
        real ov[3], vr[3], vn, vt[3], nvv[3];
        for (int k = 0; k < 3; k++) p->pos[k] = hpos[k] + hnorm[k] * sm;
        for (int k = 0; k < 3; k++) ov[k] = KDIV(p->dxp[k], s->dt, s->rdt);
        for (int k = 0; k < 3; k++) vr[k] = ov[k] - s->cvel[k];
        vn = dot3(vr, hnorm);
        for (int k = 0; k < 3; k++) vt[k] = vr[k] - vn * hnorm[k];
        real om = (real)1 - s->cfric;
        if (vn < 0) {
            for (int k = 0; k < 3; k++) nvv[k] = vt[k] * om + s->cvel[k] * vsf;
        } else {
            for (int k = 0; k < 3; k++) nvv[k] = vr[k] + s->cvel[k] * vsf;
        }
        for (int k = 0; k < 3; k++) { p->vel[k] = nvv[k]; p->dxp[k] = nvv[k] * s->dt; }
        return;
    }
    real dist = r_sqrt(min_d2);
    real df[3], pd[3] = {cnorm[0], cnorm[1], cnorm[2]};
    for (int k = 0; k < 3; k++) df[k] = cur[k] - cpos[k];
    real ld = len3(df);
    if (ld > (real)1e-6f)
        for (int k = 0; k < 3; k++) pd[k] = df[k] / ld;
    if (dist < s->cthr) {
        real ov[3], vr[3], vn, vt[3], nvv[3];
        for (int k = 0; k < 3; k++) ov[k] = KDIV(p->dxp[k], s->dt, s->rdt);
        for (int k = 0; k < 3; k++) vr[k] = ov[k] - s->cvel[k];
        vn = dot3(vr, pd);
        for (int k = 0; k < 3; k++) vt[k] = vr[k] - vn * pd[k];
        real om = (real)1 - (real)0;
        if (vn < 0) {
            for (int k = 0; k < 3; k++) nvv[k] = vt[k] * om + s->cvel[k] * vsf;
        } else {
            for (int k = 0; k < 3; k++) nvv[k] = vr[k] + s->cvel[k] * vsf;
        }
        for (int k = 0; k < 3; k++) { p->vel[k] = nvv[k]; p->dxp[k] = nvv[k] * s->dt; }
        if (dist < s->csurf)
            for (int k = 0; k < 3; k++) p->pos[k] = cpos[k] + pd[k] * s->csurf;
    }
}

/* integrateParticles (integrateParticles.wgsl:14-72) */
static void integrate(OrCtx* c, const Scene* s, const OrCollider* col, PS* p) {
    for (int k = 0; k < 3; k++) p->pos[k] = p->pos[k] + p->dxp[k];
    real IpD[9];
    for (int i = 0; i < 9; i++) IpD[i] = IDENT[i] + p->D[i];
    mul3(IpD, p->Fe, p->Fe);
    plasticity(s, p->Fe, p->Fp);
    for (int a = 0; a < 3; a++) {
        if (p->pos[a] < s->gmin[a]) {
            p->dxp[a] = p->dxp[a] * s->rest;
            p->pos[a] = s->gmin[a];
            p->vel[a] = p->vel[a] * s->rest;
        }
        if (p->pos[a] >= s->gmax[a]) {
            p->dxp[a] = p->dxp[a] * s->rest;
            p->pos[a] = s->gmax[a];
            p->vel[a] = p->vel[a] * s->rest;
        }
    }
    collide(c, s, col, p);
}

/* ------------------------------------------------------------------ */
/* the substep (GpuMpmPipelineManager.ts:327-428 explicit, :431-521 PBMPM) */
/* ------------------------------------------------------------------ */
static void clear_grid(OrCtx* c) {
    uint32_t nb = c->n_blocks < c->max_blocks ? c->n_blocks : c->max_blocks;
    memset(c->grid, 0, (size_t)nb * 256 * sizeof(*c->grid));
}

int PFX(step)(OrCtx* c, const uint8_t* uni, const OrExt* ext, PART* ps, uint32_t n,
              const OrCollider* col, int method, int stop_after) {
    if (!c || !uni || !ext || (!ps && n)) return -1;
    if (n > c->max_particles) return -2;
    Scene s;
    load_scene(&s, uni, ext);

    /* K1 clearHashMap; K2 mapAffectedBlocks (mapAffectedBlocks.wgsl:64-86) */
    clear_hash(c);
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < n; i++) {
        PS p;
        p_load(&ps[i], &p);
        int32_t cell[3];
        cell_number(&s, p.pos, cell);
        for (int oz = -1; oz <= 1; oz++)
            for (int oy = -1; oy <= 1; oy++)
                for (int ox = -1; ox <= 1; ox++) {
                    int32_t cc[3] = {cell[0] + ox, cell[1] + oy, cell[2] + oz};
                    if (!in_range(&s, cc)) continue;
                    int32_t b[3] = {cc[0] >> 2, cc[1] >> 2, cc[2] >> 2};
                    allocate_block(c, b);
                }
    }
    uint32_t nb = c->n_blocks < c->max_blocks ? c->n_blocks : c->max_blocks;

    /* K3-K6 counting sort by block (clearBlockParticleCounts.wgsl,
     * countParticlesPerBlock.wgsl:9-23, computeBlockOffsets.wgsl:7-15,
     * binParticles.wgsl:10-25).  The sort order only decides the order of the
     * i32 adds, which commute; it is kept to flag unbinned particles. */
    memset(c->counts, 0, nb * sizeof(uint32_t));
    for (uint32_t i = 0; i < n; i++) {
        int32_t cell[3];
        PS p;
        p_load(&ps[i], &p);
        cell_number(&s, p.pos, cell);
        int32_t b[3] = {cell[0] >> 2, cell[1] >> 2, cell[2] >> 2};
        uint32_t bi = lookup_block(c, b);
        if (bi != EMPTY_IDX) c->counts[bi]++;
        else c->status |= OR_STATUS_UNBINNED;
    }
    uint32_t off = 0;
    for (uint32_t b = 0; b < nb; b++) { c->offsets[b] = off; off += c->counts[b]; }

    if (method == 0) {
        clear_grid(c);
#pragma omp parallel for schedule(static)
        for (uint32_t i = 0; i < n; i++) {
            PS p;
            p_load(&ps[i], &p);
            p2g_explicit(c, &s, &p);
        }
        if (stop_after == 1) return 0;
        grid_update_explicit(c, &s);
#pragma omp parallel for schedule(static)
        for (uint32_t i = 0; i < n; i++) {
            PS p;
            p_load(&ps[i], &p);
            g2p(c, &s, &p, 0);
            integrate(c, &s, col, &p);
            p_store(&ps[i], &p);
        }
    } else {
        for (uint32_t it = 0; it < s.n_iter; it++) {
            clear_grid(c);
#pragma omp parallel for schedule(static)
            for (uint32_t i = 0; i < n; i++) {
                PS p;
                p_load(&ps[i], &p);
                pbmpm_constraints(&s, &p);
                p2g_pbmpm(c, &s, &p, 1);
                p_store(&ps[i], &p);
            }
            if (stop_after == 1) return 0;
#pragma omp parallel for schedule(static)
            for (uint32_t i = 0; i < n; i++) {
                PS p;
                p_load(&ps[i], &p);
                g2p(c, &s, &p, 1);
                p_store(&ps[i], &p);
            }
        }
#pragma omp parallel for schedule(static)
        for (uint32_t i = 0; i < n; i++) {
            PS p;
            p_load(&ps[i], &p);
            integrate(c, &s, col, &p);
            p_store(&ps[i], &p);
        }
    }
    return 0;
}

#if OR_FP64
int ord_dense_grid(const OrCtx* c, const uint8_t* uni, double* out)
#else
int orf_dense_grid(const OrCtx* c, const uint8_t* uni, int32_t* out)
#endif
{
    int32_t res[3];
    for (int i = 0; i < 3; i++) res[i] = (int32_t)rdu(uni, 208 + 4 * i);
    size_t total = (size_t)res[0] * res[1] * res[2] * 4;
    memset(out, 0, total * sizeof(*out));
    uint32_t nb = c->n_blocks < c->max_blocks ? c->n_blocks : c->max_blocks;
    for (uint32_t b = 0; b < nb; b++) {
        uint32_t slot = c->mapped[b];
        const int32_t* bn = &c->coord[slot * 3];
        for (uint32_t l = 0; l < 64; l++) {
            int32_t x = bn[0] * 4 + (int32_t)(l & 3), y = bn[1] * 4 + (int32_t)((l >> 2) & 3), z = bn[2] * 4 + (int32_t)(l >> 4);
            if (x < 0 || y < 0 || z < 0 || x >= res[0] || y >= res[1] || z >= res[2]) continue;
            size_t o = (((size_t)z * res[1] + y) * res[0] + x) * 4;
            for (int k = 0; k < 4; k++) out[o + k] = (__typeof__(*out))c->grid[((size_t)b * 64 + l) * 4 + k];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* known-answer hooks                                                  */
/* ------------------------------------------------------------------ */
#if !OR_FP64
void orf_inverse(const float* m, float* o) { inv3(m, o); }
void orf_polar(const float* m, float* o) { polar3(m, o); }
float orf_det(const float* m) { return det3(m); }
void orf_plasticity(const OrExt* ext, float* Fe, float* Fp) {
    uint8_t uni[OR_UNIFORMS_BYTES];
    memset(uni, 0, sizeof(uni));
    Scene s;
    load_scene(&s, uni, ext);
    plasticity(&s, Fe, Fp);
}
#endif

/* the selected return map on n states (f32: orf_, f64: ord_) */
void PFX(plasticity_n)(const OrExt* ext, real* Fe, real* Fp, uint32_t n) {
    uint8_t uni[OR_UNIFORMS_BYTES];
    memset(uni, 0, sizeof(uni));
    Scene s;
    load_scene(&s, uni, ext);
    for (uint32_t i = 0; i < n; i++) plasticity(&s, Fe + 9 * (size_t)i, Fp + 9 * (size_t)i);
}
