/*
 * mlp_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU reference of the learned-plasticity network of libmpm (12 -> 64 -> 64
 * -> 64 -> 11, SiLU) and of the pieces around it.  The reference
 * (luoluobuli/WebGPU-MPM-based-Snow-Simulation) has no learned model: its
 * plasticity is always the exact return map applyPlasticity
 * (src/lib/gpu/shaderPrelude/plasticityOps.wgsl:7-48, restated in
 * mpm_oracle.c), which generates the training targets.  This file is the
 * CPU reference of the GPU network's forward pass, its gradients and its strain-
 * bound check; only the tests load it.
 *
 * Two arithmetic modes:
 *   bf16 = 1  rounds weights, activations and output-gradients to BF16
 *             (round to nearest even) at the points where the tensor-core
 *             kernels round them, and accumulates in f64: the GPU's
 *             FP32-accumulated results agree to accumulation-order error;
 *   bf16 = 0  plain f64 throughout: the function whose gradient a finite
 *             difference checks.
 * Loss of a batch of B pairs: (1/B) sum_b [ sum_{i<10} (y_i - t_i)^2
 *   + w (y_10 - e_b)^2 ], e_b = |y[0..9] - t| held constant.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mpm_oracle.h"

#define IN 12
#define HID 64
#define OUT 11
#define OW1 0
#define OB1 (OW1 + HID * IN)
#define OW2 (OB1 + HID)
#define OB2 (OW2 + HID * HID)
#define OW3 (OB2 + HID)
#define OB3 (OW3 + HID * HID)
#define OW4 (OB3 + HID)
#define OB4 (OW4 + OUT * HID)
#define NPARAM (OB4 + OUT)

static float bf16r(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&x, &u, 4);
    return x;
}

static double rnd(double v, int bf16) { return bf16 ? (double)bf16r((float)v) : v; }
static double silu_d(double z) { return z / (1.0 + exp(-z)); }
static double silu_grad_d(double z) {
    double s = 1.0 / (1.0 + exp(-z));
    return s + z * s * (1.0 - s);
}

typedef struct Fwd {
    double a0[IN], z1[HID], a1[HID], z2[HID], a2[HID], z3[HID], a3[HID], y[OUT];
} Fwd;

static void forward1(const float* P, const float* x, int bf16, Fwd* f) {
    for (int k = 0; k < IN; k++) f->a0[k] = rnd(x[k], bf16);
    for (int o = 0; o < HID; o++) {
        double s = 0.0;
        for (int k = 0; k < IN; k++) s += rnd(P[OW1 + o * IN + k], bf16) * f->a0[k];
        f->z1[o] = s + P[OB1 + o];
        f->a1[o] = rnd(silu_d(f->z1[o]), bf16);
    }
    for (int o = 0; o < HID; o++) {
        double s = 0.0;
        for (int k = 0; k < HID; k++) s += rnd(P[OW2 + o * HID + k], bf16) * f->a1[k];
        f->z2[o] = s + P[OB2 + o];
        f->a2[o] = rnd(silu_d(f->z2[o]), bf16);
    }
    for (int o = 0; o < HID; o++) {
        double s = 0.0;
        for (int k = 0; k < HID; k++) s += rnd(P[OW3 + o * HID + k], bf16) * f->a2[k];
        f->z3[o] = s + P[OB3 + o];
        f->a3[o] = rnd(silu_d(f->z3[o]), bf16);
    }
    for (int o = 0; o < OUT; o++) {
        double s = 0.0;
        for (int k = 0; k < HID; k++) s += rnd(P[OW4 + o * HID + k], bf16) * f->a3[k];
        f->y[o] = s + P[OB4 + o];
    }
}

/* y: n x 11 */
void or_mlp_forward(const float* P, const float* x, uint32_t n, int bf16, double* y) {
    for (uint32_t b = 0; b < n; b++) {
        Fwd f;
        forward1(P, x + (size_t)b * IN, bf16, &f);
        for (int o = 0; o < OUT; o++) y[(size_t)b * OUT + o] = f.y[o];
    }
}

/* loss and gradient (NPARAM doubles) of the batch loss */
double or_mlp_gradient(const float* P, const float* x, const float* t, uint32_t n, float unc_weight, int bf16,
                       double* grad) {
    memset(grad, 0, sizeof(double) * NPARAM);
    double loss = 0.0, ib = 1.0 / (double)n;
    for (uint32_t b = 0; b < n; b++) {
        Fwd f;
        forward1(P, x + (size_t)b * IN, bf16, &f);
        const float* tb = t + (size_t)b * 10;
        double se = 0.0, g4[OUT];
        for (int i = 0; i < 10; i++) se += (f.y[i] - tb[i]) * (f.y[i] - tb[i]);
        double e = sqrt(se);
        for (int i = 0; i < 10; i++) g4[i] = 2.0 * ib * (f.y[i] - tb[i]);
        g4[10] = 2.0 * ib * unc_weight * (f.y[10] - e);
        loss += ib * (se + unc_weight * (f.y[10] - e) * (f.y[10] - e));
        double g4r[OUT];
        for (int o = 0; o < OUT; o++) {
            g4r[o] = rnd(g4[o], bf16);
            grad[OB4 + o] += g4[o];
            for (int k = 0; k < HID; k++) grad[OW4 + o * HID + k] += g4r[o] * f.a3[k];
        }
        double g3[HID], g3r[HID];
        for (int k = 0; k < HID; k++) {
            double dx = 0.0;
            for (int o = 0; o < OUT; o++) dx += g4r[o] * rnd(P[OW4 + o * HID + k], bf16);
            g3[k] = dx * silu_grad_d(f.z3[k]);
            g3r[k] = rnd(g3[k], bf16);
        }
        for (int o = 0; o < HID; o++) {
            grad[OB3 + o] += g3[o];
            for (int k = 0; k < HID; k++) grad[OW3 + o * HID + k] += g3r[o] * f.a2[k];
        }
        double g2[HID], g2r[HID];
        for (int k = 0; k < HID; k++) {
            double dx = 0.0;
            for (int o = 0; o < HID; o++) dx += g3r[o] * rnd(P[OW3 + o * HID + k], bf16);
            g2[k] = dx * silu_grad_d(f.z2[k]);
            g2r[k] = rnd(g2[k], bf16);
        }
        for (int o = 0; o < HID; o++) {
            grad[OB2 + o] += g2[o];
            for (int k = 0; k < HID; k++) grad[OW2 + o * HID + k] += g2r[o] * f.a1[k];
        }
        double g1[HID], g1r[HID];
        for (int k = 0; k < HID; k++) {
            double dx = 0.0;
            for (int o = 0; o < HID; o++) dx += g2r[o] * rnd(P[OW2 + o * HID + k], bf16);
            g1[k] = dx * silu_grad_d(f.z1[k]);
            g1r[k] = rnd(g1[k], bf16);
        }
        for (int o = 0; o < HID; o++) {
            grad[OB1 + o] += g1[o];
            for (int k = 0; k < IN; k++) grad[OW1 + o * IN + k] += g1r[o] * f.a0[k];
        }
    }
    return loss;
}

/* network inputs of a trial state (same formulas as mpm_plast.cuh
 * mlp_features); returns 0 outside the trained domain */
int or_mlp_features(const float* Fe, const float* Fp, float dt, float theta_c, float* x) {
    int ok = 1;
    for (int i = 0; i < 9; i++) {
        float d = Fe[i] - ((i == 0 || i == 4 || i == 8) ? 1.0f : 0.0f);
        if (fabsf(d) > 0.25f) ok = 0;
        x[i] = d * 20.0f;
    }
    float jp = orf_det(Fp);
    if (!(jp >= 0.0625f && jp <= 16.0f)) ok = 0;
    x[9] = ok ? logf(jp) * 2.0f : 0.0f;
    x[10] = log2f(dt) + 13.2877f;
    x[11] = (theta_c - 0.025f) * 100.0f;
    return ok;
}

/* targets of an exact result */
void or_mlp_targets(const float* Fe, const float* Fp, const float* Fe2, const float* Fp2, float* t) {
    for (int i = 0; i < 9; i++) t[i] = (Fe2[i] - Fe[i]) * 100.0f;
    t[9] = (logf(orf_det(Fp2)) - logf(orf_det(Fp))) * 100.0f;
}

/* strain-bound check (same operation order as mpm_plast.cuh cert_elastic) */
static float dot3f(const float* a, const float* b) { return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0])); }
int or_cert_elastic(float smin, float smax, const float* Fe) {
    float c00 = dot3f(Fe, Fe), c11 = dot3f(Fe + 3, Fe + 3), c22 = dot3f(Fe + 6, Fe + 6);
    float c01 = fabsf(dot3f(Fe, Fe + 3)), c02 = fabsf(dot3f(Fe, Fe + 6)), c12 = fabsf(dot3f(Fe + 3, Fe + 6));
    float lo = fminf(fminf((c00 - c01) - c02, (c11 - c01) - c12), (c22 - c02) - c12);
    float hi = fmaxf(fmaxf((c00 + c01) + c02, (c11 + c01) + c12), (c22 + c02) + c12);
    float a = smin + 1e-4f, b = smax - 1e-4f;
    return lo >= a * a && hi <= b * b;
}
