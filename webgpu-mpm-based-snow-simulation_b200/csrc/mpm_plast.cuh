// mpm_plast.cuh -- the snow plasticity return map and the pieces of its
// learned surrogate that sit around the network.
//
// plasticity_exact is applyPlasticity (plasticityOps.wgsl:7-48): R = polar(Fe),
// S = R^T Fe, sigma = diag(S); if every sigma lies in [1 - theta_c, 1 + theta_s]
// nothing changes, else Fe' = R diag(clamp(sigma)), Fp' = Fe'^-1 (Fe Fp).
//
// cert_elastic is the strain-bound check of the learned form: a cheap
// sufficient condition for the early return above.  C = Fe^T Fe has the
// eigenvalues sigma_k^2 of the stretch U = sqrt(C); every diagonal entry of
// the symmetric positive U lies between its extreme eigenvalues, and S equals
// U up to the rounding of the four polar averaging steps (which converge
// quadratically: for stretches within 25 % the residual is below 1e-7).  So if
// every Gershgorin disc of C lies inside [(smin + m)^2, (smax - m)^2] with the
// margin m = 1e-4, applyPlasticity returns Fe and Fp unchanged, bit for bit.
//
// The network's features and targets (learned plasticity, 12 -> 64 -> 64 ->
// 64 -> 11, SiLU): x[0..8] = (Fe_trial - I) * 20 (column-major as stored),
// x[9] = 2 ln det Fp, x[10] = log2(dt) + 13.2877 (0 at dt = 1e-4),
// x[11] = (theta_c - 0.025) * 100; targets t[0..8] = (Fe' - Fe_trial) * 100,
// t[9] = (ln det Fp' - ln det Fp) * 100; output 10 is the uncertainty head,
// trained to predict the error norm |y[0..9] - t| of the other outputs.
#pragma once
#include "mpm_math.cuh"

namespace mpm {

constexpr float CERT_MARGIN = 1e-4f;
constexpr float MLP_X_F = 20.0f, MLP_X_J = 2.0f, MLP_X_DT = 13.2877f, MLP_X_TC0 = 0.025f, MLP_X_TC = 100.0f;
constexpr float MLP_T_F = 100.0f, MLP_T_FINV = 0.01f;
constexpr float MLP_DOMAIN = 0.25f;   // max |Fe_trial - I| entry the network is asked about

__device__ __forceinline__ void plasticity_exact(float smin, float smax, float* Fe, float* Fp) {
    float R[9], Rt[9], Sm[9];
    polar3(Fe, R);
    tr3(R, Rt);
    mul3(Rt, Fe, Sm);
    float sg0 = Sm[0], sg1 = Sm[4], sg2 = Sm[8];
    if (smin <= sg0 && smin <= sg1 && smin <= sg2 && sg0 <= smax && sg1 <= smax && sg2 <= smax) return;
    float c0 = fminf(fmaxf(sg0, smin), smax);
    float c1 = fminf(fmaxf(sg1, smin), smax);
    float c2 = fminf(fmaxf(sg2, smin), smax);
    float Dg[9] = {c0, 0.f, 0.f, 0.f, c1, 0.f, 0.f, 0.f, c2};
    float Fn[9], Fni[9], F[9];
    mul3(R, Dg, Fn);
    inv3(Fn, Fni);
    mul3(Fe, Fp, F);
    mul3(Fni, F, Fp);
#pragma unroll
    for (int i = 0; i < 9; i++) Fe[i] = Fn[i];
}

// The SVD return map (return_map 1): an option of this library, not the
// reference's map.  One-sided Jacobi SVD (M. R. Hestenes, "Inversion of
// matrices by biorthogonalization and related results", J. SIAM 6, 1958): the
// column pairs (0,1), (0,2), (1,2) of A = Fe are rotated, SVD_SWEEPS sweeps,
// until A V = U diag(sigma) with sigma_k = |a_k|.  If every sigma lies in
// [smin, smax] nothing changes, else Fe' = sum_k (clamp(sigma_k) / sigma_k)
// a_k v_k^T and Fp' = Fe'^-1 (Fe Fp).  The oracle's plasticity_svd performs
// the same operations.  cert_elastic certifies this map too: it bounds the
// singular values themselves.
constexpr int SVD_SWEEPS = 4;
__device__ __forceinline__ void jrot(float* x, float* y, float c, float sn) {
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const float xr = x[r], yr = y[r];
        x[r] = fs(fm(c, xr), fm(sn, yr));
        y[r] = fa(fm(sn, xr), fm(c, yr));
    }
}

static __device__ __noinline__ void plasticity_svd(float smin, float smax, float* Fe, float* Fp) {
    float a[9], v[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
#pragma unroll
    for (int i = 0; i < 9; i++) a[i] = Fe[i];
#pragma unroll 1
    for (int sw = 0; sw < SVD_SWEEPS; sw++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int p = k == 2 ? 1 : 0, q = k == 0 ? 1 : 2;
            float* ap = a + 3 * p;
            float* aq = a + 3 * q;
            const float al = dot3(ap, ap), be = dot3(aq, aq), ga = dot3(ap, aq);
            if (ga == 0.f) continue;
            const float ze = fd(fs(be, al), fm(2.f, ga));
            const float t = fd(copysignf(1.f, ze), fa(fabsf(ze), __fsqrt_rn(ff(ze, ze, 1.f))));
            const float c = fd(1.f, __fsqrt_rn(ff(t, t, 1.f)));
            const float sn = fm(c, t);
            jrot(ap, aq, c, sn);
            jrot(v + 3 * p, v + 3 * q, c, sn);
        }
    float sg[3];
#pragma unroll
    for (int k = 0; k < 3; k++) sg[k] = __fsqrt_rn(dot3(a + 3 * k, a + 3 * k));
    if (smin <= sg[0] && smin <= sg[1] && smin <= sg[2] && sg[0] <= smax && sg[1] <= smax && sg[2] <= smax) return;
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; k++) w[k] = sg[k] > 0.f ? fd(fminf(fmaxf(sg[k], smin), smax), sg[k]) : 1.f;
    float Fn[9], Fni[9], F[9];
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int r = 0; r < 3; r++)
            Fn[3 * j + r] = ff(fm(w[2], a[6 + r]), v[6 + j], ff(fm(w[1], a[3 + r]), v[3 + j], fm(fm(w[0], a[r]), v[j])));
    inv3(Fn, Fni);
    mul3(Fe, Fp, F);
    mul3(Fni, F, Fp);
#pragma unroll
    for (int i = 0; i < 9; i++) Fe[i] = Fn[i];
}

// The return map a scene selects (MpmParams::return_map).
__device__ __forceinline__ void plasticity_map(uint32_t rmap, float smin, float smax, float* Fe, float* Fp) {
    if (rmap == 1u) plasticity_svd(smin, smax, Fe, Fp);
    else plasticity_exact(smin, smax, Fe, Fp);
}

__device__ __forceinline__ bool cert_elastic(float smin, float smax, const float* Fe) {
    // C[i][j] = dot(column i, column j)
    float c00 = dot3(Fe, Fe), c11 = dot3(Fe + 3, Fe + 3), c22 = dot3(Fe + 6, Fe + 6);
    float c01 = fabsf(dot3(Fe, Fe + 3)), c02 = fabsf(dot3(Fe, Fe + 6)), c12 = fabsf(dot3(Fe + 3, Fe + 6));
    float lo = fminf(fminf(fs(fs(c00, c01), c02), fs(fs(c11, c01), c12)), fs(fs(c22, c02), c12));
    float hi = fmaxf(fmaxf(fa(fa(c00, c01), c02), fa(fa(c11, c01), c12)), fa(fa(c22, c02), c12));
    float a = fa(smin, CERT_MARGIN), b = fs(smax, CERT_MARGIN);
    return lo >= fm(a, a) && hi <= fm(b, b);
}

// Network input of one trial state; returns false outside the trained domain.
__device__ __forceinline__ bool mlp_features(const float* Fe, const float* Fp, float dt, float theta_c, float* x) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        float d = Fe[i] - ((i == 0 || i == 4 || i == 8) ? 1.0f : 0.0f);
        ok = ok && fabsf(d) <= MLP_DOMAIN;
        x[i] = d * MLP_X_F;
    }
    float jp = det3(Fp);
    ok = ok && jp >= 0.0625f && jp <= 16.0f;
    x[9] = ok ? logf(jp) * MLP_X_J : 0.0f;
    x[10] = log2f(dt) + MLP_X_DT;
    x[11] = (theta_c - MLP_X_TC0) * MLP_X_TC;
    return ok;
}

}  // namespace mpm
