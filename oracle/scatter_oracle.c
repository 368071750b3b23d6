/*
 * scatter_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of scatterParticles
 * (luoluobuli/WebGPU-MPM-based-Snow-Simulation,
 * src/lib/gpu/particleInitialize/particleScatter.cs.wgsl:7-84), with the
 * hashes and fBm of src/lib/gpu/shaderPrelude/randomNumberGenerators.wgsl:3-94
 * and the Moller-Trumbore test of src/lib/gpu/shaderPrelude/triangleOps.wgsl.
 * Sequential loop over triangles per candidate, exactly as the shader.
 * f32 arithmetic; dot and cross in the step's canonical fused order
 * (fmaf), mix(a, b, t) = a (1 - t) + b t unfused, fract(x) = x - floor(x),
 * IEEE division; built with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

static uint32_t h1(uint32_t n) {
    uint32_t h = n + 374761393u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h = 2246822519u * (h ^ (h >> 15));
    h = 3266489917u * (h ^ (h >> 13));
    return h ^ (h >> 16);
}
static uint32_t h3(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t h = z + 374761393u + x * 3266489917u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h += y * 3266489917u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h = 2246822519u * (h ^ (h >> 15));
    h = 3266489917u * (h ^ (h >> 13));
    return h ^ (h >> 16);
}
static uint32_t h4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
    uint32_t h = w + 374761393u + x * 3266489917u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h += y * 3266489917u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h += z * 3266489917u;
    h = 668265263u * ((h << 17) | (h >> 15));
    h = 2246822519u * (h ^ (h >> 15));
    h = 3266489917u * (h ^ (h >> 13));
    return h ^ (h >> 16);
}
static float unit(uint32_t h) { return (float)h / 4294967296.0f; }
static float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static float dot3f(const float* a, const float* b) { return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0])); }
static void cross3f(const float* a, const float* b, float* o) {
    float x = fmaf(a[1], b[2], -(a[2] * b[1]));
    float y = fmaf(a[2], b[0], -(a[0] * b[2]));
    float z = fmaf(a[0], b[1], -(a[1] * b[0]));
    o[0] = x; o[1] = y; o[2] = z;
}

static int ray_x_hits(const float* o, const float* v0, const float* v1, const float* v2) {
    const float eps = 1e-6f, dir[3] = {1.0f, 0.0f, 0.0f};
    float e1[3] = {v1[0] - v0[0], v1[1] - v0[1], v1[2] - v0[2]};
    float e2[3] = {v2[0] - v0[0], v2[1] - v0[1], v2[2] - v0[2]};
    float rce2[3];
    cross3f(dir, e2, rce2);
    float det = dot3f(e1, rce2);
    if (fabsf(det) < eps) return 0;
    float inv = 1.0f / det;
    float ov[3] = {o[0] - v0[0], o[1] - v0[1], o[2] - v0[2]};
    float b0 = dot3f(ov, rce2) * inv;
    if (b0 < 0.0f || 1.0f < b0) return 0;
    float ove1[3];
    cross3f(ov, e1, ove1);
    float b1 = dot3f(dir, ove1) * inv;
    if (b1 < 0.0f || 1.0f < b1 || b0 + b1 > 1.0f) return 0;
    return dot3f(e2, ove1) * inv > eps;
}

static float noise3(const float* x) {
    float f[3], u[3];
    uint32_t n[3];
    for (int k = 0; k < 3; k++) {
        float p = floorf(x[k]);
        f[k] = x[k] - p;
        u[k] = (f[k] * f[k]) * (3.0f - 2.0f * f[k]);
        n[k] = (uint32_t)(int32_t)p;
    }
    float c[8];
    for (int i = 0; i < 8; i++) c[i] = unit(h3(n[0] + (i & 1), n[1] + ((i >> 1) & 1), n[2] + (i >> 2)));
    return mixf(mixf(mixf(c[0], c[1], u[0]), mixf(c[2], c[3], u[0]), u[1]),
                mixf(mixf(c[4], c[5], u[0]), mixf(c[6], c[7], u[0]), u[1]), u[2]);
}
static float fbm(const float* x0) {
    float v = 0.0f, a = 0.5f, p[3] = {x0[0], x0[1], x0[2]};
    for (int i = 0; i < 6; i++) {
        v = v + a * noise3(p);
        for (int k = 0; k < 3; k++) p[k] = p[k] * 2.0f;
        a = a * 0.5f;
    }
    return v;
}

/* verts: n_tris * 3 vertices of 4 floats; out: n 192-byte records */
void or_scatter(const float* verts, uint32_t n_tris, const float* mmin, const float* mmax, uint32_t n, uint8_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        uint32_t seed = h4(i, 100u, 200u, 300u);
        float cand[3] = {0, 0, 0};
        for (uint32_t attempt = 0; attempt < 512u; attempt++) {
            for (int k = 0; k < 3; k++) {
                seed = h1(seed);
                cand[k] = mixf(mmin[k], mmax[k], unit(seed));
            }
            int inside = 0;
            for (uint32_t t = 0; t < n_tris; t++)
                if (ray_x_hits(cand, verts + (size_t)t * 12, verts + (size_t)t * 12 + 4, verts + (size_t)t * 12 + 8))
                    inside = !inside;
            if (inside) break;
        }
        float x[3] = {cand[0] * 4.0f, cand[1] * 4.0f, cand[2] * 4.0f};
        float xa[3] = {x[0] + 100.0f, x[1] + 200.0f, x[2] + 300.0f};
        float xb[3] = {x[0] + -300.0f, x[1] + -200.0f, x[2] + -100.0f};
        float d[3] = {fbm(x), fbm(xa), fbm(xb)};
        float* r = (float*)(out + (size_t)i * 192u);
        memset(r, 0, 192);
        for (int k = 0; k < 3; k++) r[k] = cand[k] + (d[k] - 0.5f) * 0.1f;
        r[3] = 1.0f;
        float m1 = unit(h1(i));
        r[7] = m1 * m1;
        r[8] = 1.0f; r[13] = 1.0f; r[18] = 1.0f;    /* F_e = I (columns of 4 words) */
        r[20] = 1.0f; r[25] = 1.0f; r[30] = 1.0f;   /* F_p = I */
    }
}
