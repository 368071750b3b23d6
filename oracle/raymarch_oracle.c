/*
 * raymarch_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the volumetric renderer's ray march
 * (luoluobuli/WebGPU-MPM-based-Snow-Simulation,
 * src/lib/gpu/volumetric/volumetricRaymarch.cs.wgsl:16-226; calculateViewRay,
 * src/lib/gpu/shaderPrelude/cameraOps.wgsl:6-19; PI, shaderPrelude/constants.wgsl:1).
 * f32 arithmetic in the WGSL expression order, no contraction (the Makefile
 * builds with -ffp-contract=off); exp and pow are the oracle's f64 routines
 * rounded once (or_expf, or_powf); matrix-vector products sum the columns in
 * order; normalize divides by the square root of the ordered dot product;
 * f32 -> u32 truncates and saturates; the rgba8unorm store rounds to nearest
 * even.  One call renders the whole image; rows run in parallel (OpenMP).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "mpm_oracle.h"

#define RM_EXTINCTION 724.0f
#define RM_STEP 0.025f
#define RM_N_STEPS 256u
#define RM_N_SHADOW 64u

static const float RM_ALBEDO[3] = {0.9f, 0.985f, 0.99f};
static const float RM_FOUR_PI = (float)(4.0 * 3.1415926);
static const float RM_INV_GAMMA = (float)(1.0 / 2.2);

static uint32_t f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

/* hash4 (randomNumberGenerators.wgsl:40-55) */
static uint32_t rm_hash4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
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

static uint32_t f2bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

typedef struct {
    const uint32_t* mass;
    uint32_t res[3];
    float gmin[3], gmax[3], cell[3], volume, scale;
} rm_field;

/* readDensity (:16-57) */
static float read_density(const rm_field* F, const float* p) {
    for (int k = 0; k < 3; k++)
        if (p[k] < F->gmin[k] || p[k] >= F->gmax[k]) return 0.0f;
    uint32_t start[3];
    float w[2][3];
    for (int k = 0; k < 3; k++) {
        float gp = (p[k] - F->gmin[k]) / F->cell[k];
        float sp = gp - 0.5f;
        start[k] = f2u_sat(sp);
        float f = sp - (float)start[k];
        w[0][k] = 1.0f - f;
        w[1][k] = f;
    }
    float mass = 0.0f;
    for (int z = 0; z < 2; z++)
        for (int y = 0; y < 2; y++)
            for (int x = 0; x < 2; x++) {
                int32_t cx = (int32_t)(start[0] + x), cy = (int32_t)(start[1] + y), cz = (int32_t)(start[2] + z);
                if (cx < 0 || cy < 0 || cz < 0 || cx >= (int32_t)F->res[0] || cy >= (int32_t)F->res[1] ||
                    cz >= (int32_t)F->res[2])
                    continue;
                uint32_t idx = (uint32_t)cx + F->res[0] * ((uint32_t)cy + F->res[1] * (uint32_t)cz);
                float val = (float)F->mass[idx] / F->scale;
                float weight = (w[x][0] * w[y][1]) * w[z][2];
                mass = mass + val * weight;
            }
    return (mass / F->volume) * 0.00001f;
}

/* henyeyGreenstein (:59-63) */
static float hg(float c, float g) {
    float g2 = g * g;
    float denom = (1.0f + g2) - (2.0f * g) * c;
    return (1.0f - g2) / (RM_FOUR_PI * or_powf(denom, 1.5f));
}

/* raymarchShadow (:94-108) */
static void shadow(const rm_field* F, const float* pos, const float* ld, uint32_t time, float* T) {
    uint32_t h = rm_hash4(f2bits(pos[0]), f2bits(pos[1]), f2bits(pos[2]), time);
    float jitter = (float)h / 4294967296.0f;
    float sp[3], st[3];
    for (int k = 0; k < 3; k++) {
        st[k] = ld[k] * RM_STEP;
        sp[k] = pos[k] + st[k] * jitter;
        T[k] = 1.0f;
    }
    for (uint32_t s = 0; s < RM_N_SHADOW; s++) {
        for (int k = 0; k < 3; k++) sp[k] = sp[k] + st[k];
        float d = read_density(F, sp);
        if (d > 1e-4f) {
            float a = (-(RM_EXTINCTION * d)) * RM_STEP;
            for (int k = 0; k < 3; k++) T[k] = T[k] * or_expf(a * RM_ALBEDO[k]);
            if (T[0] < 1e-4f && T[1] < 1e-4f && T[2] < 1e-4f) break;
        }
    }
}

static void unproject(const float* M, float x, float y, float z, float* o) {
    float h[4];
    for (int r = 0; r < 4; r++) h[r] = ((M[r] * x + M[4 + r] * y) + M[8 + r] * z) + M[12 + r] * 1.0f;
    for (int k = 0; k < 3; k++) o[k] = h[k] / h[3];
}

static float dot3s(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

static void normalize3(float* v) {
    float l = sqrtf(dot3s(v, v));
    for (int k = 0; k < 3; k++) v[k] = v[k] / l;
}

static uint8_t unorm8(float v) {
    float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)nearbyintf(c * 255.0f);
}

/* doVolumetricRaymarch (:118-226) over the whole image.  Outputs: rgba
 * [h][w][4] u8, depth [h][w] f32 (left as given where the ray misses the grid),
 * color [h][w][4] f32 (optional). */
void or_raymarch(const uint32_t* mass, const uint32_t* res, const float* gmin, const float* gmax, float scale,
                 const float* inv_vp, uint32_t time, uint32_t width, uint32_t height, uint8_t* rgba, float* depth_out,
                 float* color) {
    rm_field F;
    F.mass = mass;
    for (int k = 0; k < 3; k++) {
        F.res[k] = res[k];
        F.gmin[k] = gmin[k];
        F.gmax[k] = gmax[k];
        F.cell[k] = (gmax[k] - gmin[k]) / (float)res[k];
    }
    F.volume = (F.cell[0] * F.cell[1]) * F.cell[2];
    F.scale = scale;
#pragma omp parallel for schedule(dynamic, 1)
    for (uint32_t gy = 0; gy < height; gy++) {
        for (uint32_t gx = 0; gx < width; gx++) {
            size_t pix = (size_t)gy * width + gx;
            float u = (float)gx / (float)width, v = (float)gy / (float)height;
            float ux = u * 2.0f - 1.0f, uy = (1.0f - v) * 2.0f - 1.0f;
            float org[3], far_p[3], dir[3];
            unproject(inv_vp, ux, uy, 0.0f, org);
            unproject(inv_vp, ux, uy, 1.0f, far_p);
            for (int k = 0; k < 3; k++) dir[k] = far_p[k] - org[k];
            normalize3(dir);
            float ld[3] = {0.2f, 0.18f, 0.9f};
            normalize3(ld);
            const float lc[3] = {0.95f * 5.0f, 0.995f * 5.0f, 1.0f * 5.0f};
            const float amb[3] = {0.0f, 0.1f, 0.2f};

            float t1[3], t2[3];
            for (int k = 0; k < 3; k++) {
                float dmin = (gmin[k] - org[k]) / dir[k];
                float dmax = (gmax[k] - org[k]) / dir[k];
                t1[k] = fminf(dmin, dmax);
                t2[k] = fmaxf(dmin, dmax);
            }
            float t_near = fmaxf(fmaxf(t1[0], t1[1]), t1[2]);
            float t_far = fminf(fminf(t2[0], t2[1]), t2[2]);

            float d_ground = 1e20f;
            int hit_ground = 0;
            if (fabsf(dir[2]) > 1e-4f) {
                float cand = (gmin[2] - org[2]) / dir[2];
                if (cand > 0.0f) {
                    float hx = org[0] + cand * dir[0], hy = org[1] + cand * dir[1];
                    if (hx >= gmin[0] && hy >= gmin[1] && hx <= gmax[0] && hy <= gmax[1]) {
                        d_ground = cand;
                        hit_ground = 1;
                    }
                }
            }
            if (!(t_near <= t_far && t_far >= 0.0f)) {
                memset(rgba + pix * 4, 0, 4);
                if (color) memset(color + pix * 4, 0, 16);
                continue;
            }
            float d_start = fmaxf(0.0f, t_near);
            float d_end = fminf(t_far, d_ground);
            float jitter = (float)or_hash3(gx, gy, time) / 4294967296.0f;
            float cur = d_start + jitter * RM_STEP;
            float T[3] = {1.0f, 1.0f, 1.0f}, col[3] = {0.0f, 0.0f, 0.0f};
            int depth_written = 0;
            float depth = 1e20f;
            float phase = hg(dot3s(dir, ld), -0.5f) + hg(dot3s(dir, ld), 0.5f);
            for (uint32_t i = 0; i < RM_N_STEPS; i++) {
                if (cur >= d_end || (T[0] < 0.01f && T[1] < 0.01f && T[2] < 0.01f)) break;
                float pos[3];
                for (int k = 0; k < 3; k++) pos[k] = org[k] + cur * dir[k];
                float density = read_density(&F, pos);
                if (density > 0.001f) {
                    if (!depth_written) {
                        depth = cur;
                        depth_written = 1;
                    }
                    float ext = RM_EXTINCTION * density;
                    float a_ext = (-ext) * RM_STEP;
                    float sh[3];
                    shadow(&F, pos, ld, time, sh);
                    float mext = fmaxf(ext, 1e-4f);
                    for (int k = 0; k < 3; k++) {
                        float scat = ext * RM_ALBEDO[k];
                        float stT = or_expf(a_ext * RM_ALBEDO[k]);
                        float light = amb[k] + (lc[k] * phase) * sh[k];
                        float laf = ((light * scat) * (1.0f - stT)) / mext;
                        col[k] = col[k] + T[k] * laf;
                        T[k] = T[k] * stT;
                    }
                }
                cur = cur + RM_STEP;
            }
            if (hit_ground && (T[0] > 0.01f || T[1] > 0.01f || T[2] > 0.01f)) {
                float pos[3], sh[3];
                for (int k = 0; k < 3; k++) pos[k] = org[k] + d_ground * dir[k];
                shadow(&F, pos, ld, time, sh);
                float lz = fmaxf(0.0f, ld[2]);
                for (int k = 0; k < 3; k++) {
                    float gcol = amb[k] + 0.05f * ((lc[k] * sh[k]) * lz);
                    col[k] = col[k] + T[k] * gcol;
                    T[k] = 0.0f;
                }
                if (!depth_written) depth = d_ground;
            }
            float alpha = 1.0f - fmaxf(T[0], fmaxf(T[1], T[2]));
            float o[4] = {or_powf(col[0], RM_INV_GAMMA) * alpha, or_powf(col[1], RM_INV_GAMMA) * alpha,
                          or_powf(col[2], RM_INV_GAMMA) * alpha, 1.0f * alpha};
            for (int k = 0; k < 4; k++) rgba[pix * 4 + k] = unorm8(o[k]);
            if (color) memcpy(color + pix * 4, o, 16);
            depth_out[pix] = depth;
        }
    }
}
