/*
 * splat_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the particle splats the reference's renderers run
 * (luoluobuli/WebGPU-MPM-based-Snow-Simulation):
 *   or_grid_mass   calculateGridMass, src/lib/gpu/volumetric/calculateGridMass.wgsl:8-51
 *   or_mc_density  calculateDensity,  src/lib/gpu/marchingCubes/mcDensity.cs.wgsl:14-63
 * f32 arithmetic in the WGSL expression order, no contraction (the Makefile
 * builds with -ffp-contract=off); f32 -> u32 / i32 truncating and saturating.
 * Particles are the 192-byte records (pos at word 0..2, mass at word 7).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

static uint32_t f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;            /* NaN and negatives */
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
static int32_t f2i_sat(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x < -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}

static void load(const uint8_t* recs, uint32_t i, float* pos, float* mass) {
    const float* r = (const float*)(recs + (size_t)i * 192u);
    pos[0] = r[0]; pos[1] = r[1]; pos[2] = r[2];
    *mass = r[7];
}

void or_grid_mass(const uint8_t* recs, uint32_t n, const float* gmin, const float* gmax, const uint32_t* res,
                  float scale, uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        float pos[3], mass;
        load(recs, i, pos, &mass);
        int outside = 0;
        for (int k = 0; k < 3; k++) outside |= (pos[k] < gmin[k]) || (pos[k] >= gmax[k]);
        if (outside) continue;
        uint32_t start[3];
        float w[2][3];
        for (int k = 0; k < 3; k++) {
            float cell_size = (gmax[k] - gmin[k]) / (float)res[k];
            float pc = (pos[k] - gmin[k]) / cell_size;
            float center = pc - 0.5f;
            start[k] = f2u_sat(center);
            float f = center - (float)start[k];
            w[0][k] = 1.0f - f;
            w[1][k] = f;
        }
        for (int z = 0; z < 2; z++)
            for (int y = 0; y < 2; y++)
                for (int x = 0; x < 2; x++) {
                    uint32_t cx = start[0] + x, cy = start[1] + y, cz = start[2] + z;
                    if (cx >= res[0] || cy >= res[1] || cz >= res[2]) continue;
                    float weight = (w[x][0] * w[y][1]) * w[z][2];
                    out[cx + res[0] * (cy + res[1] * cz)] += f2u_sat((mass * weight) * scale);
                }
    }
}

void or_mc_density(const uint8_t* recs, uint32_t n, const float* gmin, const float* gmax, const uint32_t* res,
                   float scale, uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        float pos[3], mass;
        load(recs, i, pos, &mass);
        int outside = 0;
        for (int k = 0; k < 3; k++) outside |= (pos[k] < gmin[k]) || (pos[k] >= gmax[k]);
        if (outside) continue;
        int32_t start[3];
        float w[2][3];
        for (int k = 0; k < 3; k++) {
            float cell_size = (gmax[k] - gmin[k]) / (float)res[k];
            float pc = (pos[k] - gmin[k]) / cell_size;
            float center = pc - 0.5f;
            start[k] = f2i_sat(floorf(center));
            float f = center - (float)start[k];
            w[0][k] = 1.0f - f;
            w[1][k] = f;
        }
        int32_t rx = (int32_t)res[0], ry = (int32_t)res[1], rz = (int32_t)res[2];
        for (int z = 0; z < 2; z++)
            for (int y = 0; y < 2; y++)
                for (int x = 0; x < 2; x++) {
                    int32_t cx = start[0] + x, cy = start[1] + y, cz = start[2] + z;
                    if (cx < 0 || cy < 0 || cz < 0 || cx >= rx || cy >= ry || cz >= rz) continue;
                    float weight = (w[x][0] * w[y][1]) * w[z][2];
                    out[cx + cy * rx + cz * (rx * ry)] += f2u_sat((mass * weight) * scale);
                }
    }
}
