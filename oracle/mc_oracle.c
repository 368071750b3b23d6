/*
 * mc_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the marching-cubes mesh generation of
 * luoluobuli/WebGPU-MPM-based-Snow-Simulation:
 *   block activity   src/lib/gpu/marchingCubes/mcListBlocks.cs.wgsl:24-96
 *   vertex density   src/lib/gpu/marchingCubes/mcVertexDensity.cs.wgsl:24-149
 *   triangles        src/lib/gpu/marchingCubes/mcGenerate.cs.wgsl:24-251,
 *                    prelude.wgsl:55-87 (edge interpolation, case index)
 * f32 arithmetic in the WGSL expression order, no contraction (the Makefile
 * builds with -ffp-contract=off); WGSL mix(a, b, t) = a (1 - t) + b t;
 * pack4x8snorm = floor(0.5 + 127 clamp(e, -1, 1)) per byte; unpack =
 * max(byte / 127, -1).  The triangulation table is an input (the caller's),
 * and the output order is: active 8^3 blocks ascending, cells in block order
 * (x fastest), triangles in table order, 6 floats per vertex.
 *
 * or_mc_tables returns the reference's case table (MC_TRI_TABLE of
 * marchingCubes/triTable.wgsl and MC_TRI_COUNTS of prelude.wgsl, a data
 * contract, shared with the CUDA passes through mpm_mc_table.h) and its edge
 * endpoints (MC_EDGE_V0 / MC_EDGE_V1, prelude.wgsl:45-46).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../webgpu-mpm-based-snow-simulation_b200/csrc/mpm_mc_table.h"

/* prelude.wgsl:45-46: edge e joins cube vertices EV0[e] and EV1[e] */
static const uint8_t EV0[12] = {0, 4, 2, 6, 0, 1, 2, 3, 0, 1, 4, 5};
static const uint8_t EV1[12] = {1, 5, 3, 7, 4, 5, 6, 7, 2, 3, 6, 7};

void or_mc_tables(int8_t* tri, uint8_t* count, uint8_t* ev) {
    memcpy(tri, MPM_MC_TRI_TABLE, sizeof(MPM_MC_TRI_TABLE));
    memcpy(count, MPM_MC_TRI_COUNTS, sizeof(MPM_MC_TRI_COUNTS));
    for (int e = 0; e < 12; e++) {
        ev[2 * e] = EV0[e];
        ev[2 * e + 1] = EV1[e];
    }
}

#define MC_ISO 0.15f

typedef struct {
    const uint32_t* density;
    uint32_t dres[3], mres[3];
    float gmin[3], scale, dcs[3], mcs[3];
} mc_ctx;

static float dens_cell(const mc_ctx* c, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= (int)c->dres[0] || y >= (int)c->dres[1] || z >= (int)c->dres[2]) return 0.0f;
    return (float)c->density[(uint32_t)x + (uint32_t)y * c->dres[0] + (uint32_t)z * c->dres[0] * c->dres[1]] / c->scale;
}

/* sampleDensityAtWorldPos (mcVertexDensity.cs.wgsl:35-61) */
static float sample(const mc_ctx* c, const float* p) {
    float cf[3], fr[3];
    int c0[3];
    for (int k = 0; k < 3; k++) {
        cf[k] = (p[k] - c->gmin[k]) / c->dcs[k] - 0.5f;
        c0[k] = (int)floorf(cf[k]);
        fr[k] = cf[k] - (float)c0[k];
    }
    float d = 0.0f;
    for (int dz = 0; dz <= 1; dz++)
        for (int dy = 0; dy <= 1; dy++)
            for (int dx = 0; dx <= 1; dx++) {
                float wx = dx ? fr[0] : 1.0f - fr[0];
                float wy = dy ? fr[1] : 1.0f - fr[1];
                float wz = dz ? fr[2] : 1.0f - fr[2];
                float w = (wx * wy) * wz;
                d = d + dens_cell(c, c0[0] + dx, c0[1] + dy, c0[2] + dz) * w;
            }
    return d;
}

static uint32_t snorm8(float e) {
    float cl = fminf(1.0f, fmaxf(-1.0f, e));
    return (uint32_t)((int)floorf(0.5f + 127.0f * cl)) & 255u;
}

static float unsnorm8(uint32_t packed, int i) {
    int v = (int)(int8_t)((packed >> (8 * i)) & 255u);
    return fmaxf((float)v / 127.0f, -1.0f);
}

static float mixf(float x, float y, float t) { return x * (1.0f - t) + y * t; }

void or_marching_cubes(const uint32_t* density, const uint32_t* dres, const uint32_t* mres, const float* gmin,
                       const float* gmax, float scale, const int8_t* tri, const uint8_t* count, const uint8_t* ev,
                       float* out, uint32_t max_vertices, uint32_t* n_vertices_out) {
    mc_ctx c;
    c.density = density;
    c.scale = scale;
    uint32_t nblk[3];
    float eps[3];
    for (int k = 0; k < 3; k++) {
        c.dres[k] = dres[k];
        c.mres[k] = mres[k];
        c.gmin[k] = gmin[k];
        float range = gmax[k] - gmin[k];
        c.mcs[k] = range / (float)mres[k];
        c.dcs[k] = range / (float)dres[k];
        eps[k] = c.dcs[k] * 0.5f;
        nblk[k] = (mres[k] + 7) / 8;
    }
    uint32_t nv = 0;
    static float vd[729];
    static uint32_t vg[729];
    for (uint32_t bz = 0; bz < nblk[2]; bz++)
        for (uint32_t by = 0; by < nblk[1]; by++)
            for (uint32_t bx = 0; bx < nblk[0]; bx++) {
                int bc[3] = {(int)bx, (int)by, (int)bz};
                /* listBlocks */
                int active = 0;
                for (int item = 0; item < 1000 && !active; item++) {
                    int off[3] = {item % 10 - 1, (item / 10) % 10 - 1, item / 100 - 1};
                    int dc[3], in = 1;
                    for (int k = 0; k < 3; k++) {
                        int cell = bc[k] * 8 + off[k];
                        float f = ((float)cell * (float)dres[k]) / (float)mres[k];
                        dc[k] = (int)floorf(f);
                        in = in && dc[k] >= 0 && dc[k] < (int)dres[k];
                    }
                    if (in && density[(uint32_t)dc[0] + (uint32_t)dc[1] * dres[0] + (uint32_t)dc[2] * dres[0] * dres[1]] > 0u)
                        active = 1;
                }
                if (!active) continue;
                /* computeVertexDensity */
                for (int vi = 0; vi < 729; vi++) {
                    int l[3] = {vi % 9, (vi / 9) % 9, vi / 81};
                    int vc[3] = {bc[0] * 8 + l[0], bc[1] * 8 + l[1], bc[2] * 8 + l[2]};
                    vd[vi] = 0.0f;
                    vg[vi] = 0u;
                    if (vc[0] > (int)mres[0] || vc[1] > (int)mres[1] || vc[2] > (int)mres[2]) continue;
                    float p[3];
                    for (int k = 0; k < 3; k++) p[k] = c.gmin[k] + (float)vc[k] * c.mcs[k];
                    vd[vi] = sample(&c, p);
                    float g[3];
                    for (int k = 0; k < 3; k++) {
                        float pp[3], pm[3];
                        for (int j = 0; j < 3; j++) {
                            pp[j] = p[j] + (j == k ? eps[k] : 0.0f);
                            pm[j] = p[j] - (j == k ? eps[k] : 0.0f);
                        }
                        g[k] = sample(&c, pp) - sample(&c, pm);
                    }
                    float d2 = (g[0] * g[0] + g[1] * g[1]) + g[2] * g[2];
                    if (d2 > 0.0f) {
                        float len = sqrtf(d2 + 0.0f * 0.0f);
                        vg[vi] = snorm8(g[0] / len) | (snorm8(g[1] / len) << 8) | (snorm8(g[2] / len) << 16) |
                                 (snorm8(0.0f / len) << 24);
                    }
                }
                /* generateMesh */
                for (int ci = 0; ci < 512; ci++) {
                    int cc[3] = {ci % 8, (ci / 8) % 8, ci / 64};
                    int cg[3] = {bc[0] * 8 + cc[0], bc[1] * 8 + cc[1], bc[2] * 8 + cc[2]};
                    if (cg[0] >= (int)mres[0] || cg[1] >= (int)mres[1] || cg[2] >= (int)mres[2]) continue;
                    float dv[8], gv[8][3];
                    uint32_t cs = 0;
                    for (int v = 0; v < 8; v++) {
                        int s = (cc[0] + (v & 1)) + 9 * (cc[1] + ((v >> 2) & 1)) + 81 * (cc[2] + ((v >> 1) & 1));
                        dv[v] = vd[s];
                        for (int k = 0; k < 3; k++) gv[v][k] = unsnorm8(vg[s], k);
                        if (dv[v] > MC_ISO) cs |= 1u << v;
                    }
                    for (int t = 0; t < count[cs]; t++)
                        for (int q = 0; q < 3; q++) {
                            int e = tri[cs * 16 + 3 * t + q];
                            int v0 = ev[2 * e], v1 = ev[2 * e + 1];
                            float d0 = dv[v0], d1 = dv[v1];
                            float ti = fminf(fmaxf((MC_ISO - d0) / ((d1 - d0) + 0.0001f), 0.0f), 1.0f);
                            float p0[3] = {(float)(v0 & 1), (float)((v0 >> 2) & 1), (float)((v0 >> 1) & 1)};
                            float p1[3] = {(float)(v1 & 1), (float)((v1 >> 2) & 1), (float)((v1 >> 1) & 1)};
                            float lp[3], wp[3], nvv[3], nrm[3] = {0.0f, 0.0f, 0.0f};
                            for (int k = 0; k < 3; k++) {
                                lp[k] = mixf(p0[k], p1[k], ti);
                                wp[k] = c.gmin[k] + ((float)cg[k] + lp[k]) * c.mcs[k];
                            }
                            for (int k = 0; k < 3; k++) {
                                float g0 = mixf(gv[0][k], gv[1][k], lp[0]), g1 = mixf(gv[2][k], gv[3][k], lp[0]);
                                float g2 = mixf(gv[4][k], gv[5][k], lp[0]), g3 = mixf(gv[6][k], gv[7][k], lp[0]);
                                nvv[k] = mixf(mixf(g0, g1, lp[2]), mixf(g2, g3, lp[2]), lp[1]);
                            }
                            float len = sqrtf((nvv[0] * nvv[0] + nvv[1] * nvv[1]) + nvv[2] * nvv[2]);
                            if (len > 0.0001f)
                                for (int k = 0; k < 3; k++) nrm[k] = (-nvv[k]) / len;
                            if (nv < max_vertices) {
                                float* o = out + (size_t)nv * 6;
                                o[0] = wp[0]; o[1] = wp[1]; o[2] = wp[2];
                                o[3] = nrm[0]; o[4] = nrm[1]; o[5] = nrm[2];
                            }
                            nv++;
                        }
                }
            }
    *n_vertices_out = nv;
}
