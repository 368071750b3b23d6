// mpm_mc.cu -- marching-cubes surface extraction of the snow density into a
// headless vertex buffer (the compute passes of the reference's
// GpuMarchingCubesRenderPipelineManager.addMeshGenerationPass,
// src/lib/gpu/marchingCubes/GpuMarchingCubesRenderPipelineManager.ts:587-633):
//   listBlocks            (mcListBlocks.cs.wgsl:24-96): an 8^3-cell block of the
//                         MC grid is active when any density cell under its
//                         cells -1..8 is nonzero;
//   computeVertexDensity  (mcVertexDensity.cs.wgsl:24-149): per vertex of an
//                         active block, the trilinear density at its world
//                         position and the central-difference gradient,
//                         normalised and packed as 4 x snorm8;
//   generateMesh          (mcGenerate.cs.wgsl:24-251, prelude.wgsl:55-87): per
//                         cell the case from the 8 vertex densities against the
//                         isovalue 0.15, one vertex per cut edge interpolated
//                         along the edge, normal = -(trilinear gradient),
//                         6 floats per vertex.
// Arithmetic follows the WGSL expressions operation by operation (-fmad=false).
//
// The case table is the reference's (triTable.wgsl, prelude.wgsl
// MC_TRI_COUNTS), written into mpm_mc_table.h by gen_mc_table.py: it fixes
// which triangles each cube case emits and in which vertex order.  The cube's
// vertex and edge numbering is the reference's (vertex bits x, z, y; edges
// along x, then y, then z).
//
// Differences by design: the active blocks are compacted in ascending order
// and triangles are placed by prefix sums (block, then cell, then table
// order) instead of atomics, so the vertex buffer is deterministic (the
// reference's order depends on workgroup timing); the vertex densities of a
// block live in a per-block workspace instead of a dense (res+1)^3 array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "mpm_engine.cuh"
#include "mpm_math.cuh"
#include "mpm_mc_table.h"

namespace mpm {

struct McTables {
    int8_t tri[256][16];   // edge indices, 3 per triangle, -1 after the last
    uint8_t count[256];    // triangles per case
    uint8_t ev[12][2];     // edge endpoints (cube vertex ids)
};

namespace {

int cube_vertex(int x, int y, int z) { return x + 2 * z + 4 * y; }

McTables build_tables() {
    McTables T;
    std::memset(&T, 0, sizeof(T));
    // edges: along axis a, the 4 positions of the other two coordinates (o0 + 2 o1)
    for (int a = 0, e = 0; a < 3; a++) {
        int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
        for (int q = 0; q < 4; q++, e++) {
            int p0[3] = {0, 0, 0};
            p0[o0] = q & 1;
            p0[o1] = q >> 1;
            int p1[3] = {p0[0], p0[1], p0[2]};
            p1[a] = 1;
            T.ev[e][0] = (uint8_t)cube_vertex(p0[0], p0[1], p0[2]);
            T.ev[e][1] = (uint8_t)cube_vertex(p1[0], p1[1], p1[2]);
        }
    }
    // the reference's case table (data contract: it fixes the triangles and
    // their vertex order, so the vertex buffer equals the reference's)
    for (int cs = 0; cs < 256; cs++) {
        std::memcpy(T.tri[cs], MPM_MC_TRI_TABLE[cs], 16);
        T.count[cs] = MPM_MC_TRI_COUNTS[cs];
    }
    return T;
}

}  // namespace

const McTables& mc_tables() {
    static const McTables T = build_tables();
    return T;
}

__constant__ McTables c_mc;

struct McArgs {
    const uint32_t* density;   // mcDensity grid, dres[0] * dres[1] * dres[2] u32
    uint32_t dres[3], mres[3], nblk[3];
    float gmin[3], gmax[3];
    float scale;
    uint32_t n_blocks;
    uint32_t* flags;           // n_blocks
    uint32_t* active;          // n_blocks (compacted)
    uint32_t* counters;        // [0] active blocks, [1] triangles
    float* vden;               // active x 729
    uint32_t* vgrad;           // active x 729
    uint32_t* tcount;          // active (triangles per block, then their offsets)
    float* out;                // max_vertices x 6
    uint32_t max_vertices;
};

constexpr float MC_ISO = 0.15f;
constexpr int MC_B = 8, MC_NV = 9 * 9 * 9;

__device__ __forceinline__ void block_coord(const McArgs& a, uint32_t b, int* bc) {
    uint32_t plane = a.nblk[0] * a.nblk[1];
    bc[2] = (int)(b / plane);
    uint32_t rem = b % plane;
    bc[1] = (int)(rem / a.nblk[0]);
    bc[0] = (int)(rem % a.nblk[0]);
}

// listBlocks: one warp per block, the 10^3 cells -1..8 spread over its lanes
__global__ void __launch_bounds__(256) k_mc_list(McArgs a) {
    const uint32_t b = blockIdx.x * 8u + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= a.n_blocks) return;
    int bc[3];
    block_coord(a, b, bc);
    bool any = false;
    for (int item = lane; item < 1000; item += 32) {
        int off[3] = {item % 10 - 1, (item / 10) % 10 - 1, item / 100 - 1};
        int dc[3];
        bool in = true;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            int cell = bc[k] * MC_B + off[k];
            float f = fd(fm((float)cell, __uint2float_rn(a.dres[k])), __uint2float_rn(a.mres[k]));
            dc[k] = (int)floorf(f);
            in = in && dc[k] >= 0 && dc[k] < (int)a.dres[k];
        }
        if (in && __ldg(a.density + (uint32_t)dc[0] + (uint32_t)dc[1] * a.dres[0] +
                        (uint32_t)dc[2] * a.dres[0] * a.dres[1]) > 0u)
            any = true;
    }
    any = __any_sync(0xffffffffu, any);
    if (lane == 0) a.flags[b] = any ? 1u : 0u;
}

// exclusive scan of n u32 (n from the argument, or *n_dev when given), one
// CTA of 1024 threads; the sum goes to *total.  compact: write the index of
// every nonzero entry to out[prefix] instead of the prefix sums.
__global__ void __launch_bounds__(1024) k_mc_scan(uint32_t* __restrict__ v, uint32_t n, const uint32_t* n_dev,
                                                  uint32_t* __restrict__ total, uint32_t* __restrict__ out, int compact) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (n_dev) n = *n_dev;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b0 = 0; b0 < n; b0 += 1024) {
        uint32_t i = b0 + threadIdx.x;
        uint32_t x0 = i < n ? v[i] : 0u;
        uint32_t x = x0;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const uint32_t incl = x + (warp > 0 ? wsum[warp - 1] : 0u);
        const uint32_t c = carry;
        if (i < n) {
            if (compact) {
                if (x0) out[c + incl - x0] = i;
            } else {
                v[i] = c + incl - x0;
            }
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = c + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__device__ __forceinline__ float density_cell(const McArgs& a, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= (int)a.dres[0] || y >= (int)a.dres[1] || z >= (int)a.dres[2]) return 0.0f;
    uint32_t u = __ldg(a.density + (uint32_t)x + (uint32_t)y * a.dres[0] + (uint32_t)z * a.dres[0] * a.dres[1]);
    return fd(__uint2float_rn(u), a.scale);
}

// sampleDensityAtWorldPos (mcVertexDensity.cs.wgsl:35-61)
__device__ float sample_density(const McArgs& a, const float* dcs, const float* p) {
    float cf[3], fr[3];
    int c0[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        cf[k] = fs(fd(fs(p[k], a.gmin[k]), dcs[k]), 0.5f);
        c0[k] = (int)floorf(cf[k]);
        fr[k] = fs(cf[k], (float)c0[k]);
    }
    float d = 0.0f;
#pragma unroll
    for (int dz = 0; dz <= 1; dz++)
#pragma unroll
        for (int dy = 0; dy <= 1; dy++)
#pragma unroll
            for (int dx = 0; dx <= 1; dx++) {
                float wx = dx ? fr[0] : fs(1.0f, fr[0]);
                float wy = dy ? fr[1] : fs(1.0f, fr[1]);
                float wz = dz ? fr[2] : fs(1.0f, fr[2]);
                float w = fm(fm(wx, wy), wz);
                d = fa(d, fm(density_cell(a, c0[0] + dx, c0[1] + dy, c0[2] + dz), w));
            }
    return d;
}

__device__ __forceinline__ uint32_t snorm8(float e) {
    float c = fminf(1.0f, fmaxf(-1.0f, e));
    return (uint32_t)((int)floorf(fa(0.5f, fm(127.0f, c)))) & 255u;
}

// computeVertexDensity of one active block into the workspace, then its
// triangle count
__global__ void __launch_bounds__(256) k_mc_vertex(McArgs a) {
    __shared__ float sd[MC_NV];
    __shared__ uint32_t wtri[8];
    const uint32_t n_active = a.counters[0];
    float mcs[3], dcs[3], eps[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float range = fs(a.gmax[k], a.gmin[k]);
        mcs[k] = fd(range, __uint2float_rn(a.mres[k]));
        dcs[k] = fd(range, __uint2float_rn(a.dres[k]));
        eps[k] = fm(dcs[k], 0.5f);
    }
    for (uint32_t slot = blockIdx.x; slot < n_active; slot += gridDim.x) {
        int bc[3];
        block_coord(a, a.active[slot], bc);
        for (int vi = threadIdx.x; vi < MC_NV; vi += 256) {
            int l[3] = {vi % 9, (vi / 9) % 9, vi / 81};
            int vc[3] = {bc[0] * MC_B + l[0], bc[1] * MC_B + l[1], bc[2] * MC_B + l[2]};
            float den = 0.0f;
            uint32_t packed = 0u;
            if (vc[0] <= (int)a.mres[0] && vc[1] <= (int)a.mres[1] && vc[2] <= (int)a.mres[2]) {
                float p[3];
#pragma unroll
                for (int k = 0; k < 3; k++) p[k] = fa(a.gmin[k], fm((float)vc[k], mcs[k]));
                den = sample_density(a, dcs, p);
                float g[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    float pp[3], pm[3];
#pragma unroll
                    for (int j = 0; j < 3; j++) {
                        pp[j] = fa(p[j], j == k ? eps[k] : 0.0f);
                        pm[j] = fs(p[j], j == k ? eps[k] : 0.0f);
                    }
                    g[k] = fs(sample_density(a, dcs, pp), sample_density(a, dcs, pm));
                }
                float d2 = fa(fa(fm(g[0], g[0]), fm(g[1], g[1])), fm(g[2], g[2]));
                if (d2 > 0.0f) {
                    float len = __fsqrt_rn(fa(d2, fm(0.0f, 0.0f)));
                    packed = snorm8(fd(g[0], len)) | (snorm8(fd(g[1], len)) << 8) | (snorm8(fd(g[2], len)) << 16) |
                             (snorm8(fd(0.0f, len)) << 24);
                }
            }
            sd[vi] = den;
            a.vden[(size_t)slot * MC_NV + vi] = den;
            a.vgrad[(size_t)slot * MC_NV + vi] = packed;
        }
        __syncthreads();
        uint32_t ntri = 0;
        for (int ci = threadIdx.x; ci < 512; ci += 256) {
            int c[3] = {ci % 8, (ci / 8) % 8, ci / 64};
            if (bc[0] * MC_B + c[0] >= (int)a.mres[0] || bc[1] * MC_B + c[1] >= (int)a.mres[1] ||
                bc[2] * MC_B + c[2] >= (int)a.mres[2])
                continue;
            uint32_t cs = 0;
#pragma unroll
            for (int v = 0; v < 8; v++) {
                int x = c[0] + (v & 1), y = c[1] + ((v >> 2) & 1), z = c[2] + ((v >> 1) & 1);
                if (sd[x + 9 * y + 81 * z] > MC_ISO) cs |= 1u << v;
            }
            ntri += c_mc.count[cs];
        }
        for (int o = 16; o > 0; o >>= 1) ntri += __shfl_xor_sync(0xffffffffu, ntri, o);
        if ((threadIdx.x & 31) == 0) wtri[threadIdx.x >> 5] = ntri;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = 0;
            for (int w = 0; w < 8; w++) s += wtri[w];
            a.tcount[slot] = s;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ float unsnorm8(uint32_t packed, int i) {
    int v = (int)(int8_t)((packed >> (8 * i)) & 255u);
    return fmaxf(fd((float)v, 127.0f), -1.0f);
}

__device__ __forceinline__ float mixf(float x, float y, float t) { return fa(fm(x, fs(1.0f, t)), fm(y, t)); }

// generateMesh of one active block at its triangle offset
__global__ void __launch_bounds__(256) k_mc_generate(McArgs a) {
    __shared__ float sd[MC_NV];
    __shared__ uint32_t sg[MC_NV];
    __shared__ uint32_t wsum[8];
    const uint32_t n_active = a.counters[0];
    float mcs[3];
#pragma unroll
    for (int k = 0; k < 3; k++) mcs[k] = fd(fs(a.gmax[k], a.gmin[k]), __uint2float_rn(a.mres[k]));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t slot = blockIdx.x; slot < n_active; slot += gridDim.x) {
        int bc[3];
        block_coord(a, a.active[slot], bc);
        for (int vi = threadIdx.x; vi < MC_NV; vi += 256) {
            sd[vi] = a.vden[(size_t)slot * MC_NV + vi];
            sg[vi] = a.vgrad[(size_t)slot * MC_NV + vi];
        }
        __syncthreads();
        // thread t owns cells 2t and 2t+1: cell order = thread order, so the
        // block prefix sum places triangles in cell order
        uint32_t cs[2], nt[2];
        bool valid[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int ci = 2 * threadIdx.x + h;
            int c[3] = {ci % 8, (ci / 8) % 8, ci / 64};
            valid[h] = bc[0] * MC_B + c[0] < (int)a.mres[0] && bc[1] * MC_B + c[1] < (int)a.mres[1] &&
                       bc[2] * MC_B + c[2] < (int)a.mres[2];
            cs[h] = 0;
            if (valid[h]) {
#pragma unroll
                for (int v = 0; v < 8; v++) {
                    int x = c[0] + (v & 1), y = c[1] + ((v >> 2) & 1), z = c[2] + ((v >> 1) & 1);
                    if (sd[x + 9 * y + 81 * z] > MC_ISO) cs[h] |= 1u << v;
                }
            }
            nt[h] = valid[h] ? c_mc.count[cs[h]] : 0u;
        }
        uint32_t mine = nt[0] + nt[1], x = mine;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        uint32_t before = x - mine;
        for (int w = 0; w < warp; w++) before += wsum[w];
        uint32_t tri = a.tcount[slot] + before;   // first triangle of cell 2t
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (nt[h] == 0) continue;
            int ci = 2 * threadIdx.x + h;
            int c[3] = {ci % 8, (ci / 8) % 8, ci / 64};
            float dv[8], gv[8][3];
#pragma unroll
            for (int v = 0; v < 8; v++) {
                int s = (c[0] + (v & 1)) + 9 * (c[1] + ((v >> 2) & 1)) + 81 * (c[2] + ((v >> 1) & 1));
                dv[v] = sd[s];
#pragma unroll
                for (int k = 0; k < 3; k++) gv[v][k] = unsnorm8(sg[s], k);
            }
            for (uint32_t t = 0; t < nt[h]; t++, tri++) {
                for (int q = 0; q < 3; q++) {
                    int e = c_mc.tri[cs[h]][3 * t + q];
                    int v0 = c_mc.ev[e][0], v1 = c_mc.ev[e][1];
                    float d0 = dv[v0], d1 = dv[v1];
                    float ti = fminf(fmaxf(fd(fs(MC_ISO, d0), fa(fs(d1, d0), 0.0001f)), 0.0f), 1.0f);
                    float p0[3] = {(float)(v0 & 1), (float)((v0 >> 2) & 1), (float)((v0 >> 1) & 1)};
                    float p1[3] = {(float)(v1 & 1), (float)((v1 >> 2) & 1), (float)((v1 >> 1) & 1)};
                    float lp[3], wp[3], nv[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        lp[k] = mixf(p0[k], p1[k], ti);
                        wp[k] = fa(a.gmin[k], fm(fa((float)(bc[k] * MC_B + c[k]), lp[k]), mcs[k]));
                    }
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        float g0 = mixf(gv[0][k], gv[1][k], lp[0]), g1 = mixf(gv[2][k], gv[3][k], lp[0]);
                        float g2 = mixf(gv[4][k], gv[5][k], lp[0]), g3 = mixf(gv[6][k], gv[7][k], lp[0]);
                        nv[k] = mixf(mixf(g0, g1, lp[2]), mixf(g2, g3, lp[2]), lp[1]);
                    }
                    float len = __fsqrt_rn(fa(fa(fm(nv[0], nv[0]), fm(nv[1], nv[1])), fm(nv[2], nv[2])));
                    float nrm[3] = {0.0f, 0.0f, 0.0f};
                    if (len > 0.0001f) {
#pragma unroll
                        for (int k = 0; k < 3; k++) nrm[k] = fd(-nv[k], len);
                    }
                    uint32_t vert = 3u * tri + (uint32_t)q;
                    if (vert < a.max_vertices) {
                        float* o = a.out + (size_t)vert * 6;
                        o[0] = wp[0]; o[1] = wp[1]; o[2] = wp[2];
                        o[3] = nrm[0]; o[4] = nrm[1]; o[5] = nrm[2];
                    }
                }
            }
        }
        __syncthreads();
    }
}

cudaError_t mc_upload_tables(cudaStream_t s) {
    return cudaMemcpyToSymbolAsync(c_mc, &mc_tables(), sizeof(McTables), 0, cudaMemcpyHostToDevice, s);
}

// Enqueues the MC passes; *vertices_total receives the number of vertices
// generated (3 per triangle; the buffer holds the first max_vertices).
int mc_run(const uint32_t* density, const uint32_t* dres, const uint32_t* mres, const float* gmin, const float* gmax,
           float scale, float* out, uint32_t max_vertices, uint32_t* vertices_total, int n_sms, cudaStream_t s,
           cudaError_t* err) {
    McArgs a{};
    a.density = density;
    for (int k = 0; k < 3; k++) {
        a.dres[k] = dres[k];
        a.mres[k] = mres[k];
        a.nblk[k] = (mres[k] + MC_B - 1) / MC_B;
        a.gmin[k] = gmin[k];
        a.gmax[k] = gmax[k];
    }
    a.scale = scale;
    a.n_blocks = a.nblk[0] * a.nblk[1] * a.nblk[2];
    a.out = out;
    a.max_vertices = max_vertices;
    const uint32_t nb = a.n_blocks;
    char* ws = nullptr;
    const size_t per_block = (size_t)MC_NV * 8 + 16;
    const size_t bytes = (size_t)nb * per_block + 64;
    cudaError_t e = cudaMallocAsync(&ws, bytes, s);
    if (e != cudaSuccess) { *err = e; return -1; }
    a.counters = reinterpret_cast<uint32_t*>(ws);
    a.flags = reinterpret_cast<uint32_t*>(ws + 64);
    a.active = a.flags + nb;
    a.tcount = a.active + nb;
    a.vden = reinterpret_cast<float*>(a.tcount + nb + (nb & 1u));   // 8-byte aligned
    a.vgrad = reinterpret_cast<uint32_t*>(a.vden + (size_t)nb * MC_NV);
    e = mc_upload_tables(s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.counters, 0, 64, s);
    if (e == cudaSuccess && nb) {
        k_mc_list<<<(nb + 7) / 8, 256, 0, s>>>(a);
        k_mc_scan<<<1, 1024, 0, s>>>(a.flags, nb, nullptr, a.counters + 0, a.active, 1);
        const int grid = std::max(1, std::min<int>((int)nb, n_sms * 4));
        k_mc_vertex<<<grid, 256, 0, s>>>(a);
        k_mc_scan<<<1, 1024, 0, s>>>(a.tcount, 0, a.counters + 0, a.counters + 1, nullptr, 0);
        k_mc_generate<<<grid, 256, 0, s>>>(a);
        e = cudaGetLastError();
    }
    uint32_t tri = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tri, a.counters + 1, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(ws, s);
    *err = e;
    if (e != cudaSuccess) return -1;
    *vertices_total = 3u * tri;
    return 0;
}

}  // namespace mpm

extern "C" int mpm_mc_tables(int8_t* tri_out, uint8_t* count_out, uint8_t* edge_vertices_out) {
    const mpm::McTables& T = mpm::mc_tables();
    if (tri_out) std::memcpy(tri_out, T.tri, sizeof(T.tri));
    if (count_out) std::memcpy(count_out, T.count, sizeof(T.count));
    if (edge_vertices_out) std::memcpy(edge_vertices_out, T.ev, sizeof(T.ev));
    return 0;
}
