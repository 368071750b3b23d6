// mpm_splat.cu -- the particle splats the reference's renderers consume,
// into headless device buffers:
//   grid mass   calculateGridMass (src/lib/gpu/volumetric/calculateGridMass.wgsl:8-51):
//               linear-spline splat of particle mass onto the simulation grid,
//               u32 fixed point, for the volumetric ray march;
//   MC density  calculateDensity (src/lib/gpu/marchingCubes/mcDensity.cs.wgsl:14-63):
//               the same splat onto the marching-cubes density grid (half the
//               simulation resolution by default, GpuMarchingCubesBufferManager.ts:44-48),
//               with floor() instead of truncation for the base cell.
// One thread per particle, eight u32 adds, aggregated per warp (agg_add)
// on grids with fewer cells than particles; unsigned addition commutes, so
// every cell equals the reference's total in any order.  Arithmetic follows
// the WGSL expressions operation by operation (no contraction; the kernels are
// compiled with -fmad=false): cellSize = range / res, posCell = (pos - min) /
// cellSize, weight = (wx * wy) * wz, contribution = u32((mass * weight) * scale),
// f32 -> u32 truncating and saturating.
#include <cuda_runtime.h>

#include "mpm_engine.cuh"

namespace mpm {

struct SplatArgs {
    const float4* particles;
    uint32_t first, count;
    float gmin[3], gmax[3];
    uint32_t res[3];       // splat grid resolution
    float scale;           // fixedPointScale
    uint32_t* out;         // res[0] * res[1] * res[2] u32
};

__device__ __forceinline__ uint32_t f2u(float x) { return __float2uint_rz(x); }

constexpr uint32_t NO_CELL = 0xFFFFFFFFu;

// Warp-aggregated add: lanes holding the same cell sum their contributions
// first (u32 addition commutes and wraps, so the cell total is unchanged) and
// one lane adds the sum; coarse grids, where many particles of a warp share
// a cell, otherwise serialise on the same address.  Every lane of the warp
// calls it; lanes with nothing to add pass NO_CELL.
__device__ __forceinline__ void agg_add(uint32_t* out, uint32_t cell, uint32_t v) {
    const uint32_t peers = __match_any_sync(0xffffffffu, cell);
    const uint32_t sum = __reduce_add_sync(peers, v);
    if (cell != NO_CELL && (int)(threadIdx.x & 31u) == __ffs(peers) - 1) atomicAdd(out + cell, sum);
}

// KIND 0: calculateGridMass (truncated base cell, u32 coordinates);
// KIND 1: calculateDensity (floor of the base cell, i32 coordinates).
// AGG: warp-aggregated adds (grids with fewer cells than particles, where
// lanes of a warp often share a cell); else one atomic add per contribution.
template <int KIND, bool AGG>
__global__ void __launch_bounds__(256) k_splat(SplatArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < a.count;
    float pos[3] = {0.f, 0.f, 0.f}, mass = 0.f;
    if (valid) {
        const float4* rec = a.particles + (size_t)(a.first + i) * 12;
        float4 q0 = __ldg(rec), q1 = __ldg(rec + 1);
        pos[0] = q0.x; pos[1] = q0.y; pos[2] = q0.z;
        mass = q1.w;
#pragma unroll
        for (int k = 0; k < 3; k++)
            if (pos[k] < a.gmin[k] || pos[k] >= a.gmax[k]) valid = false;
    }
    int start[3] = {0, 0, 0};
    float w[2][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float cell_size = __fdiv_rn(__fsub_rn(a.gmax[k], a.gmin[k]), __uint2float_rn(a.res[k]));
        float pc = __fdiv_rn(__fsub_rn(pos[k], a.gmin[k]), cell_size);
        float center = __fsub_rn(pc, 0.5f);
        float f;
        if (KIND == 0) {
            uint32_t s0 = f2u(center);
            start[k] = (int)s0;
            f = __fsub_rn(center, __uint2float_rn(s0));
        } else {
            start[k] = __float2int_rz(floorf(center));
            f = __fsub_rn(center, __int2float_rn(start[k]));
        }
        w[0][k] = __fsub_rn(1.0f, f);
        w[1][k] = f;
    }
    const int rx = (int)a.res[0], ry = (int)a.res[1], rz = (int)a.res[2];
#pragma unroll
    for (int z = 0; z < 2; z++)
#pragma unroll
        for (int y = 0; y < 2; y++)
#pragma unroll
            for (int x = 0; x < 2; x++) {
                uint32_t cell = NO_CELL, v = 0u;
                if (valid) {
                    bool in;
                    uint32_t idx;
                    if (KIND == 0) {
                        uint32_t cx = (uint32_t)start[0] + x, cy = (uint32_t)start[1] + y, cz = (uint32_t)start[2] + z;
                        in = cx < a.res[0] && cy < a.res[1] && cz < a.res[2];
                        idx = cx + a.res[0] * (cy + a.res[1] * cz);
                    } else {
                        int cx = start[0] + x, cy = start[1] + y, cz = start[2] + z;
                        in = cx >= 0 && cy >= 0 && cz >= 0 && cx < rx && cy < ry && cz < rz;
                        idx = (uint32_t)(cx + cy * rx + cz * (rx * ry));
                    }
                    if (in) {
                        float weight = __fmul_rn(__fmul_rn(w[x][0], w[y][1]), w[z][2]);
                        cell = idx;
                        v = f2u(__fmul_rn(__fmul_rn(mass, weight), a.scale));
                    }
                }
                if (AGG) agg_add(a.out, cell, v);
                else if (cell != NO_CELL) atomicAdd(a.out + cell, v);
            }
}

cudaError_t launch_splat(int kind, const SplatArgs& a, cudaStream_t s) {
    if (a.count == 0) return cudaSuccess;
    uint32_t blocks = (a.count + 255u) / 256u;
    const bool agg = (uint64_t)a.res[0] * a.res[1] * a.res[2] < (uint64_t)a.count;
    if (kind == 0) {
        if (agg) k_splat<0, true><<<blocks, 256, 0, s>>>(a);
        else k_splat<0, false><<<blocks, 256, 0, s>>>(a);
    } else {
        if (agg) k_splat<1, true><<<blocks, 256, 0, s>>>(a);
        else k_splat<1, false><<<blocks, 256, 0, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace mpm
