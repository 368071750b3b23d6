// mpm_splat.cu -- the particle splats the reference's renderers consume,
// into headless device buffers:
//   grid mass   calculateGridMass (src/lib/gpu/volumetric/calculateGridMass.wgsl:8-51):
//               linear-spline splat of particle mass onto the simulation grid,
//               u32 fixed point, for the volumetric ray march;
//   MC density  calculateDensity (src/lib/gpu/marchingCubes/mcDensity.cs.wgsl:14-63):
//               the same splat onto the marching-cubes density grid (half the
//               simulation resolution by default, GpuMarchingCubesBufferManager.ts:44-48),
//               with floor() instead of truncation for the base cell.
// One thread per particle, eight u32 atomic adds; unsigned addition commutes,
// so every cell equals the reference's total in any order.  Arithmetic follows
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

__global__ void __launch_bounds__(256) k_grid_mass(SplatArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const float4* rec = a.particles + (size_t)(a.first + i) * 12;
    float4 q0 = __ldg(rec), q1 = __ldg(rec + 1);
    float pos[3] = {q0.x, q0.y, q0.z};
    float mass = q1.w;
#pragma unroll
    for (int k = 0; k < 3; k++)
        if (pos[k] < a.gmin[k] || pos[k] >= a.gmax[k]) return;
    uint32_t start[3];
    float w[2][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float cell_size = __fdiv_rn(__fsub_rn(a.gmax[k], a.gmin[k]), __uint2float_rn(a.res[k]));
        float pc = __fdiv_rn(__fsub_rn(pos[k], a.gmin[k]), cell_size);
        float center = __fsub_rn(pc, 0.5f);
        start[k] = f2u(center);
        float f = __fsub_rn(center, __uint2float_rn(start[k]));
        w[0][k] = __fsub_rn(1.0f, f);
        w[1][k] = f;
    }
#pragma unroll
    for (int z = 0; z < 2; z++)
#pragma unroll
        for (int y = 0; y < 2; y++)
#pragma unroll
            for (int x = 0; x < 2; x++) {
                uint32_t cx = start[0] + x, cy = start[1] + y, cz = start[2] + z;
                if (cx >= a.res[0] || cy >= a.res[1] || cz >= a.res[2]) continue;
                float weight = __fmul_rn(__fmul_rn(w[x][0], w[y][1]), w[z][2]);
                uint32_t idx = cx + a.res[0] * (cy + a.res[1] * cz);
                atomicAdd(&a.out[idx], f2u(__fmul_rn(__fmul_rn(mass, weight), a.scale)));
            }
}

__global__ void __launch_bounds__(256) k_mc_density(SplatArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const float4* rec = a.particles + (size_t)(a.first + i) * 12;
    float4 q0 = __ldg(rec), q1 = __ldg(rec + 1);
    float pos[3] = {q0.x, q0.y, q0.z};
    float mass = q1.w;
#pragma unroll
    for (int k = 0; k < 3; k++)
        if (pos[k] < a.gmin[k] || pos[k] >= a.gmax[k]) return;
    int start[3];
    float w[2][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float cell_size = __fdiv_rn(__fsub_rn(a.gmax[k], a.gmin[k]), __uint2float_rn(a.res[k]));
        float pc = __fdiv_rn(__fsub_rn(pos[k], a.gmin[k]), cell_size);
        float center = __fsub_rn(pc, 0.5f);
        start[k] = __float2int_rz(floorf(center));
        float f = __fsub_rn(center, __int2float_rn(start[k]));
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
                int cx = start[0] + x, cy = start[1] + y, cz = start[2] + z;
                if (cx < 0 || cy < 0 || cz < 0 || cx >= rx || cy >= ry || cz >= rz) continue;
                float weight = __fmul_rn(__fmul_rn(w[x][0], w[y][1]), w[z][2]);
                int idx = cx + cy * rx + cz * (rx * ry);
                atomicAdd(&a.out[idx], f2u(__fmul_rn(__fmul_rn(mass, weight), a.scale)));
            }
}

cudaError_t launch_splat(int kind, const SplatArgs& a, cudaStream_t s) {
    if (a.count == 0) return cudaSuccess;
    uint32_t blocks = (a.count + 255u) / 256u;
    if (kind == 0) k_grid_mass<<<blocks, 256, 0, s>>>(a);
    else k_mc_density<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mpm
