// mpm_scatter.cu -- particle initialisation: scatterParticles
// (src/lib/gpu/particleInitialize/particleScatter.cs.wgsl:47-84).  Each
// particle draws candidates uniformly in the mesh's bounding box
// (uniforms.meshMinCoords / meshMaxCoords) from its own hash stream until one
// lies inside the closed triangle mesh (even-odd count of Moller-Trumbore
// hits along +x, triangleOps.wgsl), at most 512 attempts, then jitters it by
// three fBm values (randomNumberGenerators.wgsl:57-94) and draws its mass.
//
// B200 form: one thread per particle, all threads of a CTA test their current
// candidates against the mesh in rounds, the triangles streamed through
// shared memory in chunks (the reference reads every vertex from global
// memory per thread); a thread whose candidate is inside stops drawing.  The
// hit parity does not depend on the order the triangles are visited, so the
// result equals the reference's sequential loop.  Arithmetic: the step's f32
// helpers (dot and cross with the canonical fused order), IEEE division,
// mix(a, b, t) = a (1 - t) + b t unfused, fract(x) = x - floor(x).
#include <cuda_runtime.h>

#include "mpm_math.cuh"

namespace mpm {

struct ScatterArgs {
    float4* particles;         // n records (12 float4 each)
    uint32_t n;
    const float4* verts;       // triangle soup, 3 vertices per triangle (xyz, pad)
    uint32_t n_tris;
    float mmin[3], mmax[3];    // meshMinCoords, meshMaxCoords
};

constexpr int SCATTER_BS = 256;
constexpr int SCATTER_CHUNK = 512;            // triangles per shared-memory chunk
constexpr uint32_t SCATTER_MAX_ATTEMPTS = 512u;

__device__ __forceinline__ float u32_unit(uint32_t h) { return fd(__uint2float_rn(h), 4294967296.0f); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return fa(fm(a, fs(1.0f, t)), fm(b, t)); }

__device__ __forceinline__ float rand_float(uint32_t& seed) {
    seed = hash1(seed);
    return u32_unit(seed);
}

// rayIntersectsTriangle (triangleOps.wgsl), ray direction +x
__device__ __forceinline__ bool ray_x_hits(const float* o, const float* v0, const float* v1, const float* v2) {
    const float eps = 1e-6f;
    const float dir[3] = {1.0f, 0.0f, 0.0f};
    float e1[3] = {fs(v1[0], v0[0]), fs(v1[1], v0[1]), fs(v1[2], v0[2])};
    float e2[3] = {fs(v2[0], v0[0]), fs(v2[1], v0[1]), fs(v2[2], v0[2])};
    float rce2[3];
    cross3(dir, e2, rce2);
    float det = dot3(e1, rce2);
    if (fabsf(det) < eps) return false;
    float inv = fd(1.0f, det);
    float ov[3] = {fs(o[0], v0[0]), fs(o[1], v0[1]), fs(o[2], v0[2])};
    float b0 = fm(dot3(ov, rce2), inv);
    if (b0 < 0.0f || 1.0f < b0) return false;
    float ove1[3];
    cross3(ov, e1, ove1);
    float b1 = fm(dot3(dir, ove1), inv);
    if (b1 < 0.0f || 1.0f < b1 || fa(b0, b1) > 1.0f) return false;
    return fm(dot3(e2, ove1), inv) > eps;
}

__device__ __forceinline__ float noise3(float x0, float x1, float x2) {
    float x[3] = {x0, x1, x2}, f[3], u[3];
    uint32_t n[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float p = floorf(x[k]);
        f[k] = fs(x[k], p);
        u[k] = fm(fm(f[k], f[k]), fs(3.0f, fm(2.0f, f[k])));
        n[k] = (uint32_t)__float2int_rz(p);
    }
    float c[8];
#pragma unroll
    for (int i = 0; i < 8; i++) c[i] = u32_unit(hash3(n[0] + (i & 1), n[1] + ((i >> 1) & 1), n[2] + (i >> 2)));
    return mixf(mixf(mixf(c[0], c[1], u[0]), mixf(c[2], c[3], u[0]), u[1]),
                mixf(mixf(c[4], c[5], u[0]), mixf(c[6], c[7], u[0]), u[1]), u[2]);
}

__device__ __forceinline__ float fbm3(float x0, float x1, float x2) {
    float v = 0.0f, a = 0.5f;
#pragma unroll 1
    for (int i = 0; i < 6; i++) {
        v = fa(v, fm(a, noise3(x0, x1, x2)));
        x0 = fm(x0, 2.0f);
        x1 = fm(x1, 2.0f);
        x2 = fm(x2, 2.0f);
        a = fm(a, 0.5f);
    }
    return v;
}

__global__ void __launch_bounds__(SCATTER_BS) k_scatter(ScatterArgs a) {
    __shared__ float4 tri[SCATTER_CHUNK * 3];
    const uint32_t i = blockIdx.x * SCATTER_BS + threadIdx.x;
    const bool active = i < a.n;
    uint32_t seed = hash4(i, 100u, 200u, 300u);
    float cand[3] = {0.f, 0.f, 0.f};
    bool done = !active;
    for (uint32_t attempt = 0; attempt < SCATTER_MAX_ATTEMPTS; attempt++) {
        if (__syncthreads_and(done ? 1 : 0)) break;
        if (!done) {
#pragma unroll
            for (int k = 0; k < 3; k++) cand[k] = mixf(a.mmin[k], a.mmax[k], rand_float(seed));
        }
        bool inside = false;
        for (uint32_t t0 = 0; t0 < a.n_tris; t0 += SCATTER_CHUNK) {
            uint32_t nt = min((uint32_t)SCATTER_CHUNK, a.n_tris - t0);
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < nt * 3; k += SCATTER_BS) tri[k] = __ldg(a.verts + (size_t)t0 * 3 + k);
            __syncthreads();
            if (!done) {
                for (uint32_t t = 0; t < nt; t++) {
                    float4 p0 = tri[3 * t], p1 = tri[3 * t + 1], p2 = tri[3 * t + 2];
                    float v0[3] = {p0.x, p0.y, p0.z}, v1[3] = {p1.x, p1.y, p1.z}, v2[3] = {p2.x, p2.y, p2.z};
                    if (ray_x_hits(cand, v0, v1, v2)) inside = !inside;
                }
            }
        }
        if (!done && inside) done = true;
    }
    if (!active) return;
    const float freq = 4.0f, scale = 0.1f;
    float x[3] = {fm(cand[0], freq), fm(cand[1], freq), fm(cand[2], freq)};
    float d0 = fbm3(x[0], x[1], x[2]);
    float d1 = fbm3(fa(x[0], 100.0f), fa(x[1], 200.0f), fa(x[2], 300.0f));
    float d2 = fbm3(fa(x[0], -300.0f), fa(x[1], -200.0f), fa(x[2], -100.0f));
    float pos[3] = {fa(cand[0], fm(fs(d0, 0.5f), scale)), fa(cand[1], fm(fs(d1, 0.5f), scale)),
                    fa(cand[2], fm(fs(d2, 0.5f), scale))};
    float m1 = u32_unit(hash1(i));
    float4* rec = a.particles + (size_t)i * 12;
    rec[0] = make_float4(pos[0], pos[1], pos[2], 1.0f);
    rec[1] = make_float4(0.f, 0.f, 0.f, fm(m1, m1));
    rec[2] = make_float4(1.f, 0.f, 0.f, 0.f);
    rec[3] = make_float4(0.f, 1.f, 0.f, 0.f);
    rec[4] = make_float4(0.f, 0.f, 1.f, 0.f);
    rec[5] = make_float4(1.f, 0.f, 0.f, 0.f);
    rec[6] = make_float4(0.f, 1.f, 0.f, 0.f);
    rec[7] = make_float4(0.f, 0.f, 1.f, 0.f);
    for (int q = 8; q < 12; q++) rec[q] = make_float4(0.f, 0.f, 0.f, 0.f);
}

cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    k_scatter<<<(a.n + SCATTER_BS - 1) / SCATTER_BS, SCATTER_BS, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mpm
