// mpm_raymarch.cu -- the volumetric renderer's ray march
// (doVolumetricRaymarch, src/lib/gpu/volumetric/volumetricRaymarch.cs.wgsl:118-226)
// into headless device buffers: an RGBA8 image, an f32 depth image and,
// optionally, the f32 colour before quantisation.  The density field is the
// u32 fixed-point mass grid of calculateGridMass (mpm_splat.cu).
//
// One thread per pixel, 16 x 16 pixels per CTA (the reference's workgroup).
// Per sample, readDensity (:16-57) gathers 8 u32 cells through the read-only
// cache; every dense sample also marches a 64-step shadow ray (:94-108).
// Arithmetic follows the WGSL expressions operation by operation (no
// contraction, the file is compiled with -fmad=false); exp and pow are the
// project's f64 routines rounded once to f32 (mpm_math.cuh); matrix-vector
// products sum the columns in order, ((c0 x + c1 y) + c2 z) + c3 w; normalize
// divides each component by the IEEE square root of the ordered dot product.
// The workgroupBarrier() calls of the WGSL order nothing here (no shared
// memory) and are left out.
#include <cuda_runtime.h>

#include "mpm_engine.cuh"
#include "mpm_math.cuh"

namespace mpm {

namespace rm {

constexpr float EXTINCTION = 724.0f;
constexpr float STEP = 0.025f;
constexpr uint32_t N_STEPS = 256u, N_SHADOW_STEPS = 64u;
__device__ __forceinline__ float albedo(int k) { return k == 0 ? 0.9f : (k == 1 ? 0.985f : 0.99f); }
// 4 * PI with PI = 3.1415926, evaluated as an abstract-float constant and
// rounded once to f32
constexpr float FOUR_PI = (float)(4.0 * 3.1415926);
// 1 / 2.2, likewise
constexpr float INV_GAMMA = (float)(1.0 / 2.2);

struct Field {
    const uint32_t* mass;
    uint32_t res[3];
    float gmin[3], gmax[3];
    float cell[3];    // gridRange / gridRes
    float volume;     // cellSize.x * cellSize.y * cellSize.z
    float scale;
};

// readDensity (volumetricRaymarch.cs.wgsl:16-57)
__device__ __forceinline__ float read_density(const Field& F, const float* p) {
#pragma unroll
    for (int k = 0; k < 3; k++)
        if (p[k] < F.gmin[k] || p[k] >= F.gmax[k]) return 0.0f;
    uint32_t start[3];
    float w[2][3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float gp = fd(fs(p[k], F.gmin[k]), F.cell[k]);
        float sp = fs(gp, 0.5f);
        start[k] = __float2uint_rz(sp);   // saturating: negatives give 0
        float f = fs(sp, __uint2float_rn(start[k]));
        w[0][k] = fs(1.0f, f);
        w[1][k] = f;
    }
    float mass = 0.0f;
#pragma unroll
    for (int z = 0; z < 2; z++)
#pragma unroll
        for (int y = 0; y < 2; y++)
#pragma unroll
            for (int x = 0; x < 2; x++) {
                int cx = (int)(start[0] + x), cy = (int)(start[1] + y), cz = (int)(start[2] + z);
                if (cx < 0 || cy < 0 || cz < 0 || cx >= (int)F.res[0] || cy >= (int)F.res[1] || cz >= (int)F.res[2])
                    continue;
                uint32_t idx = (uint32_t)cx + F.res[0] * ((uint32_t)cy + F.res[1] * (uint32_t)cz);
                float val = fd(__uint2float_rn(__ldg(F.mass + idx)), F.scale);
                float weight = fm(fm(w[x][0], w[y][1]), w[z][2]);
                mass = fa(mass, fm(val, weight));
            }
    return fm(fd(mass, F.volume), 0.00001f);
}

// henyeyGreenstein (:59-63)
__device__ __forceinline__ float hg(float c, float g) {
    float g2 = fm(g, g);
    float denom = fs(fa(1.0f, g2), fm(fm(2.0f, g), c));
    return fd(fs(1.0f, g2), fm(FOUR_PI, powf_m(denom, 1.5f)));
}

// raymarchShadow (:94-108)
__device__ __forceinline__ void shadow(const Field& F, const float* pos, const float* ld, uint32_t time, float* T) {
    uint32_t h = hash4(__float_as_uint(pos[0]), __float_as_uint(pos[1]), __float_as_uint(pos[2]), time);
    float jitter = fd(__uint2float_rn(h), 4294967296.0f);
    float sp[3], st[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        st[k] = fm(ld[k], STEP);
        sp[k] = fa(pos[k], fm(st[k], jitter));
        T[k] = 1.0f;
    }
    for (uint32_t s = 0; s < N_SHADOW_STEPS; s++) {
#pragma unroll
        for (int k = 0; k < 3; k++) sp[k] = fa(sp[k], st[k]);
        float d = read_density(F, sp);
        if (d > 1e-4f) {
            float a = fm(-fm(EXTINCTION, d), STEP);
#pragma unroll
            for (int k = 0; k < 3; k++) T[k] = fm(T[k], expf_m(fm(a, albedo(k))));
            if (T[0] < 1e-4f && T[1] < 1e-4f && T[2] < 1e-4f) break;
        }
    }
}

// uniforms.viewProjInvMat * vec4f(x, y, z, 1), divided by w
__device__ __forceinline__ void unproject(const float* M, float x, float y, float z, float* o) {
    float h[4];
#pragma unroll
    for (int r = 0; r < 4; r++) h[r] = fa(fa(fa(fm(M[r], x), fm(M[4 + r], y)), fm(M[8 + r], z)), fm(M[12 + r], 1.0f));
#pragma unroll
    for (int k = 0; k < 3; k++) o[k] = fd(h[k], h[3]);
}

__device__ __forceinline__ float dot3s(const float* a, const float* b) {
    return fa(fa(fm(a[0], b[0]), fm(a[1], b[1])), fm(a[2], b[2]));
}

__device__ __forceinline__ void normalize3(float* v) {
    float l = __fsqrt_rn(dot3s(v, v));
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = fd(v[k], l);
}

__device__ __forceinline__ uint8_t unorm8(float v) {
    float c = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)__float2uint_rn(fm(c, 255.0f));
}

}  // namespace rm

__global__ void __launch_bounds__(256) k_raymarch(RaymarchArgs a) {
    using namespace rm;
    const uint32_t gx = blockIdx.x * 16u + threadIdx.x, gy = blockIdx.y * 16u + threadIdx.y;
    if (gx >= a.width || gy >= a.height) return;
    const size_t pix = (size_t)gy * a.width + gx;
    Field F;
    F.mass = a.mass;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        F.res[k] = a.res[k];
        F.gmin[k] = a.gmin[k];
        F.gmax[k] = a.gmax[k];
        F.cell[k] = fd(fs(a.gmax[k], a.gmin[k]), __uint2float_rn(a.res[k]));
    }
    F.volume = fm(fm(F.cell[0], F.cell[1]), F.cell[2]);
    F.scale = a.scale;

    // calculateViewRay (shaderPrelude/cameraOps.wgsl:6-19)
    float u = fd(__uint2float_rn(gx), __uint2float_rn(a.width));
    float v = fd(__uint2float_rn(gy), __uint2float_rn(a.height));
    float ux = fs(fm(u, 2.0f), 1.0f), uy = fs(fm(fs(1.0f, v), 2.0f), 1.0f);
    float org[3], far_p[3], dir[3];
    unproject(a.inv_vp, ux, uy, 0.0f, org);
    unproject(a.inv_vp, ux, uy, 1.0f, far_p);
#pragma unroll
    for (int k = 0; k < 3; k++) dir[k] = fs(far_p[k], org[k]);
    normalize3(dir);

    float ld[3] = {0.2f, 0.18f, 0.9f};
    normalize3(ld);
    const float lc[3] = {fm(0.95f, 5.0f), fm(0.995f, 5.0f), fm(1.0f, 5.0f)};
    const float amb[3] = {0.0f, 0.1f, 0.2f};

    // aabbIntersectionDistances (:72-87)
    float t_near = -__int_as_float(0x7f800000), t_far = __int_as_float(0x7f800000);
    {
        float t1[3], t2[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float dmin = fd(fs(a.gmin[k], org[k]), dir[k]);
            float dmax = fd(fs(a.gmax[k], org[k]), dir[k]);
            t1[k] = fminf(dmin, dmax);
            t2[k] = fmaxf(dmin, dmax);
        }
        t_near = fmaxf(fmaxf(t1[0], t1[1]), t1[2]);
        t_far = fminf(fminf(t2[0], t2[1]), t2[2]);
    }

    float d_ground = 1e20f;
    bool hit_ground = false;
    if (fabsf(dir[2]) > 1e-4f) {
        float cand = fd(fs(a.gmin[2], org[2]), dir[2]);
        if (cand > 0.0f) {
            float hx = fa(org[0], fm(cand, dir[0])), hy = fa(org[1], fm(cand, dir[1]));
            if (hx >= a.gmin[0] && hy >= a.gmin[1] && hx <= a.gmax[0] && hy <= a.gmax[1]) {
                d_ground = cand;
                hit_ground = true;
            }
        }
    }

    if (!(t_near <= t_far && t_far >= 0.0f)) {
        reinterpret_cast<uchar4*>(a.rgba)[pix] = make_uchar4(0, 0, 0, 0);
        if (a.color) reinterpret_cast<float4*>(a.color)[pix] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;   // the depth image keeps its previous content, as the reference's texture does
    }

    const float d_start = fmaxf(0.0f, t_near);
    const float d_end = fminf(t_far, d_ground);
    float jitter = fd(__uint2float_rn(hash3(gx, gy, a.time)), 4294967296.0f);
    float cur = fa(d_start, fm(jitter, STEP));

    float T[3] = {1.0f, 1.0f, 1.0f}, col[3] = {0.0f, 0.0f, 0.0f};
    bool depth_written = false;
    float depth = 1e20f;
    // the phase function depends only on the ray: evaluated once
    const float phase = fa(hg(dot3s(dir, ld), -0.5f), hg(dot3s(dir, ld), 0.5f));

    for (uint32_t i = 0; i < N_STEPS; i++) {
        if (cur >= d_end || (T[0] < 0.01f && T[1] < 0.01f && T[2] < 0.01f)) break;
        float pos[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pos[k] = fa(org[k], fm(cur, dir[k]));
        float density = read_density(F, pos);
        if (density > 0.001f) {
            if (!depth_written) {
                depth = cur;
                depth_written = true;
            }
            float ext = fm(EXTINCTION, density);
            float a_ext = fm(-ext, STEP);
            float sh[3];
            shadow(F, pos, ld, a.time, sh);
            float inv_ext = fmaxf(ext, 1e-4f);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                float scat = fm(ext, albedo(k));
                float stT = expf_m(fm(a_ext, albedo(k)));
                float light = fa(amb[k], fm(fm(lc[k], phase), sh[k]));
                float laf = fd(fm(fm(light, scat), fs(1.0f, stT)), inv_ext);
                col[k] = fa(col[k], fm(T[k], laf));
                T[k] = fm(T[k], stT);
            }
        }
        cur = fa(cur, STEP);
    }

    if (hit_ground && (T[0] > 0.01f || T[1] > 0.01f || T[2] > 0.01f)) {
        float pos[3], sh[3];
#pragma unroll
        for (int k = 0; k < 3; k++) pos[k] = fa(org[k], fm(d_ground, dir[k]));
        shadow(F, pos, ld, a.time, sh);
        float lz = fmaxf(0.0f, ld[2]);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float gcol = fa(amb[k], fm(0.05f, fm(fm(lc[k], sh[k]), lz)));
            col[k] = fa(col[k], fm(T[k], gcol));
            T[k] = 0.0f;
        }
        if (!depth_written) depth = d_ground;
    }

    float alpha = fs(1.0f, fmaxf(T[0], fmaxf(T[1], T[2])));
    float o[4] = {fm(powf_m(col[0], INV_GAMMA), alpha), fm(powf_m(col[1], INV_GAMMA), alpha),
                  fm(powf_m(col[2], INV_GAMMA), alpha), fm(1.0f, alpha)};
    reinterpret_cast<uchar4*>(a.rgba)[pix] = make_uchar4(unorm8(o[0]), unorm8(o[1]), unorm8(o[2]), unorm8(o[3]));
    if (a.color) reinterpret_cast<float4*>(a.color)[pix] = make_float4(o[0], o[1], o[2], o[3]);
    a.depth[pix] = depth;
}

cudaError_t launch_raymarch(const RaymarchArgs& a, cudaStream_t s) {
    if (a.width == 0 || a.height == 0) return cudaSuccess;
    dim3 grid((a.width + 15u) / 16u, (a.height + 15u) / 16u);
    k_raymarch<<<grid, dim3(16, 16), 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mpm
