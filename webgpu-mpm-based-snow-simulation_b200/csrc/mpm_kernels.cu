// mpm_kernels.cu -- the MPM substep as CUDA kernels for sm_100a.
//
// Substep (explicit):  clear_table -> bin_insert -> compact_{a,b,c} -> bin_scatter
//                      -> p2g_explicit -> g2p_explicit (G2P + integrate fused)
// Substep (PBMPM, n_iter iterations):  same binning, then
//                      pbmpm_first (constraints + affine P2G + forces)
//                      -> (n_iter-1) x pbmpm_iter (G2P, constraints, P2G fused)
//                      -> g2p_pbmpm (last G2P + integrate fused)
//
// The reference runs the same math as 11 (explicit) or 16 (PBMPM, 3 iters)
// WGSL dispatches (src/lib/gpu/mpm/GpuMpmPipelineManager.ts:327-521) with
// 108 global i32 atomics per particle per transfer; here each tile's
// particles accumulate into a shared-memory halo tile and the tile is
// written once with plain 16-byte stores.
#include "mpm_engine.cuh"
#include "mpm_math.cuh"
#include "mpm_plast.cuh"

namespace mpm {

// ------------------------------------------------------------------
// shared helpers
// ------------------------------------------------------------------
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t tile_hash(uint32_t scene, int sx, int sy, int sz) {
    return hash3((uint32_t)sx, (uint32_t)sy, (uint32_t)sz) ^ (scene * 0x9E3779B1u);
}

__device__ uint32_t tile_insert(const Ctx& c, uint64_t key, uint32_t scene, int sx, int sy, int sz) {
    uint32_t mask = c.cap - 1u;
    uint32_t s = tile_hash(scene, sx, sy, sz) & mask;
    uint32_t limit = c.cap < MAX_PROBES ? c.cap : MAX_PROBES;
    for (uint32_t probe = 0; probe < limit; probe++) {
        unsigned long long k = *((volatile unsigned long long*)&c.keys[s]);
        if (k == key) return s;
        if (k == KEY_EMPTY) {
            unsigned long long old = atomicCAS(&c.keys[s], KEY_EMPTY, (unsigned long long)key);
            if (old == KEY_EMPTY || old == key) return s;
        }
        s = (s + 1u) & mask;
    }
    atomicOr(&c.counters->status, ST_HASH_FULL);
    return INVALID;
}

__device__ uint32_t tile_lookup(const Ctx& c, uint64_t key, uint32_t scene, int sx, int sy, int sz) {
    uint32_t mask = c.cap - 1u;
    uint32_t s = tile_hash(scene, sx, sy, sz) & mask;
    uint32_t limit = c.cap < MAX_PROBES ? c.cap : MAX_PROBES;
    for (uint32_t probe = 0; probe < limit; probe++) {
        unsigned long long k = c.keys[s];
        if (k == key) return s;
        if (k == KEY_EMPTY) return INVALID;
        s = (s + 1u) & mask;
    }
    return INVALID;
}

__device__ __forceinline__ uint32_t find_scene(const Ctx& c, uint32_t p) {
    uint32_t lo = 0, hi = c.n_scenes;  // answer in [0, n_scenes)
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&c.scene_first[mid]) <= p) lo = mid; else hi = mid;
    }
    return lo;
}

// floor(a / E) for a compile-time tile edge E (also for negative a)
template <int E>
__device__ __forceinline__ int floor_div(int a) {
    int q = a / E;
    return (a < 0 && q * E != a) ? q - 1 : q;
}

__device__ __forceinline__ void load_scene_smem(SceneDev& dst, const SceneDev* src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(SceneDev) / 4); i += blockDim.x) d[i] = s[i];
}

// f32(i) / fixedPointScale
__device__ __forceinline__ float inv_s(const SceneDev& S, int32_t v) { return fm(i2f(v), S.rscale); }

// Grid-side boundary of boundary_mode 1 (an extension; the reference only
// reflects particles): sticky ground plane, slip walls.
__device__ __forceinline__ void grid_bc(const SceneDev& S, const int* gc, float* v) {
    if (S.bmode != 1u) return;
    if (gc[S.gaxis] < S.bc) { v[0] = 0.f; v[1] = 0.f; v[2] = 0.f; return; }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (gc[a] < S.bc && v[a] < 0.f) v[a] = 0.f;
        if (gc[a] >= S.res[a] - S.bc && v[a] > 0.f) v[a] = 0.f;
    }
}

// ------------------------------------------------------------------
// particle state access: the 192-byte record (12 float4 words, the
// reference's ParticleData layout) of work slot t, word q at w[q * n + t]
// ------------------------------------------------------------------
struct PState {
    float pos[3], hom, vel[3], mass;
    float Fe[9], Fp[9], dxp[3], D[9];
};

__device__ __forceinline__ void unpack_m(const float4& a, const float4& b, const float4& c, float* m) {
    m[0] = a.x; m[1] = a.y; m[2] = a.z;
    m[3] = b.x; m[4] = b.y; m[5] = b.z;
    m[6] = c.x; m[7] = c.y; m[8] = c.z;
}

template <bool RO>
__device__ __forceinline__ float4 ld4(const float4* p) {
    if (RO) return __ldg(p);
    return *p;
}

// loads record words 0..7 (position, velocity, mass, Fe, Fp) and, with
// want_dx_d, words 8..11 (displacement, D) of work slot t
template <bool RO>
__device__ __forceinline__ void load_particle(const float4* w, size_t n, uint32_t t, PState& s, bool want_dx_d) {
    const float4* r = w + t;
    float4 q0 = ld4<RO>(r), q1 = ld4<RO>(r + n);
    s.pos[0] = q0.x; s.pos[1] = q0.y; s.pos[2] = q0.z; s.hom = q0.w;
    s.vel[0] = q1.x; s.vel[1] = q1.y; s.vel[2] = q1.z; s.mass = q1.w;
    unpack_m(ld4<RO>(r + 2 * n), ld4<RO>(r + 3 * n), ld4<RO>(r + 4 * n), s.Fe);
    unpack_m(ld4<RO>(r + 5 * n), ld4<RO>(r + 6 * n), ld4<RO>(r + 7 * n), s.Fp);
    if (want_dx_d) {
        float4 q8 = ld4<RO>(r + 8 * n);
        s.dxp[0] = q8.x; s.dxp[1] = q8.y; s.dxp[2] = q8.z;
        unpack_m(ld4<RO>(r + 9 * n), ld4<RO>(r + 10 * n), ld4<RO>(r + 11 * n), s.D);
    }
}

// the record words a G2P + integrate writes (padding words 0, the position's
// fourth word kept), streamed past L1
__device__ __forceinline__ void store_particle(float4* w, size_t n, uint32_t t, const PState& s) {
    float4* r = w + t;
    __stcs(r, make_float4(s.pos[0], s.pos[1], s.pos[2], s.hom));
    __stcs(r + n, make_float4(s.vel[0], s.vel[1], s.vel[2], s.mass));
    __stcs(r + 2 * n, make_float4(s.Fe[0], s.Fe[1], s.Fe[2], 0.f));
    __stcs(r + 3 * n, make_float4(s.Fe[3], s.Fe[4], s.Fe[5], 0.f));
    __stcs(r + 4 * n, make_float4(s.Fe[6], s.Fe[7], s.Fe[8], 0.f));
    __stcs(r + 5 * n, make_float4(s.Fp[0], s.Fp[1], s.Fp[2], 0.f));
    __stcs(r + 6 * n, make_float4(s.Fp[3], s.Fp[4], s.Fp[5], 0.f));
    __stcs(r + 7 * n, make_float4(s.Fp[6], s.Fp[7], s.Fp[8], 0.f));
    __stcs(r + 8 * n, make_float4(s.dxp[0], s.dxp[1], s.dxp[2], 0.f));
    __stcs(r + 9 * n, make_float4(s.D[0], s.D[1], s.D[2], 0.f));
    __stcs(r + 10 * n, make_float4(s.D[3], s.D[4], s.D[5], 0.f));
    __stcs(r + 11 * n, make_float4(s.D[6], s.D[7], s.D[8], 0.f));
}

// cell number, fractional position, quadratic B-spline weights
// (mpmOps.wgsl:14-53)
struct Stencil {
    int cell[3];
    float f[3];
    float w[3][3];   // w[k][axis], k = offset + 1
};

__device__ __forceinline__ void make_stencil(const SceneDev& S, const float* pos, Stencil& st) {
#pragma unroll
    for (int i = 0; i < 3; i++) st.cell[i] = f2i(fm(fs(pos[i], S.gmin[i]), S.rcd[i]));
#pragma unroll
    for (int i = 0; i < 3; i++) {
        float mn = ff(S.cd[i], i2f(st.cell[i]), S.gmin[i]);
        float f = fm(fs(pos[i], mn), S.rcd[i]);
        st.f[i] = f;
        float om = fs(1.0f, f);
        st.w[0][i] = fm(fm(0.5f, om), om);
        float h = fs(f, 0.5f);
        st.w[1][i] = ff(-h, h, 0.75f);
        st.w[2][i] = fm(fm(0.5f, f), f);
    }
}

__device__ __forceinline__ float dwk(int k, float f) {
    // derivative of the B-spline weights wrt the fractional position
    return k == 0 ? fs(f, 1.0f) : (k == 1 ? fm(-2.0f, fs(f, 0.5f)) : f);
}

// ------------------------------------------------------------------
// constitutive pieces
// ------------------------------------------------------------------
// hardenLameParameters + calculateStressFirstPiolaKirchhoff
// (stressTensorOps.wgsl:9-22, 39-56); returns M = (-V) * P^T.
__device__ __forceinline__ void stress_matrix(const SceneDev& S, const PState& p, float* M) {
    float Jp = det3(p.Fp);
    float ef = expf_m(fm(S.xi_e, fs(1.0f, Jp)));
    float mu = fm(S.mu0, ef);
    float la = fm(S.la0, ef);
    float J = det3(p.Fe);
    float R[9], Fi[9];
    polar3(p.Fe, R);
    inv3(p.Fe, Fi);
    float a = fm(2.0f, mu);
    float b = fm(fm(la, fs(J, 1.0f)), J);
    float V = fm(p.mass, S.inv_rho);
    float nV = -V;
    // P[c][r] = a*(F[c][r]-R[c][r]) + b*Fi^T[c][r], Fi^T[c][r] = Fi[r][c]
    // M[c][r] = (-V) * P^T[c][r] = (-V) * P[r][c]
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            float Prc = ff(b, Fi[c * 3 + r], fm(a, fs(p.Fe[r * 3 + c], R[r * 3 + c])));
            M[c * 3 + r] = fm(nV, Prc);
        }
}

// elasticity relaxation factor 0.5 + 0.5 (1 - exp(-xi / det Fp)) (pbmpm.wgsl:29-35)
__device__ __forceinline__ float pbmpm_relax(const SceneDev& S, const float* Fp) {
    float J = det3(Fp);
    return ff(0.5f, fs(1.0f, expf_m(fd(-S.xi_p, J))), 0.5f);
}

// solveParticleConstraints (pbmpm.wgsl:16-39): updates D, given Fe, its
// inverse and the relaxation factor (both fixed within a substep).
__device__ __forceinline__ void pbmpm_constraints(const SceneDev& S, const float* Fe, const float* Fei, float relax,
                                                  float* D) {
    float IpD[9], Ft[9], Rt[9];
#pragma unroll
    for (int i = 0; i < 9; i++) IpD[i] = fa((i == 0 || i == 4 || i == 8) ? 1.0f : 0.0f, D[i]);
    mul3(IpD, Fe, Ft);
    polar3(Ft, Rt);
    float tv = det3(Ft);
    float vs = powf_m(fabsf(tv), S.vexp);
    float ob = fs(1.0f, S.blend);
    float tb[9], Dc[9];
    // tb = blend (R vs) + (1 - blend) R, D += relax (Dc - I - D), in pairs
    const float2 vs2 = dup2(vs), ob2 = dup2(ob), bl2 = dup2(S.blend), rx2 = dup2(relax);
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const float2 r = make_float2(Rt[i], Rt[i + 1]);
        const float2 v = ff2(bl2, fm2(r, vs2), fm2(ob2, r));
        tb[i] = v.x;
        tb[i + 1] = v.y;
    }
    tb[8] = ff(S.blend, fm(Rt[8], vs), fm(ob, Rt[8]));
    mul3(tb, Fei, Dc);
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        const float2 id = make_float2((i == 0 || i == 4) ? 1.0f : 0.0f, (i + 1 == 4) ? 1.0f : 0.0f);
        const float2 d = make_float2(D[i], D[i + 1]);
        const float2 v = ff2(rx2, fa2(fa2(make_float2(Dc[i], Dc[i + 1]), neg2(id)), neg2(d)), d);
        D[i] = v.x;
        D[i + 1] = v.y;
    }
    D[8] = ff(relax, fs(fs(Dc[8], 1.0f), D[8]), D[8]);
}

// applyPlasticity (plasticityOps.wgsl:7-48), in mpm_plast.cuh
__device__ __forceinline__ void plasticity(const SceneDev& S, float* Fe, float* Fp) {
    plasticity_exact(S.smin, S.smax, Fe, Fp);
}

// ------------------------------------------------------------------
// collider (colliderPrelude.wgsl:29-356)
// ------------------------------------------------------------------
__device__ __forceinline__ void col_vertex(const SceneDev& S, uint32_t idx, float* v) {
    uint32_t base = S.c_nidx + idx * 3u;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        uint32_t w = (base + (uint32_t)k < S.col_words) ? __ldg(&S.col_data[base + k]) : 0u;
        v[k] = __uint_as_float(w);
    }
}

__device__ void closest_point_tri(const float* p, const float* a, const float* b, const float* c, float* o) {
    float ab[3], ac[3], ap[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { ab[k] = fs(b[k], a[k]); ac[k] = fs(c[k], a[k]); ap[k] = fs(p[k], a[k]); }
    float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) { o[0] = a[0]; o[1] = a[1]; o[2] = a[2]; return; }
    float bp[3];
#pragma unroll
    for (int k = 0; k < 3; k++) bp[k] = fs(p[k], b[k]);
    float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.f && d4 <= d3) { o[0] = b[0]; o[1] = b[1]; o[2] = b[2]; return; }
    float vc = fs(fm(d1, d4), fm(d3, d2));
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        float v = fd(d1, fs(d1, d3));
#pragma unroll
        for (int k = 0; k < 3; k++) o[k] = fa(a[k], fm(v, ab[k]));
        return;
    }
    float cp[3];
#pragma unroll
    for (int k = 0; k < 3; k++) cp[k] = fs(p[k], c[k]);
    float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.f && d5 <= d6) { o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; return; }
    float vb = fs(fm(d5, d2), fm(d1, d6));
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        float w = fd(d2, fs(d2, d6));
#pragma unroll
        for (int k = 0; k < 3; k++) o[k] = fa(a[k], fm(w, ac[k]));
        return;
    }
    float va = fs(fm(d3, d6), fm(d5, d4));
    if (va <= 0.f && fs(d4, d3) >= 0.f && fs(d5, d6) >= 0.f) {
        float w = fd(fs(d4, d3), fa(fs(d4, d3), fs(d5, d6)));
#pragma unroll
        for (int k = 0; k < 3; k++) o[k] = fa(b[k], fm(w, fs(c[k], b[k])));
        return;
    }
    float denom = fd(1.0f, fa(fa(va, vb), vc));
    float v = fm(vb, denom), w = fm(vc, denom);
#pragma unroll
    for (int k = 0; k < 3; k++) o[k] = fa(fa(a[k], fm(v, ab[k])), fm(w, ac[k]));
}

__device__ float ray_tri(const float* org, const float* dir, const float* a, const float* b, const float* c) {
    const float EPS = 1e-6f;
    float e1[3], e2[3], h[3], sv[3], q[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { e1[k] = fs(b[k], a[k]); e2[k] = fs(c[k], a[k]); }
    cross3(dir, e2, h);
    float aa = dot3(e1, h);
    if (aa > -EPS && aa < EPS) return -1.f;
    float f = fd(1.0f, aa);
#pragma unroll
    for (int k = 0; k < 3; k++) sv[k] = fs(org[k], a[k]);
    float u = fm(f, dot3(sv, h));
    if (u < 0.f || u > 1.f) return -1.f;
    cross3(sv, e1, q);
    float v = fm(f, dot3(dir, q));
    if (v < 0.f || fa(u, v) > 1.f) return -1.f;
    float t = fm(f, dot3(e2, q));
    if (t > EPS) return t;
    return -1.f;
}

__device__ void collide(const SceneDev& S, PState& p, Counters* ctr) {
    if (S.n_nodes == 0u) return;
    float mnb[3], mxb[3];
    xform_point(S.xf, S.cmin, mnb);
    xform_point(S.xf, S.cmax, mxb);
    const float margin = S.cmargin;
    float cur[3], prev[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { cur[k] = p.pos[k]; prev[k] = fs(cur[k], p.dxp[k]); }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float smin = fs(fminf(mnb[k], mxb[k]), margin);
        float smax = fa(fmaxf(mnb[k], mxb[k]), margin);
        if (fminf(cur[k], prev[k]) > smax || fmaxf(cur[k], prev[k]) < smin) return;
    }
    if (S.c_nobj == 0u) return;

    float min_d2 = 1e20f;
    float cnorm[3] = {0.f, 0.f, 1.f}, cpos[3] = {cur[0], cur[1], cur[2]};
    float min_t = 1.f;
    float hnorm[3] = {0.f, 0.f, 1.f}, hpos[3] = {cur[0], cur[1], cur[2]};
    bool has_hit = false;
    float rd[3] = {p.dxp[0], p.dxp[1], p.dxp[2]};
    const float rd_len = len3(rd);
    bool do_ccd = rd_len > 1e-4f;
    float curl[3], prevl[3], pminl[3], pmaxl[3];
    xform_point(S.xfi, cur, curl);
    xform_point(S.xfi, prev, prevl);
#pragma unroll
    for (int k = 0; k < 3; k++) { pminl[k] = fminf(curl[k], prevl[k]); pmaxl[k] = fmaxf(curl[k], prevl[k]); }

    // Early skip (identity transform only): a triangle whose bounds are
    // farther than the threshold (plus a rounding allowance) from the
    // particle and do not meet its path can neither bring the closest
    // distance under the threshold nor be hit by the path, so it cannot
    // change the outcome; the other triangles run in the same order.
    const float slack = fa(1e-4f, fm(1e-5f, fmaxf(fmaxf(fabsf(cur[0]), fabsf(cur[1])), fabsf(cur[2]))));
    const float reach = fa(S.cthr, slack);
    const float reach2 = fm(reach, reach);
    // Whole-query skip (identity transform only): when the collider's
    // distance field bounds the distance from the particle to every triangle
    // from below by more than the threshold plus the path length, every point
    // of the path is farther than the threshold from every triangle, so no
    // triangle can bring the closest distance under the threshold and the path
    // hits none: the query's outcome is "unchanged" without traversing.
    if (S.cull && S.dfield != nullptr) {
        bool in = true;
        uint32_t fc[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float u = fm(fs(cur[k], S.df_lo[k]), S.df_rcs[k]);
            in = in && u >= 0.f && u < (float)S.df_res;
            fc[k] = in ? (uint32_t)u : 0u;
        }
        if (in && fc[0] < S.df_res && fc[1] < S.df_res && fc[2] < S.df_res) {
            const float lb = __ldg(S.dfield + ((size_t)fc[2] * S.df_res + fc[1]) * S.df_res + fc[0]);
            if (lb > fa(reach, rd_len)) return;
        }
    }
    float seg_lo[3], seg_hi[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        seg_lo[k] = fs(fminf(cur[k], prev[k]), slack);
        seg_hi[k] = fa(fmaxf(cur[k], prev[k]), slack);
    }
    uint32_t stack[32];
    uint32_t sp = 0;
    stack[sp++] = 0u;
    // a well-formed tree visits each node at most once; the cap only ends
    // traversal of a malformed (cyclic) node array
    uint32_t visits = 0, max_visits = 2u * S.n_nodes + 64u;
    while (sp > 0u) {
        if (++visits > max_visits) { atomicOr(&ctr->status, ST_BVH_STACK); break; }
        uint32_t ni = stack[--sp];
        if (ni >= S.n_nodes) continue;
        const uint4* nd = reinterpret_cast<const uint4*>(S.bvh + (size_t)ni * 8);
        uint4 n0 = __ldg(nd), n1 = __ldg(nd + 1);
        float bmin0 = fs(__uint_as_float(n0.x), margin), bmin1 = fs(__uint_as_float(n0.y), margin), bmin2 = fs(__uint_as_float(n0.z), margin);
        float bmax0 = fa(__uint_as_float(n1.x), margin), bmax1 = fa(__uint_as_float(n1.y), margin), bmax2 = fa(__uint_as_float(n1.z), margin);
        if (pminl[0] > bmax0 || pminl[1] > bmax1 || pminl[2] > bmax2 ||
            pmaxl[0] < bmin0 || pmaxl[1] < bmin1 || pmaxl[2] < bmin2) continue;
        if (n1.w & 0x80000000u) {
            uint32_t start = n0.w, end = start + (n1.w & 0x7FFFFFFFu);
            for (uint32_t i = start; i < end; i++) {
                uint32_t tb = i * 3u;
                if (tb + 2u >= S.col_words) break;
                if (S.cull) {
                    const float4 blo = __ldg(S.tbox + 2 * i), bhi = __ldg(S.tbox + 2 * i + 1);
                    const float lo3[3] = {blo.x, blo.y, blo.z}, hi3[3] = {bhi.x, bhi.y, bhi.z};
                    float dl = 0.f;
                    bool apart = false;
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        float gap = fmaxf(0.f, fmaxf(fs(lo3[k], cur[k]), fs(cur[k], hi3[k])));
                        dl = fa(dl, fm(gap, gap));
                        apart = apart || seg_hi[k] < lo3[k] || seg_lo[k] > hi3[k];
                    }
                    if (dl > reach2 && (!do_ccd || apart)) continue;
                }
                float v0l[3], v1l[3], v2l[3], v0[3], v1[3], v2[3];
                col_vertex(S, __ldg(&S.col_data[tb]), v0l);
                col_vertex(S, __ldg(&S.col_data[tb + 1]), v1l);
                col_vertex(S, __ldg(&S.col_data[tb + 2]), v2l);
                xform_point(S.xf, v0l, v0);
                xform_point(S.xf, v1l, v1);
                xform_point(S.xf, v2l, v2);
                float cp[3], df[3];
                closest_point_tri(cur, v0, v1, v2, cp);
#pragma unroll
                for (int k = 0; k < 3; k++) df[k] = fs(cur[k], cp[k]);
                float d2 = dot3(df, df);
                if (d2 < min_d2) {
                    min_d2 = d2;
                    cpos[0] = cp[0]; cpos[1] = cp[1]; cpos[2] = cp[2];
                    float e1[3], e2[3], n[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) { e1[k] = fs(v1[k], v0[k]); e2[k] = fs(v2[k], v0[k]); }
                    cross3(e1, e2, n);
                    float ln = len3(n);
                    if (ln > 1e-6f) {
#pragma unroll
                        for (int k = 0; k < 3; k++) cnorm[k] = fd(n[k], ln);
                    }
                }
                if (do_ccd) {
                    float t = ray_tri(prev, rd, v0, v1, v2);
                    if (t > 0.f && t < min_t) {
                        min_t = t;
                        has_hit = true;
#pragma unroll
                        for (int k = 0; k < 3; k++) hpos[k] = fa(prev[k], fm(rd[k], t));
                        float e1[3], e2[3], n[3];
#pragma unroll
                        for (int k = 0; k < 3; k++) { e1[k] = fs(v1[k], v0[k]); e2[k] = fs(v2[k], v0[k]); }
                        cross3(e1, e2, n);
                        float ln = len3(n);
                        float fn[3] = {fd(n[0], ln), fd(n[1], ln), fd(n[2], ln)};
                        float dd = dot3(rd, fn);
                        float sg = dd > 0.f ? 1.f : (dd < 0.f ? -1.f : 0.f);
#pragma unroll
                        for (int k = 0; k < 3; k++) hnorm[k] = fm(fn[k], sg);
                    }
                }
            }
        } else {
            if (sp < 31u) {
                stack[sp++] = n0.w;
                stack[sp++] = n1.w;
            } else {
                atomicOr(&ctr->status, ST_BVH_STACK);
            }
        }
    }
    float vsf = fm(S.cvs, S.rdt);
    if (has_hit) {
        float nvv[3], vr[3];
#pragma unroll
        for (int k = 0; k < 3; k++) p.pos[k] = fa(hpos[k], fm(hnorm[k], S.csurf));
#pragma unroll
        for (int k = 0; k < 3; k++) vr[k] = fs(fm(p.dxp[k], S.rdt), S.cvel[k]);
        float vn = dot3(vr, hnorm);
        float om = fs(1.0f, S.cfric);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float vt = fs(vr[k], fm(vn, hnorm[k]));
            nvv[k] = vn < 0.f ? fa(fm(vt, om), fm(S.cvel[k], vsf)) : fa(vr[k], fm(S.cvel[k], vsf));
        }
#pragma unroll
        for (int k = 0; k < 3; k++) { p.vel[k] = nvv[k]; p.dxp[k] = fm(nvv[k], S.dt); }
        return;
    }
    float dist = __fsqrt_rn(min_d2);
    float df[3], pd[3] = {cnorm[0], cnorm[1], cnorm[2]};
#pragma unroll
    for (int k = 0; k < 3; k++) df[k] = fs(cur[k], cpos[k]);
    float ld = len3(df);
    if (ld > 1e-6f) {
#pragma unroll
        for (int k = 0; k < 3; k++) pd[k] = fd(df[k], ld);
    }
    if (dist < S.cthr) {
        float nvv[3], vr[3];
#pragma unroll
        for (int k = 0; k < 3; k++) vr[k] = fs(fm(p.dxp[k], S.rdt), S.cvel[k]);
        float vn = dot3(vr, pd);
        float om = fs(1.0f, 0.0f);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float vt = fs(vr[k], fm(vn, pd[k]));
            nvv[k] = vn < 0.f ? fa(fm(vt, om), fm(S.cvel[k], vsf)) : fa(vr[k], fm(S.cvel[k], vsf));
        }
#pragma unroll
        for (int k = 0; k < 3; k++) { p.vel[k] = nvv[k]; p.dxp[k] = fm(nvv[k], S.dt); }
        if (dist < S.csurf) {
#pragma unroll
            for (int k = 0; k < 3; k++) p.pos[k] = fa(cpos[k], fm(pd[k], S.csurf));
        }
    }
}

// Appends particle pid to the deferred plasticity list (warp-aggregated).
__device__ __forceinline__ void defer_plasticity(const Ctx& c, uint32_t pid) {
    unsigned m = __activemask();
    int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&c.counters->n_plast, (uint32_t)__popc(m));
    base = __shfl_sync(m, base, leader);
    c.plast_list[base + (uint32_t)__popc(m & lanemask_lt())] = pid;
}

// integrateParticles (integrateParticles.wgsl:14-72).  The return map runs
// only for particles the strain-bound check does not clear (for the others it
// returns Fe and Fp unchanged, bit for bit).  With deferred plasticity the
// record keeps the trial Fe and those particles are listed for the plasticity
// pass (exact or learned).
__device__ __forceinline__ void integrate(const Ctx& c, const SceneDev& S, PState& p, uint32_t pid) {
    Counters* ctr = c.counters;
#pragma unroll
    for (int k = 0; k < 3; k++) p.pos[k] = fa(p.pos[k], p.dxp[k]);
    float IpD[9];
#pragma unroll
    for (int i = 0; i < 9; i++) IpD[i] = fa((i == 0 || i == 4 || i == 8) ? 1.0f : 0.0f, p.D[i]);
    mul3(IpD, p.Fe, p.Fe);
    const bool certified = cert_elastic(S.smin, S.smax, p.Fe);
    if (c.plast_defer) {
        if (!certified) defer_plasticity(c, pid);
    } else if (!certified) {
        plasticity(S, p.Fe, p.Fp);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (p.pos[a] < S.gmin[a]) { p.dxp[a] = fm(p.dxp[a], S.rest); p.pos[a] = S.gmin[a]; p.vel[a] = fm(p.vel[a], S.rest); }
        if (p.pos[a] >= S.gmax[a]) { p.dxp[a] = fm(p.dxp[a], S.rest); p.pos[a] = S.gmax[a]; p.vel[a] = fm(p.vel[a], S.rest); }
    }
    collide(S, p, ctr);
}

// ------------------------------------------------------------------
// binning kernels
// ------------------------------------------------------------------
__global__ void k_clear_table(Ctx c) {
    uint32_t n = c.counters->n_st;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c.counters->n_plast = 0u;
        c.counters->step += 1u;
        c.counters->tile_ticket = 0u;
        c.counters->tile_done = 0u;
        c.counters->n_carry = 0u;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t s = c.st_slot[i];
        c.keys[s] = KEY_EMPTY;
        c.slot_count[s] = 0u;
    }
}

template <int E>
__global__ void __launch_bounds__(256) k_bin_insert(Ctx c) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    bool act = t < c.n_particles;
    uint64_t key = KEY_EMPTY;
    uint32_t scene = 0;
    int st[3] = {0, 0, 0};
    if (act) {
        float4 q0 = __ldg(c.work_in + t);
        scene = c.n_scenes > 1u ? find_scene(c, __ldg(c.ids_in + t)) : 0u;
        const SceneDev* S = c.scenes + scene;
        float pos[3] = {q0.x, q0.y, q0.z};
#pragma unroll
        for (int i = 0; i < 3; i++) {
            int cell = f2i(fm(fs(pos[i], __ldg(&S->gmin[i])), __ldg(&S->rcd[i])));
            int res = __ldg(&S->res[i]);
            // cells below -1 or above res reach no grid cell; clamping them
            // only decides which tile processes the particle
            cell = max(-2, min(cell, res + 1));
            st[i] = floor_div<E>(cell);
        }
        key = pack_key(scene, st[0], st[1], st[2]);
    }
    unsigned am = __ballot_sync(0xffffffffu, act);
    if (!act) return;
    unsigned grp = __match_any_sync(am, key);
    int leader = __ffs(grp) - 1;
    int lane = threadIdx.x & 31;
    uint32_t slot = 0, base = 0;
    if (lane == leader) {
        slot = tile_insert(c, key, scene, st[0], st[1], st[2]);
        base = (slot != INVALID) ? atomicAdd(&c.slot_count[slot], (uint32_t)__popc(grp)) : 0u;
    }
    slot = __shfl_sync(grp, slot, leader);
    base = __shfl_sync(grp, base, leader);
    c.bin_slot[t] = slot;
    c.bin_rank[t] = base + (uint32_t)__popc(grp & lanemask_lt());
}

// per chunk of COMPACT_CHUNK slots: number of occupied slots and particles
__global__ void __launch_bounds__(256) k_compact_a(Ctx c) {
    uint32_t base = blockIdx.x * COMPACT_CHUNK + threadIdx.x * 16u;
    uint32_t ns = 0, np = 0;
#pragma unroll 4
    for (int i = 0; i < 16; i++) {
        if (c.keys[base + i] != KEY_EMPTY) { ns++; np += c.slot_count[base + i]; }
    }
    __shared__ uint32_t r_ns[8], r_np[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { ns += __shfl_xor_sync(0xffffffffu, ns, o); np += __shfl_xor_sync(0xffffffffu, np, o); }
    if ((threadIdx.x & 31) == 0) { r_ns[threadIdx.x >> 5] = ns; r_np[threadIdx.x >> 5] = np; }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0, b = 0;
        for (int w = 0; w < 8; w++) { a += r_ns[w]; b += r_np[w]; }
        c.chunk_nst[blockIdx.x] = a;
        c.chunk_np[blockIdx.x] = b;
    }
}

// exclusive scan of the chunk totals (one block of 1024 threads)
__global__ void __launch_bounds__(1024) k_compact_b(Ctx c, uint32_t n_chunks) {
    __shared__ uint32_t s_ns[32], s_np[32];
    __shared__ uint32_t carry_ns, carry_np;
    if (threadIdx.x == 0) { carry_ns = 0; carry_np = 0; }
    __syncthreads();
    for (uint32_t base = 0; base < n_chunks; base += 1024u) {
        uint32_t i = base + threadIdx.x;
        uint32_t vns = i < n_chunks ? c.chunk_nst[i] : 0u;
        uint32_t vnp = i < n_chunks ? c.chunk_np[i] : 0u;
        uint32_t ins = vns, inp = vnp;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t a = __shfl_up_sync(0xffffffffu, ins, o), b = __shfl_up_sync(0xffffffffu, inp, o);
            if (lane >= o) { ins += a; inp += b; }
        }
        if (lane == 31) { s_ns[w] = ins; s_np[w] = inp; }
        __syncthreads();
        if (w == 0) {
            uint32_t a = s_ns[lane], b = s_np[lane];
            uint32_t xa = a, xb = b;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t ta = __shfl_up_sync(0xffffffffu, xa, o), tb = __shfl_up_sync(0xffffffffu, xb, o);
                if (lane >= o) { xa += ta; xb += tb; }
            }
            s_ns[lane] = xa - a;
            s_np[lane] = xb - b;
        }
        __syncthreads();
        uint32_t ex_ns = carry_ns + s_ns[w] + ins - vns;
        uint32_t ex_np = carry_np + s_np[w] + inp - vnp;
        if (i < n_chunks) { c.chunk_nst[i] = ex_ns; c.chunk_np[i] = ex_np; }
        __syncthreads();
        if (threadIdx.x == 1023) { carry_ns = ex_ns + vns; carry_np = ex_np + vnp; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c.counters->n_st = carry_ns;
        c.counters->n_binned = carry_np;
        if (carry_ns > c.max_tiles) atomicOr(&c.counters->status, ST_TILE_OVERFLOW);
    }
}

// compact tile records in slot order
__global__ void __launch_bounds__(256) k_compact_c(Ctx c) {
    uint32_t base = blockIdx.x * COMPACT_CHUNK + threadIdx.x * 16u;
    uint32_t ns = 0, np = 0;
    unsigned long long k[16];
    uint32_t cnt[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        k[i] = c.keys[base + i];
        cnt[i] = (k[i] != KEY_EMPTY) ? c.slot_count[base + i] : 0u;
        ns += (k[i] != KEY_EMPTY) ? 1u : 0u;
        np += cnt[i];
    }
    // block exclusive scan of (ns, np)
    __shared__ uint32_t w_ns[8], w_np[8];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t ins = ns, inp = np;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t a = __shfl_up_sync(0xffffffffu, ins, o), b = __shfl_up_sync(0xffffffffu, inp, o);
        if (lane >= o) { ins += a; inp += b; }
    }
    if (lane == 31) { w_ns[w] = ins; w_np[w] = inp; }
    __syncthreads();
    uint32_t pre_ns = c.chunk_nst[blockIdx.x], pre_np = c.chunk_np[blockIdx.x];
    for (int j = 0; j < w; j++) { pre_ns += w_ns[j]; pre_np += w_np[j]; }
    uint32_t st = pre_ns + ins - ns;
    uint32_t off = pre_np + inp - np;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        if (k[i] != KEY_EMPTY) {
            uint32_t s = base + i;
            c.slot_st[s] = st;
            c.slot_off[s] = off;
            c.st_slot[st] = s;
            c.st_key[st] = k[i];
            c.st_begin[st] = off;
            c.st_count[st] = cnt[i];
            st++;
            off += cnt[i];
        }
    }
}

// Places work slot t at its position in this substep's tile order.  A
// particle that no tile kernel will advance (no hash slot, or a tile past the
// tile storage: both reported in the status) is copied unchanged to its
// output slot, so the state stays complete.
__global__ void __launch_bounds__(256) k_bin_scatter(Ctx c) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= c.n_particles) return;
    uint32_t slot = c.bin_slot[t];
    uint32_t dst;
    bool carry;
    if (slot == INVALID) {
        dst = c.counters->n_binned + atomicAdd(&c.counters->n_carry, 1u);
        carry = true;
    } else {
        dst = c.slot_off[slot] + c.bin_rank[t];
        c.sorted[dst] = t;
        carry = c.slot_st[slot] >= c.max_tiles;
    }
    if (carry) {
        const size_t n = c.n_particles;
#pragma unroll
        for (int q = 0; q < REC_PLANES; q++) c.work_out[q * n + dst] = c.work_in[q * n + t];
        c.ids_out[dst] = c.ids_in[t];
    }
}

// ------------------------------------------------------------------
// tile helpers
// ------------------------------------------------------------------
template <int E>
struct TileCtx {
    uint32_t scene;
    int origin[3];  // first core cell
    uint64_t key;
};

template <int E>
__device__ __forceinline__ void tile_begin(const Ctx& c, uint32_t st, SceneDev& S, TileCtx<E>& T, uint32_t& cur_scene) {
    uint64_t key = c.st_key[st];
    uint32_t scene;
    int sx, sy, sz;
    unpack_key(key, scene, sx, sy, sz);
    T.scene = scene;
    T.key = key;
    T.origin[0] = sx * E; T.origin[1] = sy * E; T.origin[2] = sz * E;
    if (scene != cur_scene) {
        __syncthreads();
        load_scene_smem(S, c.scenes + scene);
        cur_scene = scene;
    }
}

__device__ __forceinline__ int4 add4(int4 s, int4 v) {
    s.x = (int)((uint32_t)s.x + (uint32_t)v.x);
    s.y = (int)((uint32_t)s.y + (uint32_t)v.y);
    s.z = (int)((uint32_t)s.z + (uint32_t)v.z);
    s.w = (int)((uint32_t)s.w + (uint32_t)v.w);
    return s;
}

// Sum of all tile halos covering cell j of this tile's (E+2)^3 region, read
// cell by cell from global memory (inspection kernel only).
template <int E>
__device__ __forceinline__ int4 assemble_cell(const int4* tiles, const int* nbr, int j) {
    constexpr int H = E + 2, NC = H * H * H;
    int lx = j % H, ly = (j / H) % H, lz = j / (H * H);
    int4 s = __ldg(&tiles[(size_t)nbr[13] * NC + j]);
    int dx0 = lx <= 1 ? -1 : 0, dx1 = lx >= E ? 1 : 0;
    int dy0 = ly <= 1 ? -1 : 0, dy1 = ly >= E ? 1 : 0;
    int dz0 = lz <= 1 ? -1 : 0, dz1 = lz >= E ? 1 : 0;
    for (int dz = dz0; dz <= dz1; dz++)
        for (int dy = dy0; dy <= dy1; dy++)
            for (int dx = dx0; dx <= dx1; dx++) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                int t = nbr[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
                if (t < 0) continue;
                int jj = ((lz - E * dz) * H + (ly - E * dy)) * H + (lx - E * dx);
                s = add4(s, __ldg(&tiles[(size_t)t * NC + jj]));
            }
    return s;
}

// Compact indices of this tile's 27 neighbours (built by k_tile_nbr) into
// shared memory; d = 9(dz+1) + 3(dy+1) + (dx+1), -1 where no tile exists.
__device__ __forceinline__ void load_neighbors(const Ctx& c, uint32_t st, int* nbr) {
    if (threadIdx.x < 27) nbr[threadIdx.x] = __ldg(&c.st_nbr[(size_t)st * 27u + threadIdx.x]);
}

// Cell velocity the G2P kernels read.  Explicit mode first applies the grid
// update (gridUpdate.cs.wgsl:15-53) with its i32 round trip; PBMPM reads the
// transferred momentum directly (gridToParticle.cs.wgsl:102-108).  Cells the
// reference skips (outside the grid, or mass <= 0) get velocity 0.
template <bool PB>
__device__ __forceinline__ float4 cell_velocity(const SceneDev& S, int4 s, const int* gc) {
    bool in = gc[0] >= 0 && gc[1] >= 0 && gc[2] >= 0 && gc[0] < S.res[0] && gc[1] < S.res[1] && gc[2] < S.res[2];
    float cm = inv_s(S, s.x);
    if (!in || cm <= 0.0f) return make_float4(0.f, 0.f, 0.f, 0.f);
    float rm = __frcp_rn(cm);
    int32_t mi[3] = {s.y, s.z, s.w};
    if (!PB) {
        float u[3];
#pragma unroll
        for (int k = 0; k < 3; k++) u[k] = fa(fm(inv_s(S, mi[k]), rm), S.gdt[k]);
        grid_bc(S, gc, u);
#pragma unroll
        for (int k = 0; k < 3; k++) mi[k] = f2i(fm(fm(u[k], cm), S.scale));
    }
    float v[3];
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] = fm(inv_s(S, mi[k]), rm);
    if (PB) grid_bc(S, gc, v);
    return make_float4(v[0], v[1], v[2], 0.f);
}

// The parts of the 26 neighbour tiles' halos that overlap this tile's
// (E+2)^3 region, flattened into one index space: 6 face slabs (2 x H x H),
// then 12 edge bars (2 x 2 x H), then 8 corner cubes (2 x 2 x 2).  Entry e
// maps to the neighbour direction d (0..26), the cell j of this region and
// the cell jj of the neighbour's region; every divisor is a compile-time
// constant.
template <int E>
struct HaloEntries {
    static constexpr int H = E + 2;
    static constexpr int FACE = 2 * H * H, EDGE = 4 * H;
    static constexpr int NF = 6 * FACE, NED = 12 * EDGE;
    static constexpr int N = NF + NED + 64;
};

template <int E>
__host__ __device__ constexpr void halo_entry(int e, int& d, int& j, int& jj) {
    constexpr int H = E + 2;
    using HE = HaloEntries<E>;
    int dx = 0, dy = 0, dz = 0, ix = 0, iy = 0, iz = 0;
    if (e < HE::NF) {
        int r = e / HE::FACE, o = e - r * HE::FACE;
        int axis = r >> 1, sg = (r & 1) ? 1 : -1;
        if (axis == 0) { ix = o & 1; iy = (o >> 1) % H; iz = (o >> 1) / H; dx = sg; }
        else if (axis == 1) { ix = o % H; iy = (o / H) & 1; iz = o / (2 * H); dy = sg; }
        else { ix = o % H; iy = (o / H) % H; iz = o / (H * H); dz = sg; }
    } else if (e < HE::NF + HE::NED) {
        int e2 = e - HE::NF;
        int r = e2 / HE::EDGE, o = e2 - r * HE::EDGE;
        int za = r >> 2, s1 = (r & 1) ? 1 : -1, s2 = (r & 2) ? 1 : -1;
        if (za == 0) { ix = o % H; iy = (o / H) & 1; iz = o / (2 * H); dy = s1; dz = s2; }
        else if (za == 1) { ix = o & 1; iy = (o >> 1) % H; iz = (o >> 1) / H; dx = s1; dz = s2; }
        else { ix = o & 1; iy = (o >> 1) & 1; iz = o >> 2; dx = s1; dy = s2; }
    } else {
        int o = e - HE::NF - HE::NED;
        int r = o >> 3;
        o &= 7;
        dx = (r & 1) ? 1 : -1; dy = (r & 2) ? 1 : -1; dz = (r & 4) ? 1 : -1;
        ix = o & 1; iy = (o >> 1) & 1; iz = o >> 2;
    }
    int lx = (dx > 0 ? E : 0) + ix, ly = (dy > 0 ? E : 0) + iy, lz = (dz > 0 ? E : 0) + iz;
    j = (lz * H + ly) * H + lx;
    jj = ((lz - E * dz) * H + (ly - E * dy)) * H + (lx - E * dx);
    d = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
}

// The halo entries decoded once, at compile time: entry e packs its
// neighbour direction d (5 bits), its cell j in this tile's region (13 bits)
// and the cell jj in the neighbour's region (13 bits).
template <int E>
struct HaloTable {
    uint32_t v[HaloEntries<E>::N];
};
static_assert((18 * 18 * 18) < (1 << 13), "halo cell index must fit 13 bits");

template <int E>
__host__ __device__ constexpr HaloTable<E> make_halo_table() {
    HaloTable<E> t{};
    for (int e = 0; e < HaloEntries<E>::N; e++) {
        int d = 0, j = 0, jj = 0;
        halo_entry<E>(e, d, j, jj);
        t.v[e] = (uint32_t)d | ((uint32_t)j << 5) | ((uint32_t)jj << 18);
    }
    return t;
}

__device__ const HaloTable<8> g_halo8 = make_halo_table<8>();
__device__ const HaloTable<12> g_halo12 = make_halo_table<12>();
__device__ const HaloTable<14> g_halo14 = make_halo_table<14>();
__device__ const HaloTable<16> g_halo16 = make_halo_table<16>();

template <int E>
__device__ __forceinline__ const uint32_t* halo_table() {
    return E == 8 ? g_halo8.v : (E == 12 ? g_halo12.v : (E == 14 ? g_halo14.v : g_halo16.v));
}

// ---- TMA bulk copies into shared memory, completing on an mbarrier ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init1(uint64_t* mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
}
// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(mbar))
                 : "memory");
}
// waits for the phase of the given parity; false after `limit` polls
__device__ __forceinline__ bool mbar_wait_parity(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(mbar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
constexpr uint32_t COPY_WAIT_LIMIT = 1u << 22;

// Per-CTA state of the halo copies of the tile kernels: the mbarrier the
// bulk copies complete on and the parity of its current phase.
struct HaloCopy {
    uint64_t* mbar;
    uint32_t parity;
};

// Thread 0 issues the bulk copies of tile st's own (E+2)^3 sums into shared
// memory; they complete on hc's mbarrier.
template <int E>
__device__ __forceinline__ void halo_issue(const int4* tiles, uint32_t st, int4* cell, HaloCopy& hc) {
    constexpr int H = E + 2, NC = H * H * H;
    if (threadIdx.x == 0) {
        const int4* own = tiles + (size_t)st * NC;
        // the previous tile's shared-memory reads (generic proxy) come before these writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(hc.mbar, (uint32_t)(NC * 16));
        constexpr uint32_t CH = (NC * 16) / 4 / 16 * 16;   // four chunks, 16-byte multiples
        bulk_g2s(cell, own, CH, hc.mbar);
        bulk_g2s(reinterpret_cast<char*>(cell) + CH, reinterpret_cast<const char*>(own) + CH, CH, hc.mbar);
        bulk_g2s(reinterpret_cast<char*>(cell) + 2 * CH, reinterpret_cast<const char*>(own) + 2 * CH, CH, hc.mbar);
        bulk_g2s(reinterpret_cast<char*>(cell) + 3 * CH, reinterpret_cast<const char*>(own) + 3 * CH,
                 (uint32_t)(NC * 16) - 3 * CH, hc.mbar);
    }
}

// Sum this tile's halo region into `cell`: the tile's own (E+2)^3 sums (one
// TMA bulk copy) plus the overlapping parts of the neighbour halos (entries
// of the compile-time halo table, loaded into registers in batches of U per
// thread and added with shared i32 atomics).  The first batch of neighbour
// loads is issued before the wait for the bulk copy, so both latencies
// overlap.  MASS = false adds only the momentum components: the mass field
// of the result keeps the tile's own record (in the PBMPM iterations' halo
// records, the reciprocal cell mass).  Returns false (on every thread) when
// the copy wait ran out; the caller then stops.  PRE = true: the caller issued
// the own-halo copies earlier (halo_issue).
template <int E, int BS, bool MASS = true, bool PRE = false>
__device__ __forceinline__ bool assemble_sums(const int4* tiles, const int* nbr, int4* cell, HaloCopy& hc) {
    constexpr int H = E + 2, NC = H * H * H;
    constexpr int NE = HaloEntries<E>::N;
    constexpr int PER = (NE + BS - 1) / BS;      // entries per thread
    constexpr int U = PER <= 10 ? PER : 8;       // entries per register batch
    const uint32_t* tab = halo_table<E>();
    if (!PRE) halo_issue<E>(tiles, (uint32_t)nbr[13], cell, hc);
    int4 v[U];
    int jd[U];
    auto fetch = [&](int base) {
#pragma unroll
        for (int u = 0; u < U; u++) {
            int e = base + u * BS;
            jd[u] = -1;
            v[u] = make_int4(0, 0, 0, 0);
            if (e < NE) {
                uint32_t w = __ldg(tab + e);
                int t = nbr[w & 31u];
                if (t >= 0) {
                    v[u] = __ldg(tiles + (size_t)t * NC + (w >> 18));
                    jd[u] = (int)((w >> 5) & 0x1fffu);
                }
            }
        }
    };
    auto add = [&]() {
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (jd[u] >= 0) {
                int* dst = reinterpret_cast<int*>(&cell[jd[u]]);
                if (MASS) atomicAdd(dst + 0, v[u].x);
                atomicAdd(dst + 1, v[u].y);
                atomicAdd(dst + 2, v[u].z);
                atomicAdd(dst + 3, v[u].w);
            }
        }
    };
    fetch(threadIdx.x);
    bool ok = mbar_wait_parity(hc.mbar, hc.parity, COPY_WAIT_LIMIT);
    hc.parity ^= 1u;
    if (__syncthreads_or(ok ? 0 : 1)) return false;
    add();
    for (int base = threadIdx.x + U * BS; base < NE; base += U * BS) {
        fetch(base);
        add();
    }
    return true;
}

// Reciprocal cell mass RN(1 / m) of the velocity m^-1 p, 0 for the cells the
// reference skips (outside the grid or mass <= 0): a momentum scaled by 0
// gives a velocity of +-0, whose products add nothing to the G2P sums.
__device__ __forceinline__ float mass_recip(const SceneDev& S, int32_t m, const int* gc) {
    bool in = gc[0] >= 0 && gc[1] >= 0 && gc[2] >= 0 && gc[0] < S.res[0] && gc[1] < S.res[1] && gc[2] < S.res[2];
    float cm = inv_s(S, m);
    return (in && cm > 0.0f) ? __frcp_rn(cm) : 0.0f;
}

// PBMPM cell velocity from momentum and the reciprocal mass (gridToParticle.cs.wgsl:102-108)
__device__ __forceinline__ float4 cell_velocity_rm(const SceneDev& S, int4 s, float rm, const int* gc) {
    float v[3] = {fm(inv_s(S, s.y), rm), fm(inv_s(S, s.z), rm), fm(inv_s(S, s.w), rm)};
    grid_bc(S, gc, v);
    return make_float4(v[0], v[1], v[2], 0.f);
}

// Assemble this tile's (E+2)^3 cell velocities in shared memory: halo sums
// (assemble_sums), then each sum turned into the velocity in place.  RM
// selects where the cell masses come from: 0, the assembled mass sums (the
// reference path, explicit grid update included); 1, the same, and the
// reciprocal masses RN(1/m) are kept in rm_s for the tile's flush; 2, the
// reciprocal masses carried in the mass word of the tile's own halo record
// (written there by the previous PBMPM iteration's flush; the halo sums then
// carry momentum only), also kept in rm_s when it is given.  Returns false (on
// every thread) when the halo copy wait ran out.
template <int E, int BS, bool PB, int RM = 0, bool PRE = false>
__device__ __forceinline__ bool assemble_velocity_tile(const int4* tiles, const SceneDev& S, const TileCtx<E>& T,
                                                       const int* nbr, int4* cell, HaloCopy& hc,
                                                       float* rm_s = nullptr) {
    constexpr int H = E + 2, NC = H * H * H;
    if (!assemble_sums<E, BS, RM != 2, PRE>(tiles, nbr, cell, hc)) return false;
    __syncthreads();
    // batches of CB cells per thread: all loads, then all conversions, then
    // all stores, so the cells' dependency chains overlap
    constexpr int CB = (BS >= 512 && RM != 0) ? 4 : 1;
    for (int j0 = threadIdx.x; j0 < NC; j0 += CB * BS) {
        int4 sm[CB];
        float rmu[CB];
#pragma unroll
        for (int u = 0; u < CB; u++) {
            int j = j0 + u * BS;
            sm[u] = j < NC ? cell[j] : make_int4(0, 0, 0, 0);
            rmu[u] = (RM == 2 && j < NC) ? __int_as_float(sm[u].x) : 0.0f;
        }
        float4 v[CB];
#pragma unroll
        for (int u = 0; u < CB; u++) {
            int j = j0 + u * BS;
            int lx = j % H, ly = (j / H) % H, lz = j / (H * H);
            int gc[3] = {T.origin[0] - 1 + lx, T.origin[1] - 1 + ly, T.origin[2] - 1 + lz};
            if (RM == 0) {
                v[u] = cell_velocity<PB>(S, sm[u], gc);
            } else {
                float rm;
                if (RM == 1) {
                    rm = mass_recip(S, sm[u].x, gc);
                } else {
                    rm = rmu[u];
                }
                if (rm_s != nullptr && j < NC) rm_s[j] = rm;
                v[u] = cell_velocity_rm(S, sm[u], rm, gc);
            }
        }
#pragma unroll
        for (int u = 0; u < CB; u++) {
            int j = j0 + u * BS;
            if (j < NC) reinterpret_cast<float4*>(cell)[j] = v[u];
        }
    }
    return true;
}

// G2P gather from the shared velocity tile (gridToParticle.cs.wgsl:28-130).
// Cells the reference skips hold velocity 0 here: each of their terms is a
// product with a zero factor, and adding +-0 to a sum that started at +0
// leaves it unchanged, so the sums are equal.  The summation order is the
// reference's loop order (z outermost, x innermost).
template <int E, bool PB>
__device__ __forceinline__ void g2p_gather(const TileCtx<E>& T, const float4* vel, const Stencil& sc, float* nv,
                                           float* G) {
    constexpr int H = E + 2;
#pragma unroll
    for (int k = 0; k < 3; k++) nv[k] = 0.f;
#pragma unroll
    for (int i = 0; i < 9; i++) G[i] = 0.f;
    int l0[3];
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        l0[k] = sc.cell[k] - T.origin[k];
        inside = inside && l0[k] >= 0 && l0[k] < E;
    }
    if (!inside) return;
    float offs[3][3];  // offs[axis][o] = (cell + o - 1) - particle_cell_pos
    float dwv[3][3];
    if (PB) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float pcp = fs(fa(i2f(sc.cell[k]), sc.f[k]), 0.5f);
#pragma unroll
            for (int o = 0; o < 3; o++) offs[k][o] = fs(i2f(sc.cell[k] + o - 1), pcp);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int a = 0; a < 3; a++) dwv[k][a] = dwk(k, sc.f[a]);
    }
    const float4* row = vel + (l0[2] * H + l0[1]) * H + l0[0];
    if (PB) {
        // the same sums in paired form: (nv0, nv1), (G[3c], G[3c+1]) per
        // column c, (G[2], G[5]); nv2 and G[8] scalar
        float2 nv01 = make_float2(0.f, 0.f), g01[3], g25 = make_float2(0.f, 0.f);
        float nv2 = 0.f, g8 = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) g01[c] = make_float2(0.f, 0.f);
#pragma unroll
        for (int oz = 0; oz < 3; oz++)
#pragma unroll
            for (int oy = 0; oy < 3; oy++) {
                float wxy[3];
#pragma unroll
                for (int ox = 0; ox < 3; ox++) wxy[ox] = fm(sc.w[ox][0], sc.w[oy][1]);
#pragma unroll
                for (int ox = 0; ox < 3; ox++) {
                    float4 c4 = row[(oz * H + oy) * H + ox];
                    const float wgt = fm(wxy[ox], sc.w[oz][2]);
                    const float2 w2 = dup2(wgt), cv01 = make_float2(c4.x, c4.y);
                    nv01 = ff2(w2, cv01, nv01);
                    nv2 = ff(wgt, c4.z, nv2);
                    const float2 wv01 = fm2(w2, cv01);
                    const float wv2 = fm(wgt, c4.z);
                    const float dist[3] = {offs[0][ox], offs[1][oy], offs[2][oz]};
#pragma unroll
                    for (int c = 0; c < 3; c++) g01[c] = ff2(wv01, dup2(dist[c]), g01[c]);
                    g25 = ff2(dup2(wv2), make_float2(dist[0], dist[1]), g25);
                    g8 = ff(wv2, dist[2], g8);
                }
            }
        nv[0] = nv01.x; nv[1] = nv01.y; nv[2] = nv2;
#pragma unroll
        for (int c = 0; c < 3; c++) { G[3 * c] = g01[c].x; G[3 * c + 1] = g01[c].y; }
        G[2] = g25.x; G[5] = g25.y; G[8] = g8;
        return;
    }
#pragma unroll
    for (int oz = 0; oz < 3; oz++)
#pragma unroll
        for (int oy = 0; oy < 3; oy++) {
            float wxy[3];
#pragma unroll
            for (int ox = 0; ox < 3; ox++) wxy[ox] = fm(sc.w[ox][0], sc.w[oy][1]);
#pragma unroll
            for (int ox = 0; ox < 3; ox++) {
                float4 c4 = row[(oz * H + oy) * H + ox];
                float cv[3] = {c4.x, c4.y, c4.z};
                float wgt = fm(wxy[ox], sc.w[oz][2]);
#pragma unroll
                for (int k = 0; k < 3; k++) nv[k] = ff(wgt, cv[k], nv[k]);
                if (!PB) {
                    float g[3];
                    g[0] = fm(fm(dwv[ox][0], sc.w[oy][1]), sc.w[oz][2]);
                    g[1] = fm(fm(sc.w[ox][0], dwv[oy][1]), sc.w[oz][2]);
                    g[2] = fm(wxy[ox], dwv[oz][2]);
#pragma unroll
                    for (int col = 0; col < 3; col++)
#pragma unroll
                        for (int r = 0; r < 3; r++) G[col * 3 + r] = ff(g[col], cv[r], G[col * 3 + r]);
                } else {
                    float wv[3] = {fm(wgt, cv[0]), fm(wgt, cv[1]), fm(wgt, cv[2])};
                    float dist[3] = {offs[0][ox], offs[1][oy], offs[2][oz]};
#pragma unroll
                    for (int col = 0; col < 3; col++)
#pragma unroll
                        for (int r = 0; r < 3; r++) G[col * 3 + r] = ff(wv[r], dist[col], G[col * 3 + r]);
                }
            }
        }
}

template <bool PB>
__device__ __forceinline__ void g2p_finish(const SceneDev& S, const float* nv, const float* G, float* vel, float* dxp,
                                           float* D) {
#pragma unroll
    for (int k = 0; k < 3; k++) { vel[k] = nv[k]; dxp[k] = fm(nv[k], S.dt); }
    if (!PB) {
#pragma unroll
        for (int i = 0; i < 9; i++) D[i] = fm(G[i], S.dt);
    } else {
#pragma unroll
        for (int i = 0; i < 9; i++) D[i] = fm(fm(G[i], S.dt), 4.0f);
    }
}

// Interaction force at grid cell cc (pbmpm.wgsl:104-134), added to f.
__device__ __noinline__ void interaction_force(const SceneDev& S, const int* cc, float* f) {
    float dv[3] = {fs(i2f(cc[0]), S.ipos[0]), fs(i2f(cc[1]), S.ipos[1]), fs(i2f(cc[2]), S.ipos[2])};
    float dist = len3(dv);
    if (!(dist < S.irad)) return;
    float pd[3] = {0.f, 0.f, 1.f};
    float l = len3(dv);
    if (l > 0.001f) {
#pragma unroll
        for (int k = 0; k < 3; k++) pd[k] = fd(dv[k], l);
    }
    float fl = fd(dist, S.irad);
    float falloff = fs(1.0f, fm(fl, fl));
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float af = (S.imode == 0u) ? fm(fm(pd[k], S.istr), falloff)
                                   : fm(fm(fm(-pd[k], S.istr), falloff), fs(1.0f, falloff));
        f[k] = fa(f[k], af);
    }
}

// i32((x * RN(1/dt)) * scale) and i32((x * dt) * scale), folded into one
// product when the scale is a power of two (SceneDev::fold)
template <bool FOLD>
__device__ __forceinline__ int32_t enc_rdt(const SceneDev& S, float x) {
    return FOLD ? f2i(fm(x, S.rdts)) : f2i(fm(fm(x, S.rdt), S.scale));
}
template <bool FOLD>
__device__ __forceinline__ int32_t enc_dt(const SceneDev& S, float x) {
    return FOLD ? f2i(fm(x, S.dts)) : f2i(fm(fm(x, S.dt), S.scale));
}

// affine P2G + particle-side forces (pbmpm.wgsl:41-147) into the shared tile.
// WITH_MASS = false skips the mass adds: within one substep positions and
// masses do not change between PBMPM iterations, so every iteration's mass
// sums equal the first iteration's (the caller carries them over).  The
// i32 adds commute, so the cells are visited in any order: (x, y) pairs
// outside, z inside, sharing the partial affine sums of each pair.
template <int E, bool WITH_MASS, bool FOLD>
__device__ __forceinline__ void p2g_pbmpm_particle(const SceneDev& S, const TileCtx<E>& T, const Stencil& sc,
                                                   float mass, const float* dxp, const float* D, uint32_t* acc) {
    constexpr int H = E + 2, NC = H * H * H;
    int l0[3];
    bool inside = true;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        l0[k] = sc.cell[k] - T.origin[k];
        inside = inside && l0[k] >= 0 && l0[k] < E;
    }
    if (!inside) return;
    float off[3][3];  // off[axis][o] = (cell + o - 1) - particle_cell_pos
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float pcp = fs(fa(i2f(sc.cell[a]), sc.f[a]), 0.5f);
#pragma unroll
        for (int o = 0; o < 3; o++) off[a][o] = fs(i2f(sc.cell[a] + o - 1), pcp);
    }
    const bool iact = S.iact != 0u;
    // a force component that is zero for every cell adds i32(0) = 0
    bool fon[3];
#pragma unroll
    for (int k = 0; k < 3; k++) fon[k] = iact || S.gdiv[k] != 0.0f;
    uint32_t* base = acc + (l0[2] * H + l0[1]) * H + l0[0];
    if (FOLD && !iact) {
        // components 0 and 1 in paired form, component 2 scalar; same
        // per-component operations as the general loop below
        const float2 D01 = make_float2(D[0], D[1]), D34 = make_float2(D[3], D[4]), D67 = make_float2(D[6], D[7]);
        const float2 dxp01 = make_float2(dxp[0], dxp[1]), rdts2 = dup2(S.rdts);
#pragma unroll
        for (int oy = 0; oy < 3; oy++)
#pragma unroll
            for (int ox = 0; ox < 3; ox++) {
                const float2 pxy01 = ff2(D34, dup2(off[1][oy]), fm2(D01, dup2(off[0][ox])));
                const float pxy2 = ff(D[5], off[1][oy], fm(D[2], off[0][ox]));
                const float wxy = fm(sc.w[ox][0], sc.w[oy][1]);
#pragma unroll
                for (int oz = 0; oz < 3; oz++) {
                    const float wgt = fm(wxy, sc.w[oz][2]);
                    const float wm = fm(wgt, mass);
                    const float2 aff01 = ff2(D67, dup2(off[2][oz]), pxy01);
                    const float aff2 = ff(D[8], off[2][oz], pxy2);
                    const float2 x01 = fm2(fm2(dup2(wm), fa2(dxp01, aff01)), rdts2);
                    uint32_t v[3] = {(uint32_t)f2i(x01.x), (uint32_t)f2i(x01.y),
                                     (uint32_t)f2i(fm(fm(wm, fa(dxp[2], aff2)), S.rdts))};
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (fon[k]) v[k] += (uint32_t)enc_dt<FOLD>(S, fm(S.gdiv[k], wm));
                    uint32_t* cell = base + (oz * H + oy) * H + ox;
#pragma unroll
                    for (int k = 0; k < 3; k++) atomicAdd(cell + (k + (WITH_MASS ? 1 : 0)) * NC, v[k]);
                    if (WITH_MASS) atomicAdd(cell, (uint32_t)f2i(fm(wm, S.scale)));
                }
            }
        return;
    }
#pragma unroll
    for (int oy = 0; oy < 3; oy++)
#pragma unroll(FOLD ? 3 : 1)
        for (int ox = 0; ox < 3; ox++) {
            // aff[r] = fma(D[2][r], off_z, fma(D[1][r], off_y, D[0][r] * off_x))
            float pxy[3];
#pragma unroll
            for (int r = 0; r < 3; r++) pxy[r] = ff(D[3 + r], off[1][oy], fm(D[r], off[0][ox]));
            float wxy = fm(sc.w[ox][0], sc.w[oy][1]);
#pragma unroll
            for (int oz = 0; oz < 3; oz++) {
                float wgt = fm(wxy, sc.w[oz][2]);
                float wm = fm(wgt, mass);
                float fo[3] = {S.gdiv[0], S.gdiv[1], S.gdiv[2]};
                if (iact) {
                    int cc[3] = {sc.cell[0] + ox - 1, sc.cell[1] + oy - 1, sc.cell[2] + oz - 1};
                    float f3[3] = {S.g[0], S.g[1], S.g[2]};
                    interaction_force(S, cc, f3);
#pragma unroll
                    for (int k = 0; k < 3; k++) fo[k] = fm(f3[k], S.rfdiv);
                }
                uint32_t* cell = base + (oz * H + oy) * H + ox;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    float aff = ff(D[6 + k], off[2][oz], pxy[k]);
                    uint32_t v = (uint32_t)enc_rdt<FOLD>(S, fm(wm, fa(dxp[k], aff)));
                    if (fon[k]) v += (uint32_t)enc_dt<FOLD>(S, fm(fo[k], wm));
                    atomicAdd(cell + (k + (WITH_MASS ? 1 : 0)) * NC, v);
                }
                if (WITH_MASS) atomicAdd(cell, (uint32_t)f2i(fm(wm, S.scale)));
            }
        }
}

template <int E, bool WITH_MASS>
__device__ __forceinline__ void p2g_pbmpm(const SceneDev& S, const TileCtx<E>& T, const Stencil& sc, float mass,
                                          const float* dxp, const float* D, uint32_t* acc) {
    if (S.fold) p2g_pbmpm_particle<E, WITH_MASS, true>(S, T, sc, mass, dxp, D, acc);
    else p2g_pbmpm_particle<E, WITH_MASS, false>(S, T, sc, mass, dxp, D, acc);
}

template <int E>
__device__ __forceinline__ void flush_tile(uint32_t* acc, int4* dst) {
    constexpr int H = E + 2, NC = H * H * H;
    for (int j = threadIdx.x; j < NC; j += blockDim.x)
        dst[j] = make_int4((int)acc[j], (int)acc[NC + j], (int)acc[2 * NC + j], (int)acc[3 * NC + j]);
}

// momentum-only accumulator of the PBMPM iterations: 3 planes x (E+2)^3
template <int E>
__device__ __forceinline__ void zero_mom(uint32_t* acc) {
    constexpr int H = E + 2, NC = H * H * H;
    uint4* a4 = reinterpret_cast<uint4*>(acc);
    for (int j = threadIdx.x; j < 3 * NC / 4; j += blockDim.x) a4[j] = make_uint4(0u, 0u, 0u, 0u);
}

// halo record of a PBMPM iteration: the cell's reciprocal mass RN(1/m) of the
// substep (the same in every tile that covers the cell) in the mass word,
// this tile's momentum sums in the other three
template <int E>
__device__ __forceinline__ void flush_mom(const uint32_t* acc, const float* rm_s, int4* dst) {
    constexpr int H = E + 2, NC = H * H * H;
#pragma unroll 4
    for (int j = threadIdx.x; j < NC; j += blockDim.x)
        dst[j] = make_int4(__float_as_int(rm_s[j]), (int)acc[j], (int)acc[NC + j], (int)acc[2 * NC + j]);
}

template <int E>
__device__ __forceinline__ void zero_acc(uint32_t* acc) {
    constexpr int H = E + 2, NC = H * H * H;
    uint4* a4 = reinterpret_cast<uint4*>(acc);
    for (int j = threadIdx.x; j < NC; j += blockDim.x) a4[j] = make_uint4(0u, 0u, 0u, 0u);
}

// A halo copy wait ran out: report it, give the copy in flight a second
// bounded wait (so no bulk write lands after the CTA has exited), and let the
// caller return.
__device__ __noinline__ void copy_wait_failed(const Ctx& c, HaloCopy& hc) {
    if (threadIdx.x == 0) {
        atomicOr(&c.counters->status, ST_COPY_TIMEOUT);
        mbar_wait_parity(hc.mbar, hc.parity ^ 1u, COPY_WAIT_LIMIT);
    }
    __syncthreads();
}

__device__ __forceinline__ uint32_t n_tiles_now(const Ctx& c) {
    uint32_t n = c.counters->n_st;
    return n < c.max_tiles ? n : c.max_tiles;
}

// Tile scheduling of the persistent tile kernels: CTA b takes claim slot b
// first, then the next unclaimed slot (gridDim.x + ticket) each time it
// finishes a tile, so CTAs with light tiles take more of them and a launch
// ends within about one tile of the average.  Slot k maps to a tile through
// tile_order (Morton order, so the tiles in flight at one time are neighbours
// and share their halo data in L2; read from its end on alternate launches,
// so a launch starts on the tiles the previous one wrote last).  Each tile's
// results go to its own slots, so which CTA runs a tile, and when, changes
// nothing in them.  Returns n (stop) past the last slot.
__device__ __forceinline__ uint32_t tile_at(const Ctx& c, uint32_t k, uint32_t n) {
    if (k >= n) return n;
    if (!c.tile_order) return k;
    const uint32_t st = __ldg(c.tile_order + (c.order_rev ? n - 1u - k : k));
    return st < n ? st : n;
}

// Called by thread 0; the caller broadcasts the result through shared memory.
__device__ __forceinline__ uint32_t claim_tile(const Ctx& c, uint32_t n) {
    return tile_at(c, gridDim.x + atomicAdd(&c.counters->tile_ticket, 1u), n);
}

// Claim order of the tiles: a counting sort in one CTA by a 12- or 15-bit
// Morton bucket of the tile coordinates (4 or 5 low bits per axis, offset per
// scene), so the tiles of a 16^3- or 32^3-tile neighbourhood are ordered along
// the Morton curve (tiles in one bucket keep an arbitrary order).  The scatter
// positions are the buckets' prefix offsets, so the result is always a
// permutation.
constexpr uint32_t TILE_ORDER_BUCKETS = 1u << 15;   // the wider bucket count
constexpr size_t TILE_ORDER_SMEM = TILE_ORDER_BUCKETS * 4;
constexpr uint32_t TILE_ORDER_MIN = 256;    // at most this many tiles keep the compact order

__device__ __forceinline__ uint32_t spread3_5(uint32_t v) {
    uint32_t x = v & 31u;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// bucket of a tile key: the Morton code of the low `bits` bits of each
// coordinate (bits = 4 or 5), offset per scene, modulo nb = 2^(3 bits)
__device__ __forceinline__ uint32_t tile_bucket(uint64_t key, uint32_t axis_mask, uint32_t nb) {
    const uint32_t m = spread3_5((uint32_t)(key >> 32) & axis_mask) |
                       (spread3_5((uint32_t)(key >> 16) & axis_mask) << 1) |
                       (spread3_5((uint32_t)key & axis_mask) << 2);
    return (m + (uint32_t)(key >> 48) * 0x9E3779B1u) & (nb - 1u);
}

template <uint32_t BITS>
__device__ __forceinline__ void tile_order_sort(const Ctx& c, uint32_t n, uint32_t* hist, uint32_t* warp_sum) {
    constexpr uint32_t NB = 1u << (3 * BITS), PER = NB / 1024u;   // buckets, buckets per thread
    constexpr uint32_t AXIS = (1u << BITS) - 1u;
    for (uint32_t b = threadIdx.x; b < NB; b += 1024) hist[b] = 0u;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += 1024) atomicAdd(&hist[tile_bucket(c.st_key[i], AXIS, NB)], 1u);
    __syncthreads();
    // exclusive prefix sums: each thread scans its PER consecutive buckets,
    // the thread totals are scanned across the block
    const uint32_t b0 = threadIdx.x * PER;
    uint32_t tot = 0;
#pragma unroll
    for (uint32_t k = 0; k < PER; k++) tot += hist[b0 + k];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = tot;
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc += v;
    }
    if (lane == 31u) warp_sum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane], wi = w;
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += v;
        }
        warp_sum[lane] = wi - w;   // exclusive over warps
    }
    __syncthreads();
    uint32_t run = warp_sum[warp] + inc - tot;
#pragma unroll
    for (uint32_t k = 0; k < PER; k++) {
        const uint32_t h = hist[b0 + k];
        hist[b0 + k] = run;
        run += h;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += 1024) {
        const uint32_t pos = atomicAdd(&hist[tile_bucket(c.st_key[i], AXIS, NB)], 1u);
        if (pos < n) c.tile_order[pos] = i;
    }
}

__global__ void __launch_bounds__(1024) k_tile_order(Ctx c) {
    extern __shared__ uint4 smem_raw[];
    uint32_t* hist = reinterpret_cast<uint32_t*>(smem_raw);
    __shared__ uint32_t warp_sum[32];
    const uint32_t n = n_tiles_now(c);
    uint32_t mode = c.order_mode;
    // automatic: few tiles nearly all run at once, so their order gains
    // nothing; up to 4,096 tiles 4 bits per axis (4,096 buckets), else 5 (32,768)
    if (mode != 1u && mode != 4u && mode != 5u) mode = n <= TILE_ORDER_MIN ? 1u : (n <= 4096u ? 4u : 5u);
    if (mode == 1u) {
        for (uint32_t i = threadIdx.x; i < n; i += 1024) c.tile_order[i] = i;
        return;
    }
    if (mode == 4u) tile_order_sort<4>(c, n, hist, warp_sum);
    else tile_order_sort<5>(c, n, hist, warp_sum);
}

// A CTA leaves a tile kernel: the last one to leave zeroes the ticket for the
// next launch (every CTA has claimed its last ticket before it counts itself).
__device__ __forceinline__ void tiles_done(const Ctx& c) {
    if (threadIdx.x == 0) {
        if (atomicAdd(&c.counters->tile_done, 1u) == gridDim.x - 1u) {
            c.counters->tile_ticket = 0u;
            c.counters->tile_done = 0u;
        }
    }
}

// Neighbour table of the compact tiles, once per substep: entry st*27 + d is
// the compact index of the tile at offset d = 9(dz+1) + 3(dy+1) + (dx+1), or
// -1 when that tile is unoccupied or past the tile storage.
template <int E>
__global__ void __launch_bounds__(256) k_tile_nbr(Ctx c) {
    uint32_t n = n_tiles_now(c) * 27u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t st = i / 27u, d = i - st * 27u;
        int r = (int)st;
        if (d != 13u) {
            uint32_t scene;
            int sx, sy, sz;
            unpack_key(c.st_key[st], scene, sx, sy, sz);
            sx += (int)(d % 3u) - 1;
            sy += (int)((d / 3u) % 3u) - 1;
            sz += (int)(d / 9u) - 1;
            uint32_t slot = tile_lookup(c, pack_key(scene, sx, sy, sz), scene, sx, sy, sz);
            r = (slot == INVALID) ? -1 : (int)c.slot_st[slot];
            if (r >= (int)c.max_tiles) r = -1;
        }
        c.st_nbr[i] = r;
    }
}

// ------------------------------------------------------------------
// explicit P2G (particleToGrid.cs.wgsl:27-79)
// ------------------------------------------------------------------
template <int E, int BS>
__global__ void __launch_bounds__(BS) k_p2g_explicit(Ctx c) {
    constexpr int H = E + 2, NC = H * H * H;
    extern __shared__ uint4 smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    __shared__ SceneDev S;
    __shared__ uint32_t s_next;
    uint32_t cur_scene = INVALID;
    uint32_t n_st = n_tiles_now(c);
    for (uint32_t st = tile_at(c, blockIdx.x, n_st); st < n_st; st = s_next) {
        TileCtx<E> T;
        tile_begin<E>(c, st, S, T, cur_scene);
        zero_acc<E>(acc);
        __syncthreads();
        uint32_t begin = c.st_begin[st], cnt = c.st_count[st];
        for (uint32_t i = threadIdx.x; i < cnt; i += BS) {
            uint32_t pid = c.sorted[begin + i];
            PState p;
            load_particle<true>(c.work_in, c.n_particles, pid, p, false);
            Stencil sc;
            make_stencil(S, p.pos, sc);
            int l0[3];
            bool inside = true;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                l0[k] = sc.cell[k] - T.origin[k];
                inside = inside && l0[k] >= 0 && l0[k] < E;
            }
            if (!inside) continue;
            float M[9];
            stress_matrix(S, p, M);
            float pm[3] = {fm(p.mass, p.vel[0]), fm(p.mass, p.vel[1]), fm(p.mass, p.vel[2])};
            float dw[3][3];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int a = 0; a < 3; a++) dw[k][a] = dwk(k, sc.f[a]);
            uint32_t* base = acc + (l0[2] * H + l0[1]) * H + l0[0];
#pragma unroll 1
            for (int oz = 0; oz < 3; oz++) {
                const float wz = oz == 0 ? sc.w[0][2] : (oz == 1 ? sc.w[1][2] : sc.w[2][2]);
                const float dwz = oz == 0 ? dw[0][2] : (oz == 1 ? dw[1][2] : dw[2][2]);
#pragma unroll
                for (int oy = 0; oy < 3; oy++)
#pragma unroll
                    for (int ox = 0; ox < 3; ox++) {
                        float wxy = fm(sc.w[ox][0], sc.w[oy][1]);
                        float wgt = fm(wxy, wz);
                        float g[3];
                        g[0] = fm(fm(fm(dw[ox][0], sc.w[oy][1]), wz), S.rcd[0]);
                        g[1] = fm(fm(fm(sc.w[ox][0], dw[oy][1]), wz), S.rcd[1]);
                        g[2] = fm(fm(wxy, dwz), S.rcd[2]);
                        float sf[3];
                        mv3(M, g, sf);
                        uint32_t* cell = base + (oz * H + oy) * H + ox;
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            float mom = ff(wgt, pm[k], fm(sf[k], S.dt));
                            atomicAdd(cell + (k + 1) * NC, (uint32_t)f2i(fm(mom, S.scale)));
                        }
                        atomicAdd(cell, (uint32_t)f2i(fm(fm(wgt, p.mass), S.scale)));
                    }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_next = claim_tile(c, n_st);
        flush_tile<E>(acc, c.tiles_a + (size_t)st * NC);
        __syncthreads();
    }
    tiles_done(c);
}

// ------------------------------------------------------------------
// G2P + integrate (explicit: gridToParticle.cs.wgsl:28-80; PBMPM :82-130;
// integrateParticles.wgsl:14-72)
// ------------------------------------------------------------------
template <int E, bool PB, int BS, int RM = 0>
__global__ void __launch_bounds__(BS) k_g2p_integrate(Ctx c) {
    extern __shared__ uint4 smem_raw[];
    int4* cell = reinterpret_cast<int4*>(smem_raw);
    const float4* vel = reinterpret_cast<const float4*>(smem_raw);
    __shared__ SceneDev S;
    __shared__ int nbr[27];
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) mbar_init1(&mbar);
    __syncthreads();
    HaloCopy hc{&mbar, 0u};
    __shared__ uint32_t s_next;
    uint32_t cur_scene = INVALID;
    uint32_t n_st = n_tiles_now(c);
    for (uint32_t st = tile_at(c, blockIdx.x, n_st); st < n_st; st = s_next) {
        TileCtx<E> T;
        tile_begin<E>(c, st, S, T, cur_scene);
        load_neighbors(c, st, nbr);
        __syncthreads();
        if (!assemble_velocity_tile<E, BS, PB, RM>(c.tiles_b, S, T, nbr, cell, hc)) {
            copy_wait_failed(c, hc);
            tiles_done(c);
            return;
        }
        __syncthreads();
        uint32_t begin = c.st_begin[st], cnt = c.st_count[st];
        for (uint32_t i = threadIdx.x; i < cnt; i += BS) {
            const uint32_t slot = begin + i;
            const uint32_t pid = c.sorted[slot];
            PState p;
            load_particle<true>(c.work_in, c.n_particles, pid, p, false);
            Stencil sc;
            make_stencil(S, p.pos, sc);
            float nv[3], G[9];
            g2p_gather<E, PB>(T, vel, sc, nv, G);
            g2p_finish<PB>(S, nv, G, p.vel, p.dxp, p.D);
            integrate(c, S, p, slot);
            store_particle(c.work_out, c.n_particles, slot, p);
            c.ids_out[slot] = __ldg(c.ids_in + pid);
        }
        if (threadIdx.x == 0) s_next = claim_tile(c, n_st);
        __syncthreads();
    }
    tiles_done(c);
}

// ------------------------------------------------------------------
// PBMPM first iteration: constraints + affine P2G + forces
// (pbmpm.wgsl:154-178); writes the iteration records
// ------------------------------------------------------------------
__device__ __forceinline__ void store_iter_rec(const Ctx& c, uint32_t t, const float* pos, float mass, const float* Fe,
                                               const float* Fei, float relax) {
    float4* r = c.iter_rec + t;
    const size_t n = c.n_particles;
    r[0] = make_float4(pos[0], pos[1], pos[2], mass);
    r[n] = make_float4(Fe[0], Fe[1], Fe[2], Fe[3]);
    r[2 * n] = make_float4(Fe[4], Fe[5], Fe[6], Fe[7]);
    r[3 * n] = make_float4(Fe[8], Fei[0], Fei[1], Fei[2]);
    r[4 * n] = make_float4(Fei[3], Fei[4], Fei[5], Fei[6]);
    r[5 * n] = make_float4(Fei[7], Fei[8], relax, 0.f);
}

__device__ __forceinline__ void load_iter_rec(const Ctx& c, uint32_t t, float* pos, float& mass, float* Fe,
                                              float* Fei, float& relax) {
    const float4* r = c.iter_rec + t;
    const size_t n = c.n_particles;
    float4 q0 = __ldg(r), q1 = __ldg(r + n), q2 = __ldg(r + 2 * n), q3 = __ldg(r + 3 * n), q4 = __ldg(r + 4 * n),
           q5 = __ldg(r + 5 * n);
    pos[0] = q0.x; pos[1] = q0.y; pos[2] = q0.z; mass = q0.w;
    Fe[0] = q1.x; Fe[1] = q1.y; Fe[2] = q1.z; Fe[3] = q1.w;
    Fe[4] = q2.x; Fe[5] = q2.y; Fe[6] = q2.z; Fe[7] = q2.w;
    Fe[8] = q3.x; Fei[0] = q3.y; Fei[1] = q3.z; Fei[2] = q3.w;
    Fei[3] = q4.x; Fei[4] = q4.y; Fei[5] = q4.z; Fei[6] = q4.w;
    Fei[7] = q5.x; Fei[8] = q5.y; relax = q5.z;
}

template <int E, int BS>
__global__ void __launch_bounds__(BS) k_pbmpm_first(Ctx c) {
    constexpr int H = E + 2, NC = H * H * H;
    extern __shared__ uint4 smem_raw[];
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw);
    __shared__ SceneDev S;
    __shared__ uint32_t s_next;
    uint32_t cur_scene = INVALID;
    uint32_t n_st = n_tiles_now(c);
    for (uint32_t st = tile_at(c, blockIdx.x, n_st); st < n_st; st = s_next) {
        TileCtx<E> T;
        tile_begin<E>(c, st, S, T, cur_scene);
        zero_acc<E>(acc);
        __syncthreads();
        uint32_t begin = c.st_begin[st], cnt = c.st_count[st];
        for (uint32_t i = threadIdx.x; i < cnt; i += BS) {
            uint32_t pid = c.sorted[begin + i];
            PState p;
            load_particle<true>(c.work_in, c.n_particles, pid, p, true);
            float Fei[9];
            inv3(p.Fe, Fei);
            float relax = pbmpm_relax(S, p.Fp);
            store_iter_rec(c, begin + i, p.pos, p.mass, p.Fe, Fei, relax);
            pbmpm_constraints(S, p.Fe, Fei, relax, p.D);
            Stencil sc;
            make_stencil(S, p.pos, sc);
            p2g_pbmpm<E, true>(S, T, sc, p.mass, p.dxp, p.D, acc);
        }
        __syncthreads();
        if (threadIdx.x == 0) s_next = claim_tile(c, n_st);
        flush_tile<E>(acc, c.tiles_a + (size_t)st * NC);
        __syncthreads();
    }
    tiles_done(c);
}

// PBMPM iteration i>0: G2P of iteration i-1, constraints, P2G of iteration i,
// all from the iteration records (contiguous in tile order).  Positions and
// masses are fixed within a substep, so the cell masses are the first
// transfer's: the first iteration (FIRST) forms their reciprocals from the
// mass sums; every iteration accumulates momentum only and writes, per halo
// cell, the reciprocal mass and its momentum sums, so the next pass reads the
// reciprocal masses with its own halo record.  Shared memory: the halo sums /
// velocities (16 B per cell), three momentum planes (12 B per cell) and the
// reciprocal masses (4 B per cell).
template <int E, int BS, bool FIRST>
__global__ void __launch_bounds__(BS) k_pbmpm_iter(Ctx c) {
    constexpr int H = E + 2, NC = H * H * H;
    extern __shared__ uint4 smem_raw[];
    int4* cell = reinterpret_cast<int4*>(smem_raw);
    const float4* vel = reinterpret_cast<const float4*>(smem_raw);
    uint32_t* acc = reinterpret_cast<uint32_t*>(smem_raw + NC);
    float* rm_s = reinterpret_cast<float*>(acc + 3 * NC);   // reciprocal cell masses, for the flush
    __shared__ SceneDev S;
    __shared__ int nbr[27];
    __shared__ uint64_t mbar;
    __shared__ uint32_t s_next;
    if (threadIdx.x == 0) mbar_init1(&mbar);
    __syncthreads();
    HaloCopy hc{&mbar, 0u};
    uint32_t cur_scene = INVALID;
    uint32_t n_st = n_tiles_now(c);
    // a tile's own-halo copies are issued as soon as the previous tile's
    // particles are done, so they overlap that tile's flush
    const uint32_t st0 = tile_at(c, blockIdx.x, n_st);
    if (st0 < n_st)
        halo_issue<E>(c.tiles_b, st0, cell, hc);
    for (uint32_t st = st0; st < n_st; st = s_next) {
        TileCtx<E> T;
        tile_begin<E>(c, st, S, T, cur_scene);
        load_neighbors(c, st, nbr);
        zero_mom<E>(acc);
        __syncthreads();
        if (!assemble_velocity_tile<E, BS, true, FIRST ? 1 : 2, true>(c.tiles_b, S, T, nbr, cell, hc,
                                                                     rm_s)) {
            copy_wait_failed(c, hc);
            tiles_done(c);
            return;
        }
        __syncthreads();
        uint32_t begin = c.st_begin[st], cnt = c.st_count[st];
        for (uint32_t i = threadIdx.x; i < cnt; i += BS) {
            float pos[3], mass, Fe[9], Fei[9], relax;
            load_iter_rec(c, begin + i, pos, mass, Fe, Fei, relax);
            Stencil sc;
            make_stencil(S, pos, sc);
            float nv[3], G[9], v[3], dxp[3], D[9];
            g2p_gather<E, true>(T, vel, sc, nv, G);
            g2p_finish<true>(S, nv, G, v, dxp, D);
            pbmpm_constraints(S, Fe, Fei, relax, D);
            p2g_pbmpm<E, false>(S, T, sc, mass, dxp, D, acc);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t nx = claim_tile(c, n_st);
            s_next = nx;
            if (nx < n_st)
                halo_issue<E>(c.tiles_b, nx, cell, hc);
        }
        flush_mom<E>(acc, rm_s, c.tiles_a + (size_t)st * NC);
        __syncthreads();
    }
    tiles_done(c);
}

// ------------------------------------------------------------------
// dense grid readback for one scene (inspection only)
// ------------------------------------------------------------------
template <int E>
__global__ void __launch_bounds__(256) k_grid_dense(Ctx c, uint32_t scene, int apply_update, int4* out) {
    constexpr int H = E + 2, NC = H * H * H;
    __shared__ SceneDev S;
    __shared__ int nbr[27];
    uint32_t cur_scene = INVALID;
    uint32_t n_st = n_tiles_now(c);
    for (uint32_t st = blockIdx.x; st < n_st; st += gridDim.x) {
        TileCtx<E> T;
        tile_begin<E>(c, st, S, T, cur_scene);
        __syncthreads();
        if (T.scene != scene) continue;
        load_neighbors(c, st, nbr);
        __syncthreads();
        for (int j = threadIdx.x; j < NC; j += blockDim.x) {
            int4 s = assemble_cell<E>(c.tiles_b, nbr, j);
            if (c.tiles_m) s.x = assemble_cell<E>(c.tiles_m, nbr, j).x;
            int lx = j % H, ly = (j / H) % H, lz = j / (H * H);
            int gc[3] = {T.origin[0] - 1 + lx, T.origin[1] - 1 + ly, T.origin[2] - 1 + lz};
            if (gc[0] < 0 || gc[1] < 0 || gc[2] < 0 || gc[0] >= S.res[0] || gc[1] >= S.res[1] || gc[2] >= S.res[2]) continue;
            if (apply_update) {
                float cm = inv_s(S, s.x);
                if (cm > 0.0f) {
                    float rm = __frcp_rn(cm);
                    int32_t mi[3] = {s.y, s.z, s.w};
                    float u[3];
#pragma unroll
                    for (int k = 0; k < 3; k++) u[k] = fa(fm(inv_s(S, mi[k]), rm), S.gdt[k]);
                    grid_bc(S, gc, u);
                    s.y = f2i(fm(fm(u[0], cm), S.scale));
                    s.z = f2i(fm(fm(u[1], cm), S.scale));
                    s.w = f2i(fm(fm(u[2], cm), S.scale));
                }
            }
            size_t o = ((size_t)gc[2] * S.res[1] + gc[1]) * S.res[0] + gc[0];
            out[o] = s;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------
// device self-test of the arithmetic helpers
// ------------------------------------------------------------------
__device__ __forceinline__ uint32_t mix32(uint64_t v) {
    v ^= v >> 33; v *= 0xff51afd7ed558ccdull; v ^= v >> 33; v *= 0xc4ceb9fe1a85ec53ull; v ^= v >> 33;
    return (uint32_t)v;
}

// Checks, on n pseudo-random operand pairs, the two identities the kernels
// rely on: the folded fixed-point encoding i32(x * (r * 2^k)) equals
// i32((x * r) * 2^k) for 0 <= k <= 60 (x with exponent in [-80, 40], r in
// [2^-30, 2^30]), and the reciprocal __frcp_rn(d) equals the IEEE quotient
// 1 / d; also the f32 -> i32 conversion on NaN, infinities and out-of-range
// values.  counts[0] = identity mismatches, counts[1] = conversion mismatch
// code, counts[2] = the raw hardware conversion of a NaN (informational).
__global__ void k_selftest(uint64_t n, uint64_t seed, unsigned long long* counts) {
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long bad = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t a = mix32(seed ^ (i * 2 + 0)), b = mix32(seed ^ (i * 2 + 1));
        int ex = (int)(a % 121u) - 80, er = (int)((a >> 8) % 61u) - 30, k = (int)((a >> 16) % 61u);
        float x = __uint_as_float((a & 0x80000000u) | ((uint32_t)(ex + 127) << 23) | (b & 0x7fffffu));
        float r = __uint_as_float(((uint32_t)(er + 127) << 23) | ((b >> 9) & 0x7fffffu) | ((a & 1u) << 22));
        if (i & 1) r = -r;
        float p2 = __uint_as_float((uint32_t)(k + 127) << 23);
        float rk = __fmul_rn(r, p2);
        if (f2i(__fmul_rn(__fmul_rn(x, r), p2)) != f2i(__fmul_rn(x, rk))) bad++;
        if (__float_as_uint(__frcp_rn(r)) != __float_as_uint(__fdiv_rn(1.0f, r))) bad++;
    }
    if (bad) atomicAdd(&counts[0], bad);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        volatile float nanv = __int_as_float(0x7fc00000), pinf = __int_as_float(0x7f800000),
                       ninf = __int_as_float(0xff800000), big = 3e9f, nbig = -3e9f, a = 2.9f, b = -2.9f;
        unsigned long long cb = 0;
        if (f2i(nanv) != 0) cb |= 1ull;
        if (f2i(pinf) != 2147483647) cb |= 2ull;
        if (f2i(ninf) != (int)0x80000000) cb |= 4ull;
        if (f2i(big) != 2147483647 || f2i(nbig) != (int)0x80000000) cb |= 8ull;
        if (f2i(b) != -2 || f2i(a) != 2) cb |= 16ull;
        counts[1] = cb;
        counts[2] = (unsigned long long)(uint32_t)__float2int_rz(nanv);
    }
}

// ------------------------------------------------------------------
// launch wrappers
// ------------------------------------------------------------------
constexpr int BS_DEFAULT = 256;

template <int E>
size_t smem_bytes(uint32_t kid) {
    constexpr size_t NC = (size_t)(E + 2) * (E + 2) * (E + 2);
    switch (kid) {
        case K_P2G_EXPLICIT:
        case K_PBMPM_FIRST:
        case K_G2P_EXPLICIT:
        case K_G2P_PBMPM:
        case K_P2G_EXPLICIT_128:
        case K_G2P_EXPLICIT_128:
        case K_PBMPM_FIRST_WIDE:
        case K_G2P_PBMPM_WIDE:
        case K_P2G_EXPLICIT_WIDE:
        case K_G2P_EXPLICIT_WIDE: return 16 * NC;
        case K_PBMPM_ITER:
        case K_PBMPM_ITER_WIDE: return 32 * NC;
        default: return 0;
    }
}

template <int E>
constexpr int iter_block() { return E == 16 ? 512 : 256; }

template <int E>
int block_size(uint32_t kid) {
    if (kid == K_P2G_EXPLICIT_128 || kid == K_G2P_EXPLICIT_128) return 128;
    if (kid == K_PBMPM_ITER_WIDE) return E == 8 ? 512 : iter_block<E>();
    if (kid == K_PBMPM_FIRST_WIDE || kid == K_G2P_PBMPM_WIDE || kid == K_P2G_EXPLICIT_WIDE ||
        kid == K_G2P_EXPLICIT_WIDE)
        return E == 8 ? 512 : BS_DEFAULT;
    return kid == K_PBMPM_ITER ? iter_block<E>() : BS_DEFAULT;
}

// every instantiation behind a kernel id (variants share the id's launch shape)
template <int E>
int kernel_ptrs(uint32_t kid, void** out) {
    switch (kid) {
        case K_BIN_INSERT: out[0] = (void*)k_bin_insert<E>; return 1;
        case K_P2G_EXPLICIT: out[0] = (void*)k_p2g_explicit<E, BS_DEFAULT>; return 1;
        case K_G2P_EXPLICIT: out[0] = (void*)k_g2p_integrate<E, false, BS_DEFAULT, 0>; return 1;
        case K_PBMPM_FIRST: out[0] = (void*)k_pbmpm_first<E, BS_DEFAULT>; return 1;
        case K_PBMPM_ITER:
            out[0] = (void*)k_pbmpm_iter<E, iter_block<E>(), true>;
            out[1] = (void*)k_pbmpm_iter<E, iter_block<E>(), false>;
            return 2;
        case K_PBMPM_ITER_WIDE:
            if constexpr (E == 8) {
                out[0] = (void*)k_pbmpm_iter<E, 512, true>;
                out[1] = (void*)k_pbmpm_iter<E, 512, false>;
                return 2;
            } else {
                return kernel_ptrs<E>(K_PBMPM_ITER, out);
            }
        case K_PBMPM_FIRST_WIDE:
            if constexpr (E == 8) {
                out[0] = (void*)k_pbmpm_first<E, 512>;
                return 1;
            } else {
                return kernel_ptrs<E>(K_PBMPM_FIRST, out);
            }
        case K_G2P_PBMPM_WIDE:
            if constexpr (E == 8) {
                out[0] = (void*)k_g2p_integrate<E, true, 512, 2>;
                out[1] = (void*)k_g2p_integrate<E, true, 512, 0>;
                return 2;
            } else {
                return kernel_ptrs<E>(K_G2P_PBMPM, out);
            }
        case K_P2G_EXPLICIT_WIDE:
            if constexpr (E == 8) {
                out[0] = (void*)k_p2g_explicit<E, 512>;
                return 1;
            } else {
                return kernel_ptrs<E>(K_P2G_EXPLICIT, out);
            }
        case K_G2P_EXPLICIT_WIDE:
            if constexpr (E == 8) {
                out[0] = (void*)k_g2p_integrate<E, false, 512, 0>;
                return 1;
            } else {
                return kernel_ptrs<E>(K_G2P_EXPLICIT, out);
            }
        case K_G2P_PBMPM:
            out[0] = (void*)k_g2p_integrate<E, true, BS_DEFAULT, 2>;
            out[1] = (void*)k_g2p_integrate<E, true, BS_DEFAULT, 0>;
            return 2;
        case K_GRID_DENSE: out[0] = (void*)k_grid_dense<E>; return 1;
        case K_TILE_NBR: out[0] = (void*)k_tile_nbr<E>; return 1;
        case K_P2G_EXPLICIT_128: out[0] = (void*)k_p2g_explicit<E, 128>; return 1;
        case K_G2P_EXPLICIT_128: out[0] = (void*)k_g2p_integrate<E, false, 128, 0>; return 1;
        default: return 0;
    }
}

template <int E>
cudaError_t configure_tile_kernels(int* blocks_per_sm) {
    for (uint32_t kid : {K_P2G_EXPLICIT, K_G2P_EXPLICIT, K_PBMPM_FIRST, K_PBMPM_ITER, K_G2P_PBMPM, K_GRID_DENSE,
                         K_P2G_EXPLICIT_128, K_G2P_EXPLICIT_128, K_PBMPM_ITER_WIDE, K_PBMPM_FIRST_WIDE,
                         K_G2P_PBMPM_WIDE, K_P2G_EXPLICIT_WIDE, K_G2P_EXPLICIT_WIDE}) {
        void* fs[2] = {nullptr, nullptr};
        int nf = kernel_ptrs<E>(kid, fs);
        size_t sm = smem_bytes<E>(kid);
        int nb_min = 1 << 30;
        for (int i = 0; i < nf; i++) {
            cudaError_t e = cudaFuncSetAttribute(fs[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            if (e != cudaSuccess) return e;
            int nb = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fs[i], block_size<E>(kid), sm);
            if (e != cudaSuccess) return e;
            nb_min = nb < nb_min ? nb : nb_min;
        }
        blocks_per_sm[kid] = nb_min > 0 ? nb_min : 1;
    }
    return cudaFuncSetAttribute(k_tile_order, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_ORDER_SMEM);
}

template <int E>
cudaError_t launch_kernel(uint32_t kid, const Ctx& c, cudaStream_t s, int grid_tiles, uint32_t scene, int apply,
                          int4* out) {
    uint32_t n = c.n_particles;
    uint32_t pblocks = (n + 255u) / 256u;
    uint32_t n_chunks = c.cap / COMPACT_CHUNK;
    switch (kid) {
        case K_CLEAR_TABLE: k_clear_table<<<256, 256, 0, s>>>(c); break;
        case K_BIN_INSERT: if (pblocks) k_bin_insert<E><<<pblocks, 256, 0, s>>>(c); break;
        case K_COMPACT_A: k_compact_a<<<n_chunks, 256, 0, s>>>(c); break;
        case K_COMPACT_B: k_compact_b<<<1, 1024, 0, s>>>(c, n_chunks); break;
        case K_COMPACT_C: k_compact_c<<<n_chunks, 256, 0, s>>>(c); break;
        case K_BIN_SCATTER: if (pblocks) k_bin_scatter<<<pblocks, 256, 0, s>>>(c); break;
        case K_TILE_NBR: k_tile_nbr<E><<<grid_tiles, 256, 0, s>>>(c); break;
        case K_P2G_EXPLICIT: k_p2g_explicit<E, BS_DEFAULT><<<grid_tiles, BS_DEFAULT, smem_bytes<E>(kid), s>>>(c); break;
        case K_G2P_EXPLICIT: k_g2p_integrate<E, false, BS_DEFAULT, 0><<<grid_tiles, BS_DEFAULT, smem_bytes<E>(kid), s>>>(c); break;
        case K_PBMPM_FIRST: k_pbmpm_first<E, BS_DEFAULT><<<grid_tiles, BS_DEFAULT, smem_bytes<E>(kid), s>>>(c); break;
        case K_PBMPM_ITER:
            if (c.iter_first) k_pbmpm_iter<E, iter_block<E>(), true><<<grid_tiles, iter_block<E>(), smem_bytes<E>(kid), s>>>(c);
            else k_pbmpm_iter<E, iter_block<E>(), false><<<grid_tiles, iter_block<E>(), smem_bytes<E>(kid), s>>>(c);
            break;
        case K_PBMPM_ITER_WIDE:
            if constexpr (E == 8) {
                if (c.iter_first) k_pbmpm_iter<E, 512, true><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
                else k_pbmpm_iter<E, 512, false><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
            } else {
                return launch_kernel<E>(K_PBMPM_ITER, c, s, grid_tiles, scene, apply, out);
            }
            break;
        case K_PBMPM_FIRST_WIDE:
            if constexpr (E == 8) k_pbmpm_first<E, 512><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
            else return launch_kernel<E>(K_PBMPM_FIRST, c, s, grid_tiles, scene, apply, out);
            break;
        case K_G2P_PBMPM_WIDE:
            if constexpr (E == 8) {
                if (c.g2p_rm) k_g2p_integrate<E, true, 512, 2><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
                else k_g2p_integrate<E, true, 512, 0><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
            } else {
                return launch_kernel<E>(K_G2P_PBMPM, c, s, grid_tiles, scene, apply, out);
            }
            break;
        case K_P2G_EXPLICIT_WIDE:
            if constexpr (E == 8) k_p2g_explicit<E, 512><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
            else return launch_kernel<E>(K_P2G_EXPLICIT, c, s, grid_tiles, scene, apply, out);
            break;
        case K_G2P_EXPLICIT_WIDE:
            if constexpr (E == 8) k_g2p_integrate<E, false, 512, 0><<<grid_tiles, 512, smem_bytes<E>(kid), s>>>(c);
            else return launch_kernel<E>(K_G2P_EXPLICIT, c, s, grid_tiles, scene, apply, out);
            break;
        case K_G2P_PBMPM:
            if (c.g2p_rm) k_g2p_integrate<E, true, BS_DEFAULT, 2><<<grid_tiles, BS_DEFAULT, smem_bytes<E>(kid), s>>>(c);
            else k_g2p_integrate<E, true, BS_DEFAULT, 0><<<grid_tiles, BS_DEFAULT, smem_bytes<E>(kid), s>>>(c);
            break;
        case K_GRID_DENSE: k_grid_dense<E><<<grid_tiles, 256, 0, s>>>(c, scene, apply, out); break;
        case K_TILE_ORDER: if (c.tile_order) k_tile_order<<<1, 1024, TILE_ORDER_SMEM, s>>>(c); break;
        case K_P2G_EXPLICIT_128: k_p2g_explicit<E, 128><<<grid_tiles, 128, smem_bytes<E>(kid), s>>>(c); break;
        case K_G2P_EXPLICIT_128: k_g2p_integrate<E, false, 128, 0><<<grid_tiles, 128, smem_bytes<E>(kid), s>>>(c); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_selftest(uint64_t n, uint64_t seed, unsigned long long* counts, cudaStream_t s) {
    k_selftest<<<1184, 256, 0, s>>>(n, seed, counts);
    return cudaGetLastError();
}

template cudaError_t configure_tile_kernels<8>(int*);
template cudaError_t configure_tile_kernels<12>(int*);
template cudaError_t configure_tile_kernels<14>(int*);
template cudaError_t configure_tile_kernels<16>(int*);
template cudaError_t launch_kernel<8>(uint32_t, const Ctx&, cudaStream_t, int, uint32_t, int, int4*);
template cudaError_t launch_kernel<12>(uint32_t, const Ctx&, cudaStream_t, int, uint32_t, int, int4*);
template cudaError_t launch_kernel<14>(uint32_t, const Ctx&, cudaStream_t, int, uint32_t, int, int4*);
template cudaError_t launch_kernel<16>(uint32_t, const Ctx&, cudaStream_t, int, uint32_t, int, int4*);

}  // namespace mpm
