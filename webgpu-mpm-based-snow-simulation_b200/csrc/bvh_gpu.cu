// bvh_gpu.cu -- collider BVH build on the GPU, node for node the tree of the
// reference's host build (src/lib/gpu/collider/GpuColliderBufferManager.ts:222-350,
// restated on the host in bvh_build.cpp).
//
// The reference builds top down: node bounds from the triangle bounds, split
// axis = longest extent of the node bounds (ties prefer x, then y), the
// node's triangles stably sorted by centroid along that axis (JavaScript f64
// numbers, Array.prototype.sort with a - b), split at floor(count / 2),
// leaves of at most 4 triangles, nodes numbered in pre-order.  Which
// triangles a node holds depends on the sorts above it, but the shape of the
// tree does not: a node of n triangles has children of floor(n/2) and
// n - floor(n/2), so the host lays out every node (pre-order id, first
// triangle, count, children, depth) from the triangle count alone, and the
// GPU fills in the data-dependent parts level by level:
//   k_bvh_prep    per triangle: f32 bounds, f64 centroid ((v0 + v1) + v2) / 3;
//   k_bvh_level   one CTA per node of the level: bounds by block reduction,
//                 the 32-byte node, the split axis, and the sort key of each
//                 of its triangles (segment = first position, centroid on the axis);
//   radix sort    stable LSD radix sort of (segment, centroid key, triangle)
//                 over all positions, 8-bit digits: every segment is sorted
//                 in place and keeps ties in their previous order, which is
//                 exactly what the reference's stable per-node sort does.
// Leaves keep their (segment, 0) keys and so never move again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/mpm.h"

namespace mpm {
namespace bvhg {

constexpr int LEVEL_THREADS = 256;
constexpr int RS_THREADS = 256, RS_ITEMS = 8, RS_TILE = RS_THREADS * RS_ITEMS;

struct NodePlan {
    uint32_t id, start, count, left, right;
};

// Math.min / Math.max: -0 orders below +0 (the reference's bounds use them)
__device__ __forceinline__ float js_min(float a, float b) { return (a < b || (a == b && signbit(a))) ? a : b; }
__device__ __forceinline__ float js_max(float a, float b) { return (a > b || (a == b && !signbit(a))) ? a : b; }

// per triangle: bounds (f32 values, exact as f64), centroid (f64)
__global__ void k_bvh_prep(const float* __restrict__ v, uint32_t nv, const uint32_t* __restrict__ idx, uint32_t nt,
                           float* __restrict__ tlo, float* __restrict__ thi, double* __restrict__ cen,
                           uint32_t* __restrict__ perm, int* __restrict__ err) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    float p[3][3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        uint32_t vi = idx[(size_t)t * 3 + j];
        if (vi >= nv) {
            atomicExch(err, 1);
            vi = 0;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) p[j][k] = v[(size_t)vi * 3 + k];
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        tlo[(size_t)k * nt + t] = js_min(js_min(p[0][k], p[1][k]), p[2][k]);
        thi[(size_t)k * nt + t] = js_max(js_max(p[0][k], p[1][k]), p[2][k]);
        double s = __dadd_rn(__dadd_rn((double)p[0][k], (double)p[1][k]), (double)p[2][k]);
        cen[(size_t)k * nt + t] = __ddiv_rn(s, 3.0);
    }
    perm[t] = t;
}

// f64 -> u64 whose unsigned order is the numeric order; -0 and +0 are equal
__device__ __forceinline__ unsigned long long sort_key(double x) {
    if (x == 0.0) x = 0.0;
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__device__ __forceinline__ float warp_min(float x) {
    for (int o = 16; o > 0; o >>= 1) x = js_min(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}
__device__ __forceinline__ float warp_max(float x) {
    for (int o = 16; o > 0; o >>= 1) x = js_max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

__device__ __forceinline__ void put_f(uint32_t* w, float f) { *w = __float_as_uint(f); }

__global__ void __launch_bounds__(LEVEL_THREADS) k_bvh_level(const NodePlan* __restrict__ plan, const float* __restrict__ tlo,
                                                           const float* __restrict__ thi, const double* __restrict__ cen,
                                                           uint32_t nt, const uint32_t* __restrict__ perm,
                                                           unsigned long long* __restrict__ key_lo,
                                                           uint32_t* __restrict__ key_hi, uint32_t* __restrict__ nodes) {
    const NodePlan P = plan[blockIdx.x];
    float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float hi[3] = {-__int_as_float(0x7f800000), -__int_as_float(0x7f800000), -__int_as_float(0x7f800000)};
    for (uint32_t i = P.start + threadIdx.x; i < P.start + P.count; i += LEVEL_THREADS) {
        uint32_t t = perm[i];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            lo[k] = js_min(lo[k], tlo[(size_t)k * nt + t]);
            hi[k] = js_max(hi[k], thi[(size_t)k * nt + t]);
        }
    }
    __shared__ float red[2][3][LEVEL_THREADS / 32];
    __shared__ int axis_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float a = warp_min(lo[k]), b = warp_max(hi[k]);
        if (lane == 0) {
            red[0][k][warp] = a;
            red[1][k][warp] = b;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float L[3], H[3];
        for (int k = 0; k < 3; k++) {
            L[k] = red[0][k][0];
            H[k] = red[1][k][0];
            for (int w = 1; w < LEVEL_THREADS / 32; w++) {
                L[k] = js_min(L[k], red[0][k][w]);
                H[k] = js_max(H[k], red[1][k][w]);
            }
        }
        uint32_t* w = nodes + (size_t)P.id * 8;
        put_f(w + 0, L[0]); put_f(w + 1, L[1]); put_f(w + 2, L[2]);
        put_f(w + 4, H[0]); put_f(w + 5, H[1]); put_f(w + 6, H[2]);
        if (P.count <= 4) {
            w[3] = P.start;
            w[7] = P.count | 0x80000000u;
            axis_s = -1;
        } else {
            w[3] = P.left;
            w[7] = P.right;
            double ex = __dsub_rn((double)H[0], (double)L[0]), ey = __dsub_rn((double)H[1], (double)L[1]),
                   ez = __dsub_rn((double)H[2], (double)L[2]);
            int axis = 0;
            if (ey > ex && ey > ez) axis = 1;
            else if (ez > ex && ez > ey) axis = 2;
            axis_s = axis;
        }
    }
    __syncthreads();
    const int axis = axis_s;
    for (uint32_t i = P.start + threadIdx.x; i < P.start + P.count; i += LEVEL_THREADS) {
        key_hi[i] = P.start;
        key_lo[i] = axis < 0 ? 0ull : sort_key(cen[(size_t)axis * nt + perm[i]]);
    }
}

// ---- stable LSD radix sort, 8-bit digits ----------------------------------
__device__ __forceinline__ uint32_t digit_of(const unsigned long long* klo, const uint32_t* khi, uint32_t e, int pass) {
    return pass < 8 ? (uint32_t)(klo[e] >> (8 * pass)) & 255u : (khi[e] >> (8 * (pass - 8))) & 255u;
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const unsigned long long* __restrict__ klo,
                                                       const uint32_t* __restrict__ khi, uint32_t n, int pass,
                                                       uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ITEMS; r++) {
        uint32_t e = base + r * RS_THREADS + threadIdx.x;
        if (e < n) atomicAdd(&h[digit_of(klo, khi, e, pass)], 1u);
    }
    __syncthreads();
    counts[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of `total` counts in place, one CTA of 1024 threads
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t* __restrict__ counts, uint32_t total) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t b0 = 0; b0 < total; b0 += 1024) {
        uint32_t i = b0 + threadIdx.x;
        uint32_t v = i < total ? counts[i] : 0u;
        uint32_t x = v;
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
            wsum[lane] = s;   // inclusive over warps
        }
        __syncthreads();
        uint32_t incl = x + (warp > 0 ? wsum[warp - 1] : 0u);
        uint32_t c = carry;
        if (i < total) counts[i] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = c + incl;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const unsigned long long* __restrict__ klo,
                                                          const uint32_t* __restrict__ khi,
                                                          const uint32_t* __restrict__ val, uint32_t n, int pass,
                                                          const uint32_t* __restrict__ offsets,
                                                          unsigned long long* __restrict__ klo_out,
                                                          uint32_t* __restrict__ khi_out,
                                                          uint32_t* __restrict__ val_out) {
    constexpr int NW = RS_THREADS / 32;
    __shared__ uint32_t run[256];
    __shared__ uint32_t base_off[256];
    __shared__ uint32_t wc[NW][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    run[threadIdx.x] = 0;
    base_off[threadIdx.x] = offsets[(size_t)threadIdx.x * gridDim.x + blockIdx.x];
#pragma unroll
    for (int w = 0; w < NW; w++) wc[w][threadIdx.x] = 0;
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t base = blockIdx.x * RS_TILE;
    for (int r = 0; r < RS_ITEMS; r++) {
        const uint32_t e = base + r * RS_THREADS + threadIdx.x;
        const bool valid = e < n;
        // invalid slots get a digit of their own (>= 256) and are never written
        const uint32_t d = valid ? digit_of(klo, khi, e, pass) : 256u + (uint32_t)lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t wr = __popc(peers & lt);
        if (valid && wr == 0) wc[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pre = run[d];
            for (int w = 0; w < warp; w++) pre += wc[w][d];
            const uint32_t dst = base_off[d] + pre + wr;
            klo_out[dst] = klo[e];
            khi_out[dst] = khi[e];
            val_out[dst] = val[e];
        }
        __syncthreads();
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            s += wc[w][threadIdx.x];
            wc[w][threadIdx.x] = 0;
        }
        run[threadIdx.x] += s;
        __syncthreads();
    }
}

__global__ void k_reorder_indices(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ order, uint32_t nt,
                                  uint32_t* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt * 3u) return;
    out[i] = idx[(size_t)order[i / 3u] * 3u + i % 3u];
}

// Bounds of each collider triangle in leaf order, from the collider buffer
// (indices, then vertices at word num_indices + 3 v); a triangle whose index
// points past the buffer gets infinite bounds (never skipped).
__global__ void k_tri_boxes(const uint32_t* __restrict__ col, uint32_t words, uint32_t num_indices,
                            float4* __restrict__ boxes) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_indices / 3u) return;
    const float inf = __int_as_float(0x7f800000);
    float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
    bool ok = true;
    for (int j = 0; j < 3; j++) {
        const size_t base = (size_t)num_indices + (size_t)col[t * 3u + j] * 3u;
        if (base + 2u >= words) { ok = false; break; }
        for (int k = 0; k < 3; k++) {
            float x = __uint_as_float(col[base + k]);
            lo[k] = fminf(lo[k], x);
            hi[k] = fmaxf(hi[k], x);
        }
    }
    if (!ok) {
        for (int k = 0; k < 3; k++) { lo[k] = -inf; hi[k] = inf; }
    }
    boxes[2 * t] = make_float4(lo[0], lo[1], lo[2], 0.f);
    boxes[2 * t + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
}

// Squared distance from point p to triangle (a, b, c) in f64: the closest
// point by the Voronoi-region walk of Ericson, "Real-Time Collision Detection"
// (2005), section 5.1.5.
__device__ double point_tri_dist2(const double* p, const double* a, const double* b, const double* c) {
    double ab[3], ac[3], ap[3], q[3];
    for (int k = 0; k < 3; k++) { ab[k] = b[k] - a[k]; ac[k] = c[k] - a[k]; ap[k] = p[k] - a[k]; }
    auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) {
        for (int k = 0; k < 3; k++) q[k] = a[k];
    } else {
        double bp[3], cp[3];
        for (int k = 0; k < 3; k++) { bp[k] = p[k] - b[k]; cp[k] = p[k] - c[k]; }
        const double d3 = dot(ab, bp), d4 = dot(ac, bp), d5 = dot(ab, cp), d6 = dot(ac, cp);
        const double vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
        if (d3 >= 0.0 && d4 <= d3) {
            for (int k = 0; k < 3; k++) q[k] = b[k];
        } else if (d6 >= 0.0 && d5 <= d6) {
            for (int k = 0; k < 3; k++) q[k] = c[k];
        } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
            const double v = d1 / (d1 - d3);
            for (int k = 0; k < 3; k++) q[k] = a[k] + v * ab[k];
        } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
            const double w = d2 / (d2 - d6);
            for (int k = 0; k < 3; k++) q[k] = a[k] + w * ac[k];
        } else if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
            const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
            for (int k = 0; k < 3; k++) q[k] = b[k] + w * (c[k] - b[k]);
        } else {
            const double den = 1.0 / (va + vb + vc);
            const double v = vb * den, w = vc * den;
            for (int k = 0; k < 3; k++) q[k] = a[k] + ab[k] * v + ac[k] * w;
        }
    }
    double d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
    return dot(d, d);
}

// One thread per cell of the res^3 field: the distance from the cell centre
// to the nearest triangle (vertices read as the collider query reads them:
// a word past the buffer reads as 0), minus half the cell diagonal and a
// rounding allowance, rounded down to f32: a lower bound of the distance from
// any point of the cell to every triangle (0 where it would be negative).
__global__ void k_dist_field(const uint32_t* __restrict__ col, uint32_t words, uint32_t num_indices, double lo0,
                             double lo1, double lo2, double cs0, double cs1, double cs2, uint32_t res,
                             float* __restrict__ out) {
    const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= res * res * res) return;
    const uint32_t ix = cell % res, iy = (cell / res) % res, iz = cell / (res * res);
    const double p[3] = {lo0 + (ix + 0.5) * cs0, lo1 + (iy + 0.5) * cs1, lo2 + (iz + 0.5) * cs2};
    const uint32_t nt = num_indices / 3u;
    double best = 1e300;
    for (uint32_t t = 0; t < nt; t++) {
        double v[3][3];
        for (int j = 0; j < 3; j++) {
            const size_t base = (size_t)num_indices + (size_t)__ldg(col + 3u * t + j) * 3u;
            for (int k = 0; k < 3; k++)
                v[j][k] = base + k < words ? (double)__uint_as_float(__ldg(col + base + k)) : 0.0;
        }
        best = fmin(best, point_tri_dist2(p, v[0], v[1], v[2]));
    }
    const double half = 0.5 * sqrt(cs0 * cs0 + cs1 * cs1 + cs2 * cs2);
    const double mag = fmax(fmax(fabs(p[0]), fabs(p[1])), fabs(p[2]));
    const double lb = sqrt(best) - half - 1e-6 * (1.0 + mag);
    out[cell] = lb > 0.0 ? __double2float_rd(lb) : 0.0f;
}

uint32_t plan_nodes(uint32_t start, uint32_t count, uint32_t depth, std::vector<NodePlan>& out,
                    std::vector<uint32_t>& depth_of) {
    uint32_t id = (uint32_t)out.size();
    out.push_back({id, start, count, 0u, 0u});
    depth_of.push_back(depth);
    if (count > 4) {
        uint32_t mid = count / 2;
        uint32_t l = plan_nodes(start, mid, depth + 1, out, depth_of);
        uint32_t r = plan_nodes(start + mid, count - mid, depth + 1, out, depth_of);
        out[id].left = l;
        out[id].right = r;
    }
    return id;
}

}  // namespace bvhg

// Number of nodes of the tree over nt triangles (1 for an empty mesh).
uint32_t bvh_node_count(uint32_t nt) {
    if (nt <= 4) return 1;
    uint32_t m = nt / 2;
    return 1 + bvh_node_count(m) + bvh_node_count(nt - m);
}

// Builds on `stream`; returns 0, MPM_ERR_ARG (an index >= n_vertices) or
// MPM_ERR_CUDA.  Synchronises the stream before returning.
int bvh_build_device(const float* v, uint32_t nv, const uint32_t* idx, uint32_t n_indices, void* nodes_dev,
                     uint32_t* order_dev, cudaStream_t s, cudaError_t* cuda_err) {
    using namespace bvhg;
    const uint32_t nt = n_indices / 3;
    *cuda_err = cudaSuccess;
    uint32_t* nodes = static_cast<uint32_t*>(nodes_dev);
    if (nt == 0) {
        // a single empty leaf (GpuColliderBufferManager.ts:225-235)
        static const uint32_t empty[8] = {0, 0, 0, 0, 0, 0, 0, 0x80000000u};
        cudaError_t e = cudaMemcpyAsync(nodes, empty, 32, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        *cuda_err = e;
        return e == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
    }
    if (nv == 0) return MPM_ERR_ARG;   // every index would be out of range
    std::vector<NodePlan> plan;
    std::vector<uint32_t> depth_of;
    plan.reserve(nt);
    plan_nodes(0, nt, 0, plan, depth_of);
    const uint32_t depth_max = *std::max_element(depth_of.begin(), depth_of.end());
    // nodes grouped by depth
    std::vector<uint32_t> level_first(depth_max + 2, 0);
    for (uint32_t d : depth_of) level_first[d + 1]++;
    for (uint32_t d = 0; d <= depth_max; d++) level_first[d + 1] += level_first[d];
    std::vector<NodePlan> by_level(plan.size());
    std::vector<uint32_t> fill(level_first.begin(), level_first.end() - 1);
    std::vector<int> has_internal(depth_max + 1, 0);
    for (size_t i = 0; i < plan.size(); i++) {
        by_level[fill[depth_of[i]]++] = plan[i];
        if (plan[i].count > 4) has_internal[depth_of[i]] = 1;
    }
    // digit passes: 8 over the centroid key, then enough for the segment start
    int hi_passes = 0;
    for (uint32_t m = nt - 1; m; m >>= 8) hi_passes++;
    const uint32_t nb = (nt + RS_TILE - 1) / RS_TILE;

    char* ws = nullptr;
    size_t off = 0;
    auto carve = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t o_lo = carve((size_t)nt * 3 * 4), o_hi = carve((size_t)nt * 3 * 4), o_cen = carve((size_t)nt * 3 * 8),
                 o_perm = carve((size_t)nt * 4 * 2), o_klo = carve((size_t)nt * 8 * 2), o_khi = carve((size_t)nt * 4 * 2),
                 o_cnt = carve((size_t)256 * nb * 4), o_plan = carve(by_level.size() * sizeof(NodePlan)),
                 o_err = carve(4);
    cudaError_t e = cudaMallocAsync(&ws, off, s);
    if (e != cudaSuccess) {
        *cuda_err = e;
        return MPM_ERR_CUDA;
    }
    float* tlo = reinterpret_cast<float*>(ws + o_lo);
    float* thi = reinterpret_cast<float*>(ws + o_hi);
    double* cen = reinterpret_cast<double*>(ws + o_cen);
    uint32_t* perm[2] = {reinterpret_cast<uint32_t*>(ws + o_perm), reinterpret_cast<uint32_t*>(ws + o_perm) + nt};
    unsigned long long* klo[2] = {reinterpret_cast<unsigned long long*>(ws + o_klo),
                                  reinterpret_cast<unsigned long long*>(ws + o_klo) + nt};
    uint32_t* khi[2] = {reinterpret_cast<uint32_t*>(ws + o_khi), reinterpret_cast<uint32_t*>(ws + o_khi) + nt};
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + o_cnt);
    NodePlan* dplan = reinterpret_cast<NodePlan*>(ws + o_plan);
    int* derr = reinterpret_cast<int*>(ws + o_err);
    int cur = 0;
    e = cudaMemcpyAsync(dplan, by_level.data(), by_level.size() * sizeof(NodePlan), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, 4, s);
    if (e == cudaSuccess) {
        k_bvh_prep<<<(nt + 255) / 256, 256, 0, s>>>(v, nv, idx, nt, tlo, thi, cen, perm[0], derr);
        e = cudaGetLastError();
    }
    for (uint32_t d = 0; d <= depth_max && e == cudaSuccess; d++) {
        const uint32_t n_level = level_first[d + 1] - level_first[d];
        k_bvh_level<<<n_level, LEVEL_THREADS, 0, s>>>(dplan + level_first[d], tlo, thi, cen, nt, perm[cur], klo[cur],
                                                      khi[cur], nodes);
        e = cudaGetLastError();
        if (!has_internal[d]) continue;
        for (int pass = 0; pass < 8 + hi_passes && e == cudaSuccess; pass++) {
            k_rs_hist<<<nb, RS_THREADS, 0, s>>>(klo[cur], khi[cur], nt, pass, counts);
            k_rs_scan<<<1, 1024, 0, s>>>(counts, 256u * nb);
            k_rs_scatter<<<nb, RS_THREADS, 0, s>>>(klo[cur], khi[cur], perm[cur], nt, pass, counts, klo[cur ^ 1],
                                                   khi[cur ^ 1], perm[cur ^ 1]);
            e = cudaGetLastError();
            cur ^= 1;
        }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(order_dev, perm[cur], (size_t)nt * 4, cudaMemcpyDeviceToDevice, s);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(ws, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    *cuda_err = e;
    if (e != cudaSuccess) return MPM_ERR_CUDA;
    return herr ? MPM_ERR_ARG : MPM_OK;
}

cudaError_t triangle_boxes(const uint32_t* col_data, uint32_t words, uint32_t num_indices, float4* boxes,
                           cudaStream_t s) {
    const uint32_t nt = num_indices / 3u;
    if (nt == 0) return cudaSuccess;
    bvhg::k_tri_boxes<<<(nt + 255) / 256, 256, 0, s>>>(col_data, words, num_indices, boxes);
    return cudaGetLastError();
}

cudaError_t distance_field(const uint32_t* col_data, uint32_t words, uint32_t num_indices, const double* lo,
                           const double* cs, uint32_t res, float* out, cudaStream_t s) {
    const uint32_t n = res * res * res;
    if (n == 0 || num_indices < 3) return cudaSuccess;
    bvhg::k_dist_field<<<(n + 127) / 128, 128, 0, s>>>(col_data, words, num_indices, lo[0], lo[1], lo[2], cs[0],
                                                       cs[1], cs[2], res, out);
    return cudaGetLastError();
}

cudaError_t reorder_indices(const uint32_t* idx, const uint32_t* order, uint32_t nt, uint32_t* out, cudaStream_t s) {
    if (nt == 0) return cudaSuccess;
    bvhg::k_reorder_indices<<<(nt * 3 + 255) / 256, 256, 0, s>>>(idx, order, nt, out);
    return cudaGetLastError();
}

}  // namespace mpm

extern "C" uint32_t mpm_bvh_node_count(uint32_t n_triangles) { return mpm::bvh_node_count(n_triangles); }

extern "C" int mpm_build_bvh_device(const float* vertices_dev, uint32_t n_vertices, const uint32_t* indices_dev,
                                    uint32_t n_indices, void* nodes_dev, uint32_t* tri_order_dev,
                                    uint32_t* n_nodes_out, void* stream) {
    const uint32_t nt = n_indices / 3;
    if (!nodes_dev || !n_nodes_out || (nt && (!vertices_dev || !indices_dev || !tri_order_dev))) return MPM_ERR_ARG;
    cudaError_t ce;
    int r = mpm::bvh_build_device(vertices_dev, n_vertices, indices_dev, n_indices, nodes_dev, tri_order_dev,
                                  static_cast<cudaStream_t>(stream), &ce);
    if (r == MPM_OK) *n_nodes_out = mpm::bvh_node_count(nt);
    return r;
}
