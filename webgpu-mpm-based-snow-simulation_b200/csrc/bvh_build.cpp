// bvh_build.cpp -- host-side collider BVH build in the reference node format.
//
// Follows src/lib/gpu/collider/GpuColliderBufferManager.ts:222-350 (build)
// and :183-202 (32-byte packing): per node the triangle bounds, split on the
// longest axis of the node bounds (ties prefer x, then y), triangles ordered
// by centroid with a stable sort, split at the median, leaves of at most 4
// triangles, nodes emitted in pre-order so a left child directly follows
// its parent.  The reference computes in JavaScript f64 numbers and sorts
// with the stable Array.prototype.sort; both are kept so node bounds and the
// triangle order match it exactly.  Math.min / Math.max order -0 below +0;
// js_min / js_max do the same.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/mpm.h"

namespace {

double js_min(double a, double b) { return (a < b || (a == b && std::signbit(a))) ? a : b; }
double js_max(double a, double b) { return (a > b || (a == b && !std::signbit(a))) ? a : b; }

struct TriBox {
    double lo[3], hi[3], centroid[3];
};

struct Builder {
    const std::vector<TriBox>& tris;
    std::vector<uint32_t>& order;
    uint32_t* out;  // 8 words per node
    uint32_t count = 0;

    static void put(uint32_t* w, double v) {
        float f = (float)v;
        std::memcpy(w, &f, 4);
    }

    uint32_t node(uint32_t begin, uint32_t end) {
        uint32_t id = count++;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (uint32_t i = begin; i < end; i++) {
            const TriBox& t = tris[order[i]];
            for (int k = 0; k < 3; k++) {
                lo[k] = js_min(lo[k], t.lo[k]);
                hi[k] = js_max(hi[k], t.hi[k]);
            }
        }
        uint32_t* w = out + (size_t)id * 8;
        put(w + 0, lo[0]); put(w + 1, lo[1]); put(w + 2, lo[2]);
        put(w + 4, hi[0]); put(w + 5, hi[1]); put(w + 6, hi[2]);
        uint32_t n = end - begin;
        if (n <= 4) {
            w[3] = begin;
            w[7] = n | 0x80000000u;
            return id;
        }
        double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        int axis = 0;
        if (ext[1] > ext[0] && ext[1] > ext[2]) axis = 1;
        else if (ext[2] > ext[0] && ext[2] > ext[1]) axis = 2;
        std::stable_sort(order.begin() + begin, order.begin() + end, [&](uint32_t a, uint32_t b) {
            return tris[a].centroid[axis] - tris[b].centroid[axis] < 0.0;
        });
        uint32_t mid = begin + n / 2;
        uint32_t left = node(begin, mid);
        uint32_t right = node(mid, end);
        w = out + (size_t)id * 8;
        w[3] = left;
        w[7] = right;
        return id;
    }
};

}  // namespace

extern "C" int mpm_build_bvh(const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_indices,
                             void* nodes_out, uint32_t* tri_order_out, uint32_t* n_nodes_out) {
    if (!nodes_out || !n_nodes_out || (n_indices && (!indices || !vertices || !tri_order_out))) return MPM_ERR_ARG;
    uint32_t* out = static_cast<uint32_t*>(nodes_out);
    uint32_t nt = n_indices / 3;
    if (nt == 0) {
        // a single empty leaf (GpuColliderBufferManager.ts:225-235)
        std::memset(out, 0, 32);
        out[7] = 0x80000000u;
        *n_nodes_out = 1;
        return MPM_OK;
    }
    std::vector<TriBox> tris(nt);
    for (uint32_t i = 0; i < nt; i++) {
        double v[3][3];
        for (int j = 0; j < 3; j++) {
            uint32_t vi = indices[i * 3 + j];
            if (vi >= n_vertices) return MPM_ERR_ARG;
            for (int k = 0; k < 3; k++) v[j][k] = (double)vertices[(size_t)vi * 3 + k];
        }
        for (int k = 0; k < 3; k++) {
            tris[i].lo[k] = js_min(js_min(v[0][k], v[1][k]), v[2][k]);
            tris[i].hi[k] = js_max(js_max(v[0][k], v[1][k]), v[2][k]);
            tris[i].centroid[k] = ((v[0][k] + v[1][k]) + v[2][k]) / 3.0;
        }
    }
    std::vector<uint32_t> order(nt);
    for (uint32_t i = 0; i < nt; i++) order[i] = i;
    Builder b{tris, order, out};
    b.node(0, nt);
    std::memcpy(tri_order_out, order.data(), (size_t)nt * 4);
    *n_nodes_out = b.count;
    return MPM_OK;
}
