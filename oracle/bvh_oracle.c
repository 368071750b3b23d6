/*
 * bvh_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Restatement of the reference's CPU BVH build
 * (src/lib/gpu/collider/GpuColliderBufferManager.ts:222-350) and of its
 * 32-byte node packing (:183-202).  JavaScript numbers are f64 and
 * Array.prototype.sort is stable (ES2019), so bounds, extents and centroids
 * are computed in f64 and the per-node centroid sort is a stable merge sort.
 * Math.min / Math.max order -0 below +0; js_min / js_max do the same.
 */
#include "mpm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static double js_min(double a, double b) { return (a < b || (a == b && signbit(a))) ? a : b; }
static double js_max(double a, double b) { return (a > b || (a == b && !signbit(a))) ? a : b; }

typedef struct {
    double mn[3], mx[3], ce[3];
} Tri;

typedef struct {
    const Tri* tris;
    uint32_t* order;
    uint32_t* tmp;
    uint32_t* nodes;
    uint32_t n_nodes;
} Build;

static void put_f(uint32_t* w, double v) { float f = (float)v; memcpy(w, &f, 4); }

/* stable merge sort of order[lo,hi) by centroid[axis] (comparator a - b) */
static void msort(Build* b, uint32_t lo, uint32_t hi, int axis) {
    if (hi - lo < 2) return;
    uint32_t mid = lo + (hi - lo) / 2;
    msort(b, lo, mid, axis);
    msort(b, mid, hi, axis);
    uint32_t i = lo, j = mid, k = lo;
    while (i < mid && j < hi) {
        double a = b->tris[b->order[i]].ce[axis], c = b->tris[b->order[j]].ce[axis];
        /* take from the right run only when strictly smaller: stable */
        if (c - a < 0) b->tmp[k++] = b->order[j++];
        else b->tmp[k++] = b->order[i++];
    }
    while (i < mid) b->tmp[k++] = b->order[i++];
    while (j < hi) b->tmp[k++] = b->order[j++];
    memcpy(b->order + lo, b->tmp + lo, (hi - lo) * sizeof(uint32_t));
}

static uint32_t rec(Build* b, uint32_t start, uint32_t end) {
    uint32_t node = b->n_nodes++;
    uint32_t count = end - start;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (uint32_t i = start; i < end; i++) {
        const Tri* t = &b->tris[b->order[i]];
        for (int k = 0; k < 3; k++) {
            mn[k] = js_min(mn[k], t->mn[k]);
            mx[k] = js_max(mx[k], t->mx[k]);
        }
    }
    uint32_t* w = b->nodes + (size_t)node * 8;
    put_f(w + 0, mn[0]); put_f(w + 1, mn[1]); put_f(w + 2, mn[2]);
    put_f(w + 4, mx[0]); put_f(w + 5, mx[1]); put_f(w + 6, mx[2]);
    if (count <= 4) {
        w[3] = start;
        w[7] = count | 0x80000000u;
        return node;
    }
    double ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    int axis = 0;
    if (ey > ex && ey > ez) axis = 1;
    else if (ez > ex && ez > ey) axis = 2;
    msort(b, start, end, axis);
    uint32_t mid = start + count / 2;
    uint32_t l = rec(b, start, mid);
    uint32_t r = rec(b, mid, end);
    w = b->nodes + (size_t)node * 8;
    w[3] = l;
    w[7] = r;
    return node;
}

uint32_t or_bvh_build(const float* v, uint32_t n_vertices, const uint32_t* idx, uint32_t n_indices,
                      uint32_t* nodes_out, uint32_t* tri_order_out) {
    (void)n_vertices;
    uint32_t nt = n_indices / 3;
    if (nt == 0) {
        memset(nodes_out, 0, 32);
        nodes_out[7] = 0x80000000u;
        return 1;
    }
    Tri* tris = (Tri*)malloc(sizeof(Tri) * nt);
    uint32_t* tmp = (uint32_t*)malloc(sizeof(uint32_t) * nt);
    for (uint32_t i = 0; i < nt; i++) {
        double p[3][3];
        for (int j = 0; j < 3; j++)
            for (int k = 0; k < 3; k++) p[j][k] = (double)v[(size_t)idx[i * 3 + j] * 3 + k];
        for (int k = 0; k < 3; k++) {
            double a = p[0][k], b = p[1][k], c = p[2][k];
            double mn = js_min(js_min(a, b), c);
            double mx = js_max(js_max(a, b), c);
            tris[i].mn[k] = mn;
            tris[i].mx[k] = mx;
            tris[i].ce[k] = ((a + b) + c) / 3.0;
        }
        tri_order_out[i] = i;
    }
    Build b = {tris, tri_order_out, tmp, nodes_out, 0};
    rec(&b, 0, nt);
    free(tris);
    free(tmp);
    return b.n_nodes;
}
