// mpm_api.cu -- host engine behind the C ABI of include/mpm.h.
//
// The handle owns every device buffer (allocated in mpm_create), the
// per-scene parameter table and the CUDA graphs of the two substep
// schedules.  A substep is a fixed launch sequence on one stream; counts
// that change from step to step (occupied tiles, binned particles) stay on
// the device and the kernels read them there, so the sequence is graph-
// capturable and needs no host round trip.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/mpm.h"
#include "mpm_engine.cuh"
#include "mpm_math.cuh"
#include "mpm_mlp.cuh"

namespace mpm {
template <int E> cudaError_t configure_tile_kernels(int* blocks_per_sm);
template <int E> cudaError_t launch_kernel(uint32_t kid, const Ctx& c, cudaStream_t s, int grid_tiles, uint32_t scene,
                                           int apply, int4* out);
cudaError_t launch_selftest(uint64_t n, uint64_t seed, unsigned long long* counts, cudaStream_t s);
struct SplatArgs {
    const float4* particles;
    uint32_t first, count;
    float gmin[3], gmax[3];
    uint32_t res[3];
    float scale;
    uint32_t* out;
};
cudaError_t launch_splat(int kind, const SplatArgs& a, cudaStream_t s);
struct ScatterArgs {
    float4* particles;
    uint32_t n;
    const float4* verts;
    uint32_t n_tris;
    float mmin[3], mmax[3];
};
cudaError_t launch_scatter(const ScatterArgs& a, cudaStream_t s);
uint32_t bvh_node_count(uint32_t nt);
int bvh_build_device(const float* v, uint32_t nv, const uint32_t* idx, uint32_t n_indices, void* nodes_dev,
                     uint32_t* order_dev, cudaStream_t s, cudaError_t* cuda_err);
cudaError_t reorder_indices(const uint32_t* idx, const uint32_t* order, uint32_t nt, uint32_t* out, cudaStream_t s);
cudaError_t triangle_boxes(const uint32_t* col_data, uint32_t words, uint32_t num_indices, float4* boxes, cudaStream_t s);
cudaError_t distance_field(const uint32_t* col_data, uint32_t words, uint32_t num_indices, const double* lo,
                           const double* cs, uint32_t res, float* out, cudaStream_t s);
int mc_run(const uint32_t* density, const uint32_t* dres, const uint32_t* mres, const float* gmin, const float* gmax,
           float scale, float* out, uint32_t max_vertices, uint32_t* vertices_total, int n_sms, cudaStream_t s,
           cudaError_t* err);
}  // namespace mpm

using namespace mpm;

static const char* kKernelNames[K_COUNT] = {
    "clear_table", "bin_insert", "compact_a", "compact_b", "compact_c", "bin_scatter",
    "p2g_explicit", "g2p_explicit_integrate", "pbmpm_first", "pbmpm_iter", "g2p_pbmpm_integrate", "grid_dense",
    "tile_nbr", "plasticity", "tile_order", "p2g_explicit_b128", "g2p_explicit_integrate_b128", "pbmpm_iter_wide",
    "pbmpm_first_wide", "g2p_pbmpm_integrate_wide", "p2g_explicit_wide", "g2p_explicit_integrate_wide"};

struct TimedLaunch {
    uint32_t kid;
    cudaEvent_t a, b;
};

struct SceneHost {
    SceneDev dev;
    MpmParams params;
    uint8_t uni[MPM_UNIFORMS_BYTES];
    bool have_uniforms = false;
    uint32_t* col_data = nullptr;
    uint32_t* bvh = nullptr;
    float4* tbox = nullptr;   // per-triangle bounds (collide's early skip)
    float* dfield = nullptr;  // distance field (collide's whole-query skip)
    float df_lo[3] = {0.f, 0.f, 0.f}, df_rcs[3] = {0.f, 0.f, 0.f};
    uint32_t df_res = 0;
};

// Distance field of a collider: DF_RES^3 cells over the triangles' bounds
// widened by a tenth of their largest extent per side; built for meshes of at
// most DF_MAX_TRIANGLES triangles (one thread per cell tests every triangle).
constexpr uint32_t DF_RES = 32;
constexpr uint32_t DF_MAX_TRIANGLES = 16384;

struct MpmMlp {
    int device = 0;
    int n_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    float* params = nullptr;   // NPARAM FP32 masters
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* grad = nullptr;
    float* loss = nullptr;     // [2]: batch loss accumulator, epoch accumulator
    uint32_t* err = nullptr;
    uint32_t* idx = nullptr;   // shuffled pair order of one epoch
    uint32_t idx_cap = 0;
    int adam_step = 0;
    std::string msg;
};

struct MpmHandle {
    MpmConfig cfg{};
    int device = 0;
    int n_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    uint32_t tile_edge = 16;
    bool edge_pick = false;   // created with tile_edge 0: the library picks the edge
    bool edge_auto = false;   // the next sizing pass picks it (first step, new particle count)
    bool sizing_due = false;  // a new particle count: the next step sizes automatic storage again
    uint32_t cap = 0;
    uint32_t max_tiles = 0;
    size_t tiles_nc = 0;      // halo cells per tile the tile buffers were sized for
    bool auto_tiles = true;   // tile capacity sized from the first binning, grown at sync points
    bool auto_cap = true;     // hash capacity grown at sync points

    float4* particles = nullptr;      // the reference records in the caller's order (the boundary)
    bool own_particles = true;
    uint32_t n_particles = 0;
    // the state the substeps advance: REC_PLANES planes per buffer, slots in
    // tile order; work[work_cur] is current once work_valid
    float4* work[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};   // caller index of each work slot
    uint32_t* sorted = nullptr;
    int work_cur = 0;
    bool work_valid = false;       // false: `particles` holds the state (just set, bound or scattered)
    bool records_stale = false;    // `particles` is older than work[work_cur]
    uint32_t* bin_slot = nullptr;
    uint32_t* bin_rank = nullptr;
    unsigned long long* keys = nullptr;
    uint32_t* slot_count = nullptr;
    uint32_t* slot_off = nullptr;
    uint32_t* slot_st = nullptr;
    unsigned long long* st_key = nullptr;
    uint32_t* st_slot = nullptr;
    uint32_t* st_begin = nullptr;
    uint32_t* st_count = nullptr;
    uint32_t* chunk_nst = nullptr;
    uint32_t* chunk_np = nullptr;
    int4* tiles[3] = {nullptr, nullptr, nullptr};   // first transfer, then the PBMPM iterations' ping-pong
    int32_t* st_nbr = nullptr;    // max_tiles x 27 neighbour indices
    uint32_t* tile_order = nullptr;  // max_tiles: the tile kernels' claim order
    // deferred / learned plasticity
    int plast_mode = PLAST_INLINE;
    bool svd_any = false;          // some scene selects the SVD return map: plasticity runs deferred
    MpmMlp* mlp = nullptr;
    float unc_threshold = 0.05f, det_threshold = 1e-3f;
    uint32_t audit_threshold = 0;
    uint32_t* plast_list = nullptr;   // max_particles
    PlastStats* d_stats = nullptr;
    float* pair_x = nullptr;
    float* pair_t = nullptr;
    uint32_t* d_pair_count = nullptr;
    uint32_t pair_cap = 0;
    float4* iter_rec = nullptr;   // PBMPM iteration records, IR_PLANES x N float4
    int last_tiles = 0;
    SceneDev* d_scenes = nullptr;
    uint32_t* d_scene_first = nullptr;
    Counters* counters = nullptr;

    std::vector<SceneHost> scenes;
    uint32_t n_scenes = 1;
    std::vector<uint32_t> scene_first;  // n_scenes + 1
    bool scenes_dirty = true;

    int blocks_per_sm[K_COUNT] = {0};

    bool iter_wide = false;       // 512-thread tile-kernel CTAs (tile edge 8, few tiles)
    uint32_t order_mode = 0;      // schedule knobs (mpm_set_schedule)
    uint32_t tile_block = 0;
    bool use_graphs = true;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [method][parity]
    uint64_t graph_sig[2][2] = {{0, 0}, {0, 0}};

    bool timing = false;
    std::vector<TimedLaunch> pending;
    std::vector<cudaEvent_t> event_pool;
    double kms[K_COUNT] = {0};
    uint32_t kcount[K_COUNT] = {0};
};

static void destroy_graphs(MpmHandle* h);

static cudaError_t launch_e(uint32_t edge, uint32_t kid, const Ctx& c, cudaStream_t s, int grid, uint32_t scene,
                            int apply, int4* out) {
    switch (edge) {
        case 8: return launch_kernel<8>(kid, c, s, grid, scene, apply, out);
        case 12: return launch_kernel<12>(kid, c, s, grid, scene, apply, out);
        case 14: return launch_kernel<14>(kid, c, s, grid, scene, apply, out);
        default: return launch_kernel<16>(kid, c, s, grid, scene, apply, out);
    }
}

static int fail(MpmHandle* h, int code, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

#define CK(h, expr)                                                                              \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess) return fail((h), MPM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

static uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v && p < 0x80000000u) p <<= 1;
    return p;
}

extern "C" int mpm_default_params(MpmParams* p) {
    if (!p) return MPM_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->gravity[0] = 0.0f; p->gravity[1] = 0.0f; p->gravity[2] = -9.81f;
    p->youngs_modulus = 1.4e5f;
    p->poissons_ratio = 0.2f;
    p->hardening_explicit = 5.0f;
    p->hardening_pbmpm = 20.0f;
    p->theta_c = 2.5e-2f;
    p->theta_s = 7.5e-3f;
    p->density = 400.0f;
    p->n_iter = 3;
    p->force_divisor = 3.0f;
    p->boundary_mode = 0;
    p->restitution = -0.5f;
    p->bc_cells = 2;
    p->ground_axis = 2;
    p->collider_margin = 0.05f;
    p->collider_surface_margin = 0.05f;
    p->collider_threshold = 0.05f;
    p->collider_friction = 0.1f;
    p->collider_vel_scale = 0.2f;
    p->pbmpm_blend = 0.95f;
    p->pbmpm_volume_exponent = -0.3333333f;
    return MPM_OK;
}

static float rdf(const uint8_t* u, size_t off) { float f; std::memcpy(&f, u + off, 4); return f; }
static uint32_t rdu(const uint8_t* u, size_t off) { uint32_t v; std::memcpy(&v, u + off, 4); return v; }

// Fill the device scene record from the uniform block
// (shaderPrelude/uniforms.wgsl:8-56 offsets) and the extension parameters.
static void build_scene_dev(SceneHost& s) {
    SceneDev& d = s.dev;
    const uint8_t* u = s.uni;
    const MpmParams& e = s.params;
    const uint32_t* col = d.col_data;
    const uint32_t* bvh = d.bvh;
    const float4* tbox = d.tbox;
    uint32_t col_words = d.col_words, n_nodes = d.n_nodes, p_first = d.p_first, p_count = d.p_count;
    uint32_t c_nidx_override = d.c_nidx;
    std::memset(&d, 0, sizeof(d));
    d.dt = rdf(u, 0);
    d.scale = rdf(u, 4);
    for (int i = 0; i < 3; i++) {
        d.gmin[i] = rdf(u, 16 + 4 * i);
        d.gmax[i] = rdf(u, 32 + 4 * i);
        d.res[i] = (int32_t)rdu(u, 208 + 4 * i);
        d.cmin[i] = rdf(u, 224 + 4 * i);
        d.cmax[i] = rdf(u, 240 + 4 * i);
        d.cvel[i] = rdf(u, 320 + 4 * i);
        d.cd[i] = rdf(u, 352 + 4 * i);
        d.ipos[i] = rdf(u, 496 + 4 * i);
    }
    for (int i = 0; i < 16; i++) {
        d.xf[i] = rdf(u, 256 + 4 * i);
        d.xfi[i] = rdf(u, 432 + 4 * i);
    }
    d.c_nidx = rdu(u, 348);
    if (d.c_nidx == 0u) d.c_nidx = c_nidx_override;
    d.c_nobj = rdu(u, 364);
    d.istr = rdf(u, 508);
    d.irad = rdf(u, 512);
    d.iact = rdu(u, 516);
    d.imode = rdu(u, 520);
    for (int i = 0; i < 3; i++) d.g[i] = e.gravity[i];
    // WGSL folds these constant expressions in abstract (f64) precision and
    // rounds once (stressTensorOps.wgsl:5-6, plasticityOps.wgsl:18-19,
    // particleToGrid.cs.wgsl:37).
    double E = e.youngs_modulus, nu = e.poissons_ratio;
    d.mu0 = (float)(E / (2.0 * (1.0 + nu)));
    d.la0 = (float)(E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    d.xi_e = e.hardening_explicit;
    d.xi_p = e.hardening_pbmpm;
    d.smin = (float)(1.0 - (double)e.theta_c);
    d.smax = (float)(1.0 + (double)e.theta_s);
    d.inv_rho = (float)(1.0 / (double)e.density);
    d.n_iter = e.n_iter;
    d.fdiv = e.force_divisor;
    d.bmode = e.boundary_mode;
    d.rest = e.restitution;
    d.bc = (int32_t)e.bc_cells;
    d.gaxis = e.ground_axis > 2 ? 2 : e.ground_axis;
    d.cmargin = e.collider_margin;
    d.csurf = e.collider_surface_margin;
    d.cthr = e.collider_threshold;
    d.cfric = e.collider_friction;
    d.cvs = e.collider_vel_scale;
    d.blend = e.pbmpm_blend;
    d.vexp = e.pbmpm_volume_exponent;
    d.rmap = e.return_map == 1u ? 1u : 0u;
    d.p_first = p_first;
    d.p_count = p_count;
    d.col_data = col;
    d.bvh = bvh;
    d.col_words = col_words;
    d.n_nodes = n_nodes;
    d.tbox = tbox;
    bool ident = true;
    for (int i = 0; i < 16; i++) {
        float id = (i % 5 == 0) ? 1.0f : 0.0f;
        ident = ident && d.xf[i] == id && d.xfi[i] == id;
    }
    d.cull = (tbox && ident) ? 1u : 0u;
    d.dfield = s.dfield;
    for (int i = 0; i < 3; i++) {
        d.df_lo[i] = s.df_lo[i];
        d.df_rcs[i] = s.df_rcs[i];
    }
    d.df_res = s.dfield ? s.df_res : 0u;
    // Reciprocals RN(1/d) of the substep-constant divisors: one IEEE single
    // division each on the host, the value the oracle forms the same way.
    auto recip = [](float v) {
        volatile float one = 1.0f;
        return v != 0.0f ? one / v : 0.0f;
    };
    d.rdt = recip(d.dt);
    for (int i = 0; i < 3; i++) d.rcd[i] = recip(d.cd[i]);
    d.rscale = recip(d.scale);
    d.rfdiv = recip(d.fdiv);
    // loop-invariant operands of the step, each one IEEE f32 operation
    // exactly as the kernels would compute it: g * RN(1/force_divisor)
    // (pbmpm.wgsl:137) and g * dt (gridUpdate.cs.wgsl:44)
    for (int i = 0; i < 3; i++) {
        volatile float gi = d.g[i];
        d.gdiv[i] = gi * d.rfdiv;
        d.gdt[i] = gi * d.dt;
    }
    // Folded encodings (SceneDev::fold): the scale must be 2^k, 0 <= k < 126,
    // and RN(1/dt) * 2^k, dt * 2^k finite normal numbers (then exact).
    {
        uint32_t b;
        std::memcpy(&b, &d.scale, 4);
        int ex = (int)((b >> 23) & 0xffu) - 127;
        bool pow2 = (b & 0x807fffffu) == 0u && ex >= 0 && ex < 126;
        volatile float rdts = d.rdt * d.scale, dts = d.dt * d.scale;
        bool ok = pow2 && std::isnormal((float)rdts) && std::isnormal((float)dts) && std::isnormal(d.rdt) &&
                  std::isnormal(d.dt);
        d.fold = ok ? 1u : 0u;
        d.rdts = ok ? (float)rdts : 0.0f;
        d.dts = ok ? (float)dts : 0.0f;
    }
}

static void destroy_graphs(MpmHandle* h) {
    for (int m = 0; m < 2; m++)
        for (int p = 0; p < 2; p++) {
            if (h->graph[m][p]) cudaGraphExecDestroy(h->graph[m][p]);
            h->graph[m][p] = nullptr;
            h->graph_sig[m][p] = 0;
        }
}

extern "C" int mpm_destroy(MpmHandle* h) {
    if (!h) return MPM_ERR_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    destroy_graphs(h);
    for (auto& t : h->pending) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
    for (auto e : h->event_pool) cudaEventDestroy(e);
    void* bufs[] = {h->work[0], h->work[1], h->ids[0], h->ids[1], h->sorted, h->bin_slot, h->bin_rank, h->keys, h->slot_count, h->slot_off,
                    h->slot_st, h->st_key, h->st_slot, h->st_begin, h->st_count, h->chunk_nst, h->chunk_np,
                    h->tiles[0], h->tiles[1], h->tiles[2], h->d_scenes, h->d_scene_first, h->counters,
                    h->iter_rec, h->st_nbr, h->tile_order,
                    h->plast_list, h->d_stats, h->d_pair_count};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (h->own_particles && h->particles) cudaFree(h->particles);
    for (auto& s : h->scenes) {
        if (s.col_data) cudaFree(s.col_data);
        if (s.bvh) cudaFree(s.bvh);
        if (s.tbox) cudaFree(s.tbox);
        if (s.dfield) cudaFree(s.dfield);
    }
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MPM_OK;
}

extern "C" const char* mpm_last_error(const MpmHandle* h) { return h ? h->err.c_str() : "null handle"; }

// (Re)allocate the tile hash table for `cap` slots (a power of two >=
// COMPACT_CHUNK).  Only called between substeps, with the stream idle.
static int alloc_table(MpmHandle* h, uint32_t cap) {
    void* old[] = {h->keys, h->slot_count, h->slot_off, h->slot_st, h->st_key, h->st_slot, h->st_begin,
                   h->st_count, h->chunk_nst, h->chunk_np};
    for (void* b : old)
        if (b) cudaFree(b);
    h->cap = cap;
    CK(h, cudaMalloc(&h->keys, (size_t)cap * 8));
    CK(h, cudaMalloc(&h->slot_count, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->slot_off, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->slot_st, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->st_key, (size_t)cap * 8));
    CK(h, cudaMalloc(&h->st_slot, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->st_begin, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->st_count, (size_t)cap * 4));
    CK(h, cudaMalloc(&h->chunk_nst, (size_t)(cap / COMPACT_CHUNK) * 4));
    CK(h, cudaMalloc(&h->chunk_np, (size_t)(cap / COMPACT_CHUNK) * 4));
    CK(h, cudaMemsetAsync(h->keys, 0xff, (size_t)cap * 8, h->stream));
    CK(h, cudaMemsetAsync(h->slot_count, 0, (size_t)cap * 4, h->stream));
    // a fresh table holds no slots of a previous substep to clear
    CK(h, cudaMemsetAsync(&h->counters->n_st, 0, 4, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    destroy_graphs(h);
    return MPM_OK;
}

static int alloc_tiles(MpmHandle* h, uint32_t n) {
    for (int i = 0; i < 3; i++)
        if (h->tiles[i]) { cudaFree(h->tiles[i]); h->tiles[i] = nullptr; }
    if (h->st_nbr) { cudaFree(h->st_nbr); h->st_nbr = nullptr; }
    if (h->tile_order) { cudaFree(h->tile_order); h->tile_order = nullptr; }
    size_t NC = (size_t)(h->tile_edge + 2) * (h->tile_edge + 2) * (h->tile_edge + 2);
    h->max_tiles = n;
    h->tiles_nc = NC;
    for (int i = 0; i < 3; i++) CK(h, cudaMalloc(&h->tiles[i], (size_t)n * NC * 16));
    CK(h, cudaMalloc(&h->st_nbr, (size_t)n * 27 * 4));
    CK(h, cudaMalloc(&h->tile_order, (size_t)n * 4));
    destroy_graphs(h);
    return MPM_OK;
}

// Makes `edge` the handle's tile edge: the tile kernels' shared-memory limits
// and resident CTAs per SM for that edge.
static int set_tile_edge(MpmHandle* h, uint32_t edge) {
    cudaError_t ce = edge == 8u    ? configure_tile_kernels<8>(h->blocks_per_sm)
                     : edge == 12u ? configure_tile_kernels<12>(h->blocks_per_sm)
                     : edge == 14u ? configure_tile_kernels<14>(h->blocks_per_sm)
                                   : configure_tile_kernels<16>(h->blocks_per_sm);
    if (ce != cudaSuccess) return fail(h, MPM_ERR_CUDA, "configure kernels: %s", cudaGetErrorString(ce));
    h->tile_edge = edge;
    return MPM_OK;
}

extern "C" int mpm_create(const MpmConfig* cfg, MpmHandle** out) {
    if (!cfg || !out) return MPM_ERR_ARG;
    *out = nullptr;
    MpmHandle* h = new MpmHandle();
    h->cfg = *cfg;
    h->device = cfg->device;
    if (cfg->max_particles == 0) { *out = h; return fail(h, MPM_ERR_ARG, "max_particles must be > 0"); }
    h->edge_pick = h->edge_auto = cfg->tile_edge == 0u;
    h->tile_edge = cfg->tile_edge ? cfg->tile_edge : 16u;
    if (h->tile_edge != 8u && h->tile_edge != 12u && h->tile_edge != 14u && h->tile_edge != 16u) {
        *out = h;
        return fail(h, MPM_ERR_ARG, "tile_edge must be 8, 12, 14 or 16");
    }
    uint32_t max_scenes = cfg->max_scenes ? cfg->max_scenes : 1u;
    if (max_scenes > 65534u) { *out = h; return fail(h, MPM_ERR_ARG, "max_scenes must be <= 65534"); }
    uint32_t N = cfg->max_particles;
    h->auto_tiles = cfg->max_tiles == 0;
    h->max_tiles = cfg->max_tiles;
    h->auto_cap = cfg->hash_capacity == 0;
    uint32_t cap_req = cfg->hash_capacity ? cfg->hash_capacity : std::max(4u * cfg->max_tiles, std::min(N, 1u << 20));
    h->cap = std::max(next_pow2(cap_req), (uint32_t)COMPACT_CHUNK);
    *out = h;

    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "cudaSetDevice(%d): %s", h->device, cudaGetErrorString(e));
    CK(h, cudaDeviceGetAttribute(&h->n_sms, cudaDevAttrMultiProcessorCount, h->device));
    if (cfg->stream) {
        h->stream = (cudaStream_t)cfg->stream;
    } else {
        CK(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    CK(h, cudaMalloc(&h->particles, (size_t)N * MPM_PARTICLE_BYTES));
    for (int i = 0; i < 2; i++) {
        CK(h, cudaMalloc(&h->work[i], (size_t)N * MPM_PARTICLE_BYTES));
        CK(h, cudaMalloc(&h->ids[i], (size_t)N * 4));
    }
    CK(h, cudaMalloc(&h->sorted, (size_t)N * 4));
    CK(h, cudaMalloc(&h->bin_slot, (size_t)N * 4));
    CK(h, cudaMalloc(&h->bin_rank, (size_t)N * 4));
    CK(h, cudaMalloc(&h->iter_rec, (size_t)N * IR_PLANES * sizeof(float4)));
    CK(h, cudaMalloc(&h->d_scenes, (size_t)max_scenes * sizeof(SceneDev)));
    CK(h, cudaMalloc(&h->d_scene_first, (size_t)(max_scenes + 1) * 4));
    CK(h, cudaMalloc(&h->counters, sizeof(Counters)));
    CK(h, cudaMemsetAsync(h->counters, 0, sizeof(Counters), h->stream));
    CK(h, cudaMalloc(&h->d_stats, sizeof(PlastStats)));
    CK(h, cudaMemsetAsync(h->d_stats, 0, sizeof(PlastStats), h->stream));
    CK(h, cudaMalloc(&h->d_pair_count, 4));
    CK(h, cudaMemsetAsync(h->d_pair_count, 0, 4, h->stream));
    {
        int r = alloc_table(h, h->cap);
        if (r) return r;
    }
    if (!h->auto_tiles) {
        int r = alloc_tiles(h, h->max_tiles);
        if (r) return r;
    }
    CK(h, cudaMemsetAsync(h->particles, 0, (size_t)N * MPM_PARTICLE_BYTES, h->stream));
    h->scenes.resize(max_scenes);
    for (auto& s : h->scenes) {
        std::memset(s.uni, 0, sizeof(s.uni));
        mpm_default_params(&s.params);
        std::memset(&s.dev, 0, sizeof(s.dev));
    }
    h->n_scenes = 1;
    h->scene_first.assign(2, 0);
    h->n_particles = 0;
    {
        int r = set_tile_edge(h, h->tile_edge);
        if (r) return r;
    }
    CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

static int check_scene(MpmHandle* h, uint32_t scene) {
    if (!h) return MPM_ERR_ARG;
    if (scene >= h->scenes.size()) return fail(h, MPM_ERR_ARG, "scene %u out of range (max_scenes %zu)", scene, h->scenes.size());
    return MPM_OK;
}

extern "C" int mpm_set_uniforms(MpmHandle* h, uint32_t scene, const void* bytes, size_t n) {
    int r = check_scene(h, scene);
    if (r) return r;
    if (!bytes || n < 544) return fail(h, MPM_ERR_ARG, "uniform block needs >= 544 bytes, got %zu", n);
    SceneHost& s = h->scenes[scene];
    uint8_t next[MPM_UNIFORMS_BYTES];
    std::memset(next, 0, sizeof(next));
    std::memcpy(next, bytes, std::min(n, (size_t)MPM_UNIFORMS_BYTES));
    if (s.have_uniforms && std::memcmp(next, s.uni, sizeof(next)) == 0) return MPM_OK;
    std::memcpy(s.uni, next, sizeof(next));
    s.have_uniforms = true;
    h->scenes_dirty = true;
    return MPM_OK;
}

extern "C" int mpm_set_params(MpmHandle* h, uint32_t scene, const MpmParams* p) {
    int r = check_scene(h, scene);
    if (r) return r;
    if (!p) return fail(h, MPM_ERR_ARG, "null params");
    if (p->n_iter == 0) return fail(h, MPM_ERR_ARG, "n_iter must be >= 1");
    h->scenes[scene].params = *p;
    h->scenes_dirty = true;
    destroy_graphs(h);  // n_iter may have changed the schedule
    return MPM_OK;
}

extern "C" int mpm_set_scene_count(MpmHandle* h, uint32_t n_scenes) {
    if (!h) return MPM_ERR_ARG;
    if (n_scenes == 0 || n_scenes > h->scenes.size()) return fail(h, MPM_ERR_ARG, "bad scene count %u", n_scenes);
    h->n_scenes = n_scenes;
    h->scene_first.resize(n_scenes + 1, h->n_particles);
    h->scenes_dirty = true;
    destroy_graphs(h);
    return MPM_OK;
}

extern "C" int mpm_set_scene_range(MpmHandle* h, uint32_t scene, uint32_t first, uint32_t count) {
    int r = check_scene(h, scene);
    if (r) return r;
    if (scene >= h->n_scenes) return fail(h, MPM_ERR_ARG, "scene %u >= scene count %u", scene, h->n_scenes);
    h->scenes[scene].dev.p_first = first;
    h->scenes[scene].dev.p_count = count;
    h->scenes_dirty = true;
    destroy_graphs(h);
    return MPM_OK;
}

static int set_count(MpmHandle* h, uint32_t n) {
    if (n != h->n_particles) {
        h->n_particles = n;
        h->work_valid = false;
        h->edge_auto = h->edge_pick;  // a new particle count: the next step picks the edge again
        h->sizing_due = h->auto_tiles && h->auto_cap;
        destroy_graphs(h);
        if (h->n_scenes == 1) {
            h->scenes[0].dev.p_first = 0;
            h->scenes[0].dev.p_count = n;
            h->scenes_dirty = true;
        }
    }
    return MPM_OK;
}

// Caller records -> work planes (slot t = caller index t).  One thread per
// record word: a warp reads 512 contiguous bytes of records and writes two or
// three runs of each plane.
__global__ void k_work_load(const float4* rec, uint32_t n, float4* work, uint32_t* ids) {
    const size_t total = (size_t)n * REC_PLANES;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(i / REC_PLANES), q = (uint32_t)(i % REC_PLANES);
        work[(size_t)q * n + t] = rec[i];
        if (q == 0u) ids[t] = t;
    }
}

// Work planes -> caller records: word q of slot t goes to record ids[t]
// (consecutive threads write the consecutive words of one record).
__global__ void k_work_store(const float4* work, const uint32_t* ids, uint32_t n, float4* rec) {
    const size_t total = (size_t)n * REC_PLANES;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(i / REC_PLANES), q = (uint32_t)(i % REC_PLANES);
        rec[(size_t)__ldg(ids + t) * REC_PLANES + q] = work[(size_t)q * n + t];
    }
}

static unsigned work_grid(uint32_t n) {
    size_t blocks = ((size_t)n * REC_PLANES + 255u) / 256u;
    return (unsigned)std::max<size_t>(1, std::min<size_t>(blocks, 148u * 16u));
}

// Brings the caller-order records up to date with the work state (enqueued on
// the handle's stream): called before anything reads `particles`.
static int flush_records(MpmHandle* h) {
    if (!h->records_stale || !h->work_valid || h->n_particles == 0) return MPM_OK;
    k_work_store<<<work_grid(h->n_particles), 256, 0, h->stream>>>(h->work[h->work_cur], h->ids[h->work_cur],
                                                                   h->n_particles, h->particles);
    CK(h, cudaGetLastError());
    h->records_stale = false;
    return MPM_OK;
}

extern "C" int mpm_set_particles(MpmHandle* h, const void* src, uint32_t n, int src_is_device) {
    if (!h || (!src && n)) return MPM_ERR_ARG;
    if (n > h->cfg.max_particles) return fail(h, MPM_ERR_CAPACITY, "%u particles > max_particles %u", n, h->cfg.max_particles);
    if (!h->own_particles) return fail(h, MPM_ERR_STATE, "particles are bound to a caller buffer");
    cudaSetDevice(h->device);
    if (n) CK(h, cudaMemcpyAsync(h->particles, src, (size_t)n * MPM_PARTICLE_BYTES,
                                 src_is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream));
    set_count(h, n);
    h->work_valid = false;
    h->records_stale = false;
    return MPM_OK;
}

extern "C" int mpm_get_particles(MpmHandle* h, void* dst, uint32_t n, int dst_is_device) {
    if (!h || (!dst && n)) return MPM_ERR_ARG;
    if (n > h->n_particles) return fail(h, MPM_ERR_ARG, "asked for %u particles, have %u", n, h->n_particles);
    cudaSetDevice(h->device);
    int r = flush_records(h);
    if (r) return r;
    if (n) CK(h, cudaMemcpyAsync(dst, h->particles, (size_t)n * MPM_PARTICLE_BYTES,
                                 dst_is_device == 1 ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream));
    if (dst_is_device == 0) CK(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
}

extern "C" int mpm_bind_particles_device(MpmHandle* h, void* dptr, uint32_t n) {
    if (!h || !dptr) return MPM_ERR_ARG;
    if (n > h->cfg.max_particles) return fail(h, MPM_ERR_CAPACITY, "%u particles > max_particles %u", n, h->cfg.max_particles);
    if (((uintptr_t)dptr & 15u) != 0) return fail(h, MPM_ERR_ARG, "particle buffer must be 16-byte aligned");
    cudaSetDevice(h->device);
    if (h->own_particles && h->particles) cudaFree(h->particles);
    h->particles = (float4*)dptr;
    h->own_particles = false;
    destroy_graphs(h);
    set_count(h, n);
    h->work_valid = false;
    h->records_stale = false;
    return MPM_OK;
}

extern "C" void* mpm_particles_device_ptr(MpmHandle* h) {
    if (!h) return nullptr;
    cudaSetDevice(h->device);
    if (flush_records(h)) return nullptr;
    return (void*)h->particles;
}

// (Re)builds scene s's distance field from its collider buffer and triangle
// bounds (the stream is idle on entry and on return).  No field (and so no
// whole-query skip) for meshes past DF_MAX_TRIANGLES or with non-finite bounds.
static int build_field(MpmHandle* h, SceneHost& s, size_t words, uint32_t num_indices) {
    if (s.dfield) { cudaFree(s.dfield); s.dfield = nullptr; }
    s.df_res = 0;
    const uint32_t nt = num_indices / 3u;
    if (nt == 0 || nt > DF_MAX_TRIANGLES || !s.tbox || !s.col_data) return MPM_OK;
    std::vector<float4> boxes((size_t)nt * 2);
    CK(h, cudaMemcpy(boxes.data(), s.tbox, (size_t)nt * 32, cudaMemcpyDeviceToHost));
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (uint32_t t = 0; t < nt; t++) {
        const float a[3] = {boxes[2 * t].x, boxes[2 * t].y, boxes[2 * t].z};
        const float b[3] = {boxes[2 * t + 1].x, boxes[2 * t + 1].y, boxes[2 * t + 1].z};
        for (int k = 0; k < 3; k++) {
            if (!std::isfinite(a[k]) || !std::isfinite(b[k])) return MPM_OK;
            lo[k] = std::min(lo[k], (double)a[k]);
            hi[k] = std::max(hi[k], (double)b[k]);
        }
    }
    const double ext = std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), std::max(hi[2] - lo[2], 1e-6));
    double cs[3];
    for (int k = 0; k < 3; k++) {
        lo[k] -= 0.1 * ext;
        hi[k] += 0.1 * ext;
        cs[k] = (hi[k] - lo[k]) / DF_RES;
    }
    CK(h, cudaMalloc(&s.dfield, (size_t)DF_RES * DF_RES * DF_RES * 4));
    CK(h, distance_field(s.col_data, (uint32_t)words, num_indices, lo, cs, DF_RES, s.dfield, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    // the query maps a position to cell floor((x - lo) * rcs): with lo and rcs
    // rounded to f32 that may pick a neighbouring cell, so the stored bounds
    // are each lowered to their 3^3 neighbourhood's minimum
    std::vector<float> f((size_t)DF_RES * DF_RES * DF_RES), g(f.size());
    CK(h, cudaMemcpy(f.data(), s.dfield, f.size() * 4, cudaMemcpyDeviceToHost));
    const int R = (int)DF_RES;
    for (int z = 0; z < R; z++)
        for (int y = 0; y < R; y++)
            for (int x = 0; x < R; x++) {
                float m = f[((size_t)z * R + y) * R + x];
                for (int dz = -1; dz <= 1; dz++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dx = -1; dx <= 1; dx++) {
                            const int X = x + dx, Y = y + dy, Z = z + dz;
                            if (X < 0 || Y < 0 || Z < 0 || X >= R || Y >= R || Z >= R) continue;
                            m = std::min(m, f[((size_t)Z * R + Y) * R + X]);
                        }
                g[((size_t)z * R + y) * R + x] = m;
            }
    CK(h, cudaMemcpy(s.dfield, g.data(), g.size() * 4, cudaMemcpyHostToDevice));
    s.df_res = DF_RES;
    for (int k = 0; k < 3; k++) {
        s.df_lo[k] = (float)lo[k];
        s.df_rcs[k] = (float)(1.0 / cs[k]);
    }
    return MPM_OK;
}

extern "C" int mpm_set_collider(MpmHandle* h, uint32_t scene, const uint32_t* data, size_t words, uint32_t num_indices,
                                const void* nodes, uint32_t n_nodes) {
    int r = check_scene(h, scene);
    if (r) return r;
    if ((words && !data) || (n_nodes && !nodes)) return fail(h, MPM_ERR_ARG, "null collider buffer");
    if ((size_t)num_indices > words) return fail(h, MPM_ERR_ARG, "num_indices %u > words %zu", num_indices, words);
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    SceneHost& s = h->scenes[scene];
    if (s.col_data) { cudaFree(s.col_data); s.col_data = nullptr; }
    if (s.bvh) { cudaFree(s.bvh); s.bvh = nullptr; }
    if (words) {
        CK(h, cudaMalloc(&s.col_data, words * 4));
        CK(h, cudaMemcpy(s.col_data, data, words * 4, cudaMemcpyHostToDevice));
    }
    if (n_nodes) {
        CK(h, cudaMalloc(&s.bvh, (size_t)n_nodes * MPM_BVH_NODE_BYTES));
        CK(h, cudaMemcpy(s.bvh, nodes, (size_t)n_nodes * MPM_BVH_NODE_BYTES, cudaMemcpyHostToDevice));
    }
    if (s.tbox) { cudaFree(s.tbox); s.tbox = nullptr; }
    if (num_indices >= 3 && words) {
        CK(h, cudaMalloc(&s.tbox, (size_t)(num_indices / 3) * 32));
        CK(h, triangle_boxes(s.col_data, (uint32_t)words, num_indices, s.tbox, h->stream));
        CK(h, cudaStreamSynchronize(h->stream));
    }
    {
        int fr = build_field(h, s, words, num_indices);
        if (fr) return fr;
    }
    s.dev.col_data = s.col_data;
    s.dev.bvh = s.bvh;
    s.dev.tbox = s.tbox;
    s.dev.col_words = (uint32_t)words;
    s.dev.n_nodes = n_nodes;
    s.dev.c_nidx = num_indices;  // GpuMpmPipelineManager.ts:80 writes colliderNumIndices
    if (s.have_uniforms) std::memcpy(s.uni + 348, &num_indices, 4);
    h->scenes_dirty = true;
    return MPM_OK;
}

extern "C" int mpm_set_collider_mesh_device(MpmHandle* h, uint32_t scene, const float* vertices_dev,
                                            uint32_t n_vertices, const uint32_t* indices_dev, uint32_t n_indices) {
    int r = check_scene(h, scene);
    if (r) return r;
    const uint32_t nt = n_indices / 3;
    if (n_indices % 3) return fail(h, MPM_ERR_ARG, "n_indices %u is not a multiple of 3", n_indices);
    if (nt && (!vertices_dev || !indices_dev)) return fail(h, MPM_ERR_ARG, "null mesh buffer");
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    SceneHost& s = h->scenes[scene];
    if (s.col_data) { cudaFree(s.col_data); s.col_data = nullptr; }
    if (s.bvh) { cudaFree(s.bvh); s.bvh = nullptr; }
    const uint32_t n_nodes = bvh_node_count(nt);
    const size_t words = (size_t)n_indices + (size_t)n_vertices * 3;
    uint32_t* order = nullptr;
    CK(h, cudaMalloc(&s.bvh, (size_t)n_nodes * MPM_BVH_NODE_BYTES));
    if (words) CK(h, cudaMalloc(&s.col_data, words * 4));
    if (nt) CK(h, cudaMalloc(&order, (size_t)nt * 4));
    cudaError_t ce = cudaSuccess;
    r = bvh_build_device(vertices_dev, n_vertices, indices_dev, n_indices, s.bvh, order, h->stream, &ce);
    if (r == MPM_OK && nt) ce = reorder_indices(indices_dev, order, nt, s.col_data, h->stream);
    if (r == MPM_OK && ce == cudaSuccess && n_vertices)
        ce = cudaMemcpyAsync(s.col_data + n_indices, vertices_dev, (size_t)n_vertices * 12, cudaMemcpyDeviceToDevice,
                             h->stream);
    if (s.tbox) { cudaFree(s.tbox); s.tbox = nullptr; }
    if (r == MPM_OK && ce == cudaSuccess && nt) {
        ce = cudaMalloc(&s.tbox, (size_t)nt * 32);
        if (ce == cudaSuccess) ce = triangle_boxes(s.col_data, (uint32_t)words, n_indices, s.tbox, h->stream);
    }
    if (r == MPM_OK && ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (order) cudaFree(order);
    if (r == MPM_ERR_ARG) return fail(h, MPM_ERR_ARG, "mesh index >= n_vertices (%u)", n_vertices);
    if (r != MPM_OK || ce != cudaSuccess) return fail(h, MPM_ERR_CUDA, "device BVH build: %s", cudaGetErrorString(ce));
    r = build_field(h, s, words, n_indices);
    if (r) return r;
    s.dev.col_data = s.col_data;
    s.dev.bvh = s.bvh;
    s.dev.tbox = s.tbox;
    s.dev.col_words = (uint32_t)words;
    s.dev.n_nodes = n_nodes;
    s.dev.c_nidx = n_indices;
    if (s.have_uniforms) std::memcpy(s.uni + 348, &n_indices, 4);
    h->scenes_dirty = true;
    return MPM_OK;
}

static int upload_scenes(MpmHandle* h) {
    if (!h->scenes_dirty) return MPM_OK;
    // scene ranges must tile [0, n_particles)
    std::vector<uint32_t> first(h->n_scenes + 1);
    uint32_t expect = 0;
    for (uint32_t s = 0; s < h->n_scenes; s++) {
        SceneHost& sc = h->scenes[s];
        if (!sc.have_uniforms) return fail(h, MPM_ERR_STATE, "scene %u has no uniforms", s);
        if (sc.dev.p_first != expect)
            return fail(h, MPM_ERR_ARG, "scene %u starts at %u, expected %u (ranges must tile the buffer)", s, sc.dev.p_first, expect);
        first[s] = expect;
        expect += sc.dev.p_count;
        build_scene_dev(sc);
        if (sc.dev.scale <= 0.0f || !(sc.dev.dt > 0.0f))
            return fail(h, MPM_ERR_ARG, "scene %u: fixedPointScale and timestep must be > 0", s);
        if (sc.dev.res[0] <= 0 || sc.dev.res[1] <= 0 || sc.dev.res[2] <= 0)
            return fail(h, MPM_ERR_ARG, "scene %u: grid resolution must be > 0", s);
        if (sc.params.n_iter != h->scenes[0].params.n_iter)
            return fail(h, MPM_ERR_ARG, "all scenes of a handle must share n_iter");
    }
    if (expect != h->n_particles)
        return fail(h, MPM_ERR_ARG, "scene ranges cover %u particles, buffer holds %u", expect, h->n_particles);
    first[h->n_scenes] = expect;
    h->scene_first = first;
    bool svd = false;
    for (uint32_t s = 0; s < h->n_scenes; s++) svd = svd || h->scenes[s].dev.rmap == 1u;
    if (svd != h->svd_any) {
        h->svd_any = svd;
        destroy_graphs(h);
    }
    if (svd && !h->plast_list) CK(h, cudaMalloc(&h->plast_list, (size_t)h->cfg.max_particles * 4));
    std::vector<SceneDev> tmp(h->n_scenes);
    for (uint32_t s = 0; s < h->n_scenes; s++) tmp[s] = h->scenes[s].dev;
    CK(h, cudaMemcpyAsync(h->d_scenes, tmp.data(), tmp.size() * sizeof(SceneDev), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaMemcpyAsync(h->d_scene_first, h->scene_first.data(), h->scene_first.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));  // host staging vectors go out of scope
    h->scenes_dirty = false;
    return MPM_OK;
}

// identity order for the first substep after new particles
__global__ void k_iota(uint32_t* o, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = i;
}

static Ctx make_ctx(MpmHandle* h, int cur) {
    Ctx c{};
    c.work_in = h->work[cur];
    c.work_out = h->work[cur ^ 1];
    c.ids_in = h->ids[cur];
    c.ids_out = h->ids[cur ^ 1];
    c.sorted = h->sorted;
    c.bin_slot = h->bin_slot;
    c.bin_rank = h->bin_rank;
    c.keys = h->keys;
    c.slot_count = h->slot_count;
    c.slot_off = h->slot_off;
    c.slot_st = h->slot_st;
    c.st_key = h->st_key;
    c.st_slot = h->st_slot;
    c.st_begin = h->st_begin;
    c.st_count = h->st_count;
    c.chunk_nst = h->chunk_nst;
    c.chunk_np = h->chunk_np;
    c.tiles_a = h->tiles[0];
    c.tiles_b = h->tiles[0];
    c.iter_rec = h->iter_rec;
    c.st_nbr = h->st_nbr;
    c.tile_order = h->tile_order;
    c.order_mode = h->order_mode;
    c.plast_list = h->plast_list;
    c.plast_defer = (h->plast_mode != PLAST_INLINE || h->svd_any) ? 1u : 0u;
    c.scenes = h->d_scenes;
    c.scene_first = h->d_scene_first;
    c.counters = h->counters;
    c.n_particles = h->n_particles;
    c.n_scenes = h->n_scenes;
    c.cap = h->cap;
    c.max_tiles = h->max_tiles;
    return c;
}

static cudaEvent_t get_event(MpmHandle* h) {
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

static void drain_timing(MpmHandle* h) {
    if (h->pending.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto& t : h->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
            h->kms[t.kid] += ms;
            h->kcount[t.kid] += 1;
        }
        h->event_pool.push_back(t.a);
        h->event_pool.push_back(t.b);
    }
    h->pending.clear();
}

static cudaError_t launch(MpmHandle* h, uint32_t kid, const Ctx& c, bool capturing) {
    int grid = std::max(1, h->n_sms * std::max(1, h->blocks_per_sm[kid]));
    bool timed = h->timing && !capturing;
    TimedLaunch tl{kid, nullptr, nullptr};
    if (timed) {
        tl.a = get_event(h);
        tl.b = get_event(h);
        cudaEventRecord(tl.a, h->stream);
    }
    cudaError_t e;
    if (kid == K_PLASTICITY) {
        PlastCtx pc{};
        pc.params = h->mlp ? h->mlp->params : nullptr;
        pc.unc_threshold = h->unc_threshold;
        pc.det_threshold = h->det_threshold;
        pc.audit_threshold = h->audit_threshold;
        pc.stats = h->d_stats;
        pc.pair_x = h->pair_x;
        pc.pair_t = h->pair_t;
        pc.pair_count = h->d_pair_count;
        pc.pair_cap = h->pair_cap;
        // INLINE with an SVD scene: the exact pass applies each scene's map
        const int pm = h->plast_mode == PLAST_INLINE ? PLAST_EXACT : h->plast_mode;
        e = launch_plasticity(pm, c, pc, h->n_sms * (pm == PLAST_LEARNED ? (int)MLP_CTAS_PER_SM : 8), h->stream);
    } else {
        e = launch_e(h->tile_edge, kid, c, h->stream, grid, 0, 0, nullptr);
    }
    if (timed) {
        cudaEventRecord(tl.b, h->stream);
        h->pending.push_back(tl);
        if (h->pending.size() > 4096) drain_timing(h);
    }
    return e;
}

// One substep's launch sequence (GpuMpmPipelineManager.ts:327-428 explicit,
// :431-521 PBMPM).  stop_p2g ends after the first particle-to-grid pass.
static cudaError_t enqueue_substep(MpmHandle* h, int method, int parity, bool capturing, bool stop_p2g) {
    Ctx c = make_ctx(h, parity);
    cudaError_t e;
#define L(k)                                   \
    do {                                       \
        e = launch(h, (k), c, capturing);      \
        if (e != cudaSuccess) return e;        \
    } while (0)
    L(K_CLEAR_TABLE);
    L(K_BIN_INSERT);
    L(K_COMPACT_A);
    L(K_COMPACT_B);
    L(K_COMPACT_C);
    L(K_BIN_SCATTER);
    L(K_TILE_NBR);
    L(K_TILE_ORDER);
    // each tile pass claims the tile order from the other end than the pass
    // before it (which wrote the tiles it reads)
    c.order_rev = 0u;
    if (method == MPM_METHOD_EXPLICIT) {
        // CTA width: the schedule knob, else 512 threads for few tiles at edge 8
        const bool b128 = h->tile_block == 128u;
        const uint32_t k_p2g = b128 ? K_P2G_EXPLICIT_128 : h->iter_wide ? K_P2G_EXPLICIT_WIDE : K_P2G_EXPLICIT;
        const uint32_t k_g2p = b128 ? K_G2P_EXPLICIT_128 : h->iter_wide ? K_G2P_EXPLICIT_WIDE : K_G2P_EXPLICIT;
        c.tiles_a = h->tiles[0];
        L(k_p2g);
        if (stop_p2g) { h->last_tiles = 0; return cudaSuccess; }
        c.tiles_b = h->tiles[0];
        c.order_rev = 1u;
        L(k_g2p);
        if (h->plast_mode != PLAST_INLINE || h->svd_any) L(K_PLASTICITY);
        h->last_tiles = 0;
    } else {
        // tiles[0] keeps the first transfer (with the mass sums); the
        // iterations alternate between tiles[1] and tiles[2]
        uint32_t n_iter = h->scenes[0].params.n_iter;
        int cur = 0;
        c.tiles_a = h->tiles[cur];
        L(h->iter_wide ? K_PBMPM_FIRST_WIDE : K_PBMPM_FIRST);
        if (stop_p2g) { h->last_tiles = cur; return cudaSuccess; }
        for (uint32_t it = 1; it < n_iter; it++) {
            int nxt = cur == 1 ? 2 : 1;
            c.tiles_b = h->tiles[cur];
            c.tiles_a = h->tiles[nxt];
            c.iter_first = it == 1 ? 1u : 0u;
            c.order_rev = it & 1u;
            L(h->iter_wide ? K_PBMPM_ITER_WIDE : K_PBMPM_ITER);
            cur = nxt;
        }
        c.tiles_b = h->tiles[cur];
        c.g2p_rm = n_iter > 1 ? 1u : 0u;
        c.order_rev = n_iter & 1u;
        L(h->iter_wide ? K_G2P_PBMPM_WIDE : K_G2P_PBMPM);
        if (h->plast_mode != PLAST_INLINE || h->svd_any) L(K_PLASTICITY);
        h->last_tiles = cur;
    }
#undef L
    return cudaSuccess;
}

static int read_counters(MpmHandle* h, Counters* ct) {
    CK(h, cudaStreamSynchronize(h->stream));
    CK(h, cudaMemcpy(ct, h->counters, sizeof(*ct), cudaMemcpyDeviceToHost));
    return MPM_OK;
}

static uint32_t tiles_for(uint32_t n_st) { return std::max(1024u, n_st + n_st / 2u + 256u); }

// One binning pass over the current particles at the handle's tile edge (no
// tile data is touched), growing an automatic hash table until it holds four
// slots per occupied tile.  *n_st gets the occupied tiles; *full is set when a
// table of fixed capacity overflowed.
static int binning_pass(MpmHandle* h, uint32_t* n_st, bool* full) {
    for (int attempt = 0; attempt < 4; attempt++) {
        Ctx c = make_ctx(h, h->work_cur);
        c.max_tiles = 0xFFFFFFFFu;  // no tile storage is touched by this pass
        for (uint32_t k : {K_CLEAR_TABLE, K_BIN_INSERT, K_COMPACT_A, K_COMPACT_B, K_COMPACT_C}) {
            cudaError_t e = launch_e(h->tile_edge, k, c, h->stream, h->n_sms, 0, 0, nullptr);
            if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "sizing pass: %s", cudaGetErrorString(e));
        }
        Counters ct;
        int r = read_counters(h, &ct);
        if (r) return r;
        const bool over = (ct.status & ST_HASH_FULL) != 0u;
        if (h->auto_cap && (over || ct.n_st * 4u > h->cap)) {
            uint32_t want = next_pow2(std::max(ct.n_st * 8u, h->cap * 4u));
            uint32_t z = 0;
            CK(h, cudaMemcpy(&h->counters->status, &z, 4, cudaMemcpyHostToDevice));
            r = alloc_table(h, want);
            if (r) return r;
            continue;
        }
        *n_st = ct.n_st;
        *full = over;
        return MPM_OK;
    }
    return fail(h, MPM_ERR_CAPACITY, "tile hash table could not be sized");
}

// Tile edge of a handle created with tile_edge 0, chosen at the first step
// and again at the first step after the particle count changed, from binning
// passes of the current particles at edges 16, 12 and 8.  An edge qualifies
// when its occupied tiles number at least two per SM (every SM has work and
// the dynamic tile claiming can balance it).  Among the qualifying edges the
// one whose tiles hold the fewest halo cells, (E+2)^3 per tile, is taken (the
// per-particle work is the same at every edge; the halo assembly, conversion
// and flush grow with the halo cells), a smaller edge only when it has under
// 9/10 of the larger one's; when no edge qualifies, the edge with the most
// tiles.  Edge 14 is not a candidate (its 16^3 halo buffer makes it slower
// than both 12 and 16), nor is an edge whose tiles overflow a fixed hash
// capacity or a fixed max_tiles.  Results do not depend on the edge.
static int choose_tile_edge(MpmHandle* h) {
    const uint32_t edges[3] = {16u, 12u, 8u};
    uint32_t n_st[3] = {0u, 0u, 0u}, cap_at[3] = {0u, 0u, 0u};
    bool usable[3] = {false, false, false};
    for (int i = 0; i < 3; i++) {
        int r = set_tile_edge(h, edges[i]);
        if (r) return r;
        bool full = false;
        r = binning_pass(h, &n_st[i], &full);
        if (r) return r;
        cap_at[i] = h->cap;
        usable[i] = !full && (h->auto_tiles || n_st[i] <= h->max_tiles);
        if (full) {
            // a fresh table and a clear status for the next candidate
            uint32_t z = 0;
            CK(h, cudaMemcpy(&h->counters->status, &z, 4, cudaMemcpyHostToDevice));
            r = alloc_table(h, h->cap);
            if (r) return r;
        }
    }
    const uint32_t enough = 2u * (uint32_t)std::max(h->n_sms, 1);
    auto halo_cells = [&](int i) {
        const uint64_t hh = edges[i] + 2u;
        return (uint64_t)n_st[i] * hh * hh * hh;
    };
    int pick = -1;
    for (int i = 0; i < 3; i++)
        if (usable[i] && n_st[i] >= enough && (pick < 0 || 10u * halo_cells(i) < 9u * halo_cells(pick))) pick = i;
    if (pick < 0)
        for (int i = 0; i < 3; i++)
            if (usable[i] && (pick < 0 || n_st[i] > n_st[pick])) pick = i;
    if (pick < 0) pick = 0;  // nothing fits: edge 16, whose sizing pass reports why
    int r = set_tile_edge(h, edges[pick]);
    if (r) return r;
    // a table grown for a smaller edge's tiles is brought back to its size
    if (h->auto_cap && h->cap > cap_at[pick]) {
        r = alloc_table(h, cap_at[pick]);
        if (r) return r;
    }
    h->edge_auto = false;
    destroy_graphs(h);
    return MPM_OK;
}

// Sizes the automatic capacities (and, for tile_edge 0, picks the tile edge)
// from binning passes over the current particles: the hash table to at least
// four slots per occupied tile, the tile buffers to 1.5x the occupied tiles.
static int size_from_binning(MpmHandle* h) {
    if (h->edge_auto) {
        int r = choose_tile_edge(h);
        if (r) return r;
    }
    uint32_t n_st = 0;
    bool full = false;
    int r = binning_pass(h, &n_st, &full);
    if (r) return r;
    if (full) return fail(h, MPM_ERR_CAPACITY, "tile hash table (%u slots) is full", h->cap);
    // At tile edge 8 with fewer than two occupied tiles per SM a launch lasts
    // about as long as its heaviest tile: the tile kernels then run 512-thread
    // CTAs (one per SM), which finish a tile's particles in half the rounds.
    h->iter_wide = h->tile_edge == 8u && n_st < 2u * (uint32_t)std::max(h->n_sms, 1);
    const size_t nc = (size_t)(h->tile_edge + 2) * (h->tile_edge + 2) * (h->tile_edge + 2);
    if (h->tiles[0] != nullptr && h->tiles_nc < nc) {
        // picked a larger edge than the buffers were sized for: the same tile
        // count at the larger halo size
        if (!h->auto_tiles && h->max_tiles < n_st)
            return fail(h, MPM_ERR_CAPACITY, "%u occupied tiles > max_tiles %u", n_st, h->max_tiles);
        r = alloc_tiles(h, h->auto_tiles ? tiles_for(n_st) : h->max_tiles);
        if (r) return r;
    }
    if (h->auto_tiles && (h->tiles[0] == nullptr || n_st > h->max_tiles)) {
        r = alloc_tiles(h, tiles_for(n_st));
        if (r) return r;
    }
    return MPM_OK;
}

static int prepare_step(MpmHandle* h) {
    if (h->n_particles == 0) return fail(h, MPM_ERR_STATE, "no particles");
    cudaSetDevice(h->device);
    int r = upload_scenes(h);
    if (r) return r;
    if (!h->work_valid) {
        // the caller's records become the work state, slot t = particle t
        k_work_load<<<work_grid(h->n_particles), 256, 0, h->stream>>>(h->particles, h->n_particles,
                                                                      h->work[h->work_cur], h->ids[h->work_cur]);
        CK(h, cudaGetLastError());
        h->work_valid = true;
        h->records_stale = false;
    }
    if (h->tiles[0] == nullptr || h->edge_auto || h->sizing_due) {
        r = size_from_binning(h);
        if (r) return r;
        h->sizing_due = false;
    }
    return MPM_OK;
}

static uint64_t graph_signature(MpmHandle* h) {
    uint64_t s = h->n_particles;
    s = s * 1315423911ull + h->n_scenes;
    s = s * 1315423911ull + h->scenes[0].params.n_iter;
    s = s * 1315423911ull + (uint64_t)(uintptr_t)h->work[0];
    s = s * 1315423911ull + (uint64_t)h->plast_mode;
    s = s * 1315423911ull + (uint64_t)(uintptr_t)(h->mlp ? h->mlp->params : nullptr);
    s = s * 1315423911ull + (uint64_t)(uintptr_t)h->pair_x + h->pair_cap;
    s = s * 1315423911ull + (uint64_t)h->audit_threshold + (uint64_t)__builtin_bit_cast(uint32_t, h->unc_threshold) +
        ((uint64_t)__builtin_bit_cast(uint32_t, h->det_threshold) << 32);
    s = s * 1315423911ull + (uint64_t)(uintptr_t)h->plast_list;
    s = s * 1315423911ull + (uint64_t)h->order_mode * 1024u + h->tile_block + (h->svd_any ? 7u : 0u);
    s = s * 1315423911ull + h->tile_edge * 2u + (h->iter_wide ? 1u : 0u);
    return s | 1ull;
}

static int run_substep(MpmHandle* h, int method) {
    int par = h->work_cur;
    if (h->use_graphs && !h->timing) {
        uint64_t sig = graph_signature(h);
        if (!h->graph[method][par] || h->graph_sig[method][par] != sig) {
            if (h->graph[method][par]) cudaGraphExecDestroy(h->graph[method][par]);
            h->graph[method][par] = nullptr;
            cudaGraph_t g;
            CK(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t e = enqueue_substep(h, method, par, true, false);
            cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
            if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "capture: %s", cudaGetErrorString(e));
            if (e2 != cudaSuccess) return fail(h, MPM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
            cudaError_t e3 = cudaGraphInstantiate(&h->graph[method][par], g, 0);
            cudaGraphDestroy(g);
            if (e3 != cudaSuccess) return fail(h, MPM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e3));
            h->graph_sig[method][par] = sig;
        }
        CK(h, cudaGraphLaunch(h->graph[method][par], h->stream));
        // the captured sequence leaves its last P2G result in the same buffer
        uint32_t ni = h->scenes[0].params.n_iter;
        h->last_tiles = (method == MPM_METHOD_EXPLICIT || ni <= 1) ? 0 : (((ni - 1) & 1u) ? 1 : 2);
    } else {
        cudaError_t e = enqueue_substep(h, method, par, false, false);
        if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    }
    h->work_cur ^= 1;
    h->records_stale = true;
    return MPM_OK;
}

extern "C" int mpm_step(MpmHandle* h, int method, uint32_t n_substeps) {
    if (!h) return MPM_ERR_ARG;
    if (method != MPM_METHOD_EXPLICIT && method != MPM_METHOD_PBMPM) return fail(h, MPM_ERR_ARG, "bad method %d", method);
    int r = prepare_step(h);
    if (r) return r;
    for (uint32_t i = 0; i < n_substeps; i++) {
        r = run_substep(h, method);
        if (r) return r;
    }
    // a caller-bound buffer is the caller's view of the state: bring it up to
    // date after every call (library-owned records are brought up to date
    // when read)
    if (!h->own_particles) return flush_records(h);
    return MPM_OK;
}

extern "C" int mpm_add_explicit_mpm_dispatches(MpmHandle* h, uint32_t n_particles) {
    if (!h) return MPM_ERR_ARG;
    if (n_particles != h->n_particles) return fail(h, MPM_ERR_ARG, "nParticles %u != bound %u", n_particles, h->n_particles);
    return mpm_step(h, MPM_METHOD_EXPLICIT, 1);
}

extern "C" int mpm_add_pbmpm_dispatches(MpmHandle* h, uint32_t n_particles) {
    if (!h) return MPM_ERR_ARG;
    if (n_particles != h->n_particles) return fail(h, MPM_ERR_ARG, "nParticles %u != bound %u", n_particles, h->n_particles);
    return mpm_step(h, MPM_METHOD_PBMPM, 1);
}

extern "C" int mpm_step_p2g_only(MpmHandle* h, int method) {
    if (!h) return MPM_ERR_ARG;
    if (method != MPM_METHOD_EXPLICIT && method != MPM_METHOD_PBMPM) return fail(h, MPM_ERR_ARG, "bad method %d", method);
    int r = prepare_step(h);
    if (r) return r;
    // the first transfer only: the grid is formed, the particle state is not advanced
    cudaError_t e = enqueue_substep(h, method, h->work_cur, false, true);
    if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    return MPM_OK;
}

extern "C" int mpm_sync(MpmHandle* h, uint32_t* status_out) {
    if (!h) return MPM_ERR_ARG;
    cudaSetDevice(h->device);
    Counters ct;
    int r = read_counters(h, &ct);
    if (r) return r;
    if (status_out) *status_out = ct.status;
    // grow automatic capacities for the following substeps (stream is idle)
    if (h->auto_tiles && h->tiles[0] && ct.n_st > h->max_tiles - h->max_tiles / 5u) {
        r = alloc_tiles(h, tiles_for(ct.n_st));
        if (r) return r;
    }
    if (h->auto_cap && ct.n_st * 4u > h->cap) {
        r = alloc_table(h, next_pow2(ct.n_st * 8u));
        if (r) return r;
    }
    // the CTA width of the tile kernels follows the occupied tiles (with a
    // margin, so a count near the limit does not switch it at every sync)
    if (h->tile_edge == 8u && h->tiles[0]) {
        const uint32_t s = (uint32_t)std::max(h->n_sms, 1);
        const bool wide = h->iter_wide ? ct.n_st < 3u * s : ct.n_st < 2u * s;
        if (wide != h->iter_wide) {
            h->iter_wide = wide;
            destroy_graphs(h);
        }
    }
    if (ct.status) return fail(h, MPM_ERR_DEVICE_STATUS, "device status 0x%x", ct.status);
    return MPM_OK;
}

extern "C" int mpm_selftest(int device, uint64_t n, uint64_t seed, uint64_t* ident_mismatches, uint64_t* cvt_mismatches,
                            uint64_t* nan_conversion) {
    if (cudaSetDevice(device) != cudaSuccess) return MPM_ERR_CUDA;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, 24) != cudaSuccess) return MPM_ERR_CUDA;
    unsigned long long hcnt[3] = {0, 0, 0};
    cudaError_t e = cudaMemset(d, 0, 24);
    if (e == cudaSuccess) e = launch_selftest(n, seed, d, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(hcnt, d, 24, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return MPM_ERR_CUDA;
    if (ident_mismatches) *ident_mismatches = hcnt[0];
    if (cvt_mismatches) *cvt_mismatches = hcnt[1];
    if (nan_conversion) *nan_conversion = hcnt[2];
    return MPM_OK;
}

extern "C" int mpm_clear_status(MpmHandle* h) {
    if (!h) return MPM_ERR_ARG;
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    uint32_t z = 0;
    CK(h, cudaMemcpy(&h->counters->status, &z, 4, cudaMemcpyHostToDevice));
    return MPM_OK;
}

extern "C" int mpm_get_counts(MpmHandle* h, uint32_t* n_tiles, uint32_t* n_binned) {
    if (!h) return MPM_ERR_ARG;
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    Counters ct;
    CK(h, cudaMemcpy(&ct, h->counters, sizeof(ct), cudaMemcpyDeviceToHost));
    if (n_tiles) *n_tiles = ct.n_st;
    if (n_binned) *n_binned = ct.n_binned;
    return MPM_OK;
}

extern "C" int mpm_get_tile_edge(MpmHandle* h, uint32_t* edge) {
    if (!h || !edge) return MPM_ERR_ARG;
    *edge = h->tile_edge;
    return MPM_OK;
}

extern "C" int mpm_get_grid_dense(MpmHandle* h, uint32_t scene, int apply_grid_update, int32_t* out_host, size_t n_cells) {
    int r = check_scene(h, scene);
    if (r) return r;
    if (scene >= h->n_scenes) return fail(h, MPM_ERR_ARG, "scene %u >= scene count", scene);
    const SceneDev& d = h->scenes[scene].dev;
    size_t need = (size_t)d.res[0] * d.res[1] * d.res[2];
    if (!out_host || n_cells < need) return fail(h, MPM_ERR_ARG, "grid buffer needs %zu cells", need);
    cudaSetDevice(h->device);
    int4* dout = nullptr;
    CK(h, cudaMalloc(&dout, need * 16));
    CK(h, cudaMemsetAsync(dout, 0, need * 16, h->stream));
    Ctx c = make_ctx(h, h->work_cur);
    c.tiles_b = h->tiles[h->last_tiles];
    // the PBMPM iterations write momentum only: the mass sums are the first transfer's
    c.tiles_m = h->last_tiles != 0 ? h->tiles[0] : nullptr;
    int grid = std::max(1, h->n_sms * std::max(1, h->blocks_per_sm[K_GRID_DENSE]));
    cudaError_t e = launch_e(h->tile_edge, K_GRID_DENSE, c, h->stream, grid, scene, apply_grid_update, dout);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, dout, need * 16, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "grid readback: %s", cudaGetErrorString(e));
    return MPM_OK;
}

// Particle splats for the renderers (calculateGridMass.wgsl, mcDensity.cs.wgsl):
// enqueued on the handle's stream into the caller's device buffer.
static int splat(MpmHandle* h, uint32_t scene, int kind, const uint32_t* res, uint32_t* out_dev, int accumulate) {
    int r = check_scene(h, scene);
    if (r) return r;
    if (scene >= h->n_scenes) return fail(h, MPM_ERR_ARG, "scene %u >= scene count", scene);
    if (!out_dev) return fail(h, MPM_ERR_ARG, "null output buffer");
    cudaSetDevice(h->device);
    r = upload_scenes(h);
    if (r) return r;
    r = flush_records(h);
    if (r) return r;
    const SceneDev& d = h->scenes[scene].dev;
    SplatArgs a{};
    a.particles = h->particles;
    a.first = d.p_first;
    a.count = d.p_count;
    for (int k = 0; k < 3; k++) {
        a.gmin[k] = d.gmin[k];
        a.gmax[k] = d.gmax[k];
        a.res[k] = res ? res[k] : (uint32_t)d.res[k];
        if (a.res[k] == 0) return fail(h, MPM_ERR_ARG, "splat resolution must be > 0");
    }
    a.scale = d.scale;
    a.out = out_dev;
    if (!accumulate)
        CK(h, cudaMemsetAsync(out_dev, 0, (size_t)a.res[0] * a.res[1] * a.res[2] * 4, h->stream));
    CK(h, launch_splat(kind, a, h->stream));
    return MPM_OK;
}

extern "C" int mpm_grid_mass(MpmHandle* h, uint32_t scene, uint32_t* out_dev, int accumulate) {
    if (!h) return MPM_ERR_ARG;
    return splat(h, scene, 0, nullptr, out_dev, accumulate);
}

extern "C" int mpm_mc_density(MpmHandle* h, uint32_t scene, const uint32_t* density_res, uint32_t* out_dev,
                              int accumulate) {
    if (!h || !density_res) return MPM_ERR_ARG;
    return splat(h, scene, 1, density_res, out_dev, accumulate);
}

// Volumetric ray march (volumetricRaymarch.cs.wgsl): camera and time from the
// scene's uniform block (viewProjInvMat @112, time @12), grid bounds,
// resolution and fixed-point scale from its parameters.
extern "C" int mpm_volumetric_raymarch(MpmHandle* h, uint32_t scene, const uint32_t* mass_grid_dev, uint32_t width,
                                       uint32_t height, uint8_t* rgba_dev, float* depth_dev, float* color_dev) {
    if (!h) return MPM_ERR_ARG;
    int r = check_scene(h, scene);
    if (r) return r;
    if (scene >= h->n_scenes) return fail(h, MPM_ERR_ARG, "scene %u >= scene count", scene);
    if (!mass_grid_dev || !rgba_dev || !depth_dev) return fail(h, MPM_ERR_ARG, "null buffer");
    if (width == 0 || height == 0 || width > 16384 || height > 16384)
        return fail(h, MPM_ERR_ARG, "image size %ux%u outside 1..16384", width, height);
    cudaSetDevice(h->device);
    r = upload_scenes(h);
    if (r) return r;
    const SceneDev& d = h->scenes[scene].dev;
    const uint8_t* u = h->scenes[scene].uni;
    RaymarchArgs a{};
    a.mass = mass_grid_dev;
    for (int k = 0; k < 3; k++) {
        a.res[k] = (uint32_t)d.res[k];
        a.gmin[k] = d.gmin[k];
        a.gmax[k] = d.gmax[k];
    }
    a.scale = d.scale;
    for (int k = 0; k < 16; k++) a.inv_vp[k] = rdf(u, 112 + 4 * k);
    a.time = rdu(u, 12);
    a.width = width;
    a.height = height;
    a.rgba = rgba_dev;
    a.depth = depth_dev;
    a.color = color_dev;
    CK(h, launch_raymarch(a, h->stream));
    return MPM_OK;
}

// Marching cubes (mcListBlocks, mcVertexDensity, mcGenerate) over a density
// grid of the mcDensity splat; grid bounds and fixed-point scale of the scene.
extern "C" int mpm_marching_cubes(MpmHandle* h, uint32_t scene, const uint32_t* density_dev,
                                  const uint32_t* density_res, const uint32_t* mc_res, float* vertices_dev,
                                  uint32_t max_vertices, uint32_t* vertex_count_out, uint32_t* vertices_generated_out) {
    if (!h) return MPM_ERR_ARG;
    int r = check_scene(h, scene);
    if (r) return r;
    if (scene >= h->n_scenes) return fail(h, MPM_ERR_ARG, "scene %u >= scene count", scene);
    if (!density_dev || !density_res || !mc_res || !vertex_count_out || (max_vertices && !vertices_dev))
        return fail(h, MPM_ERR_ARG, "null argument");
    for (int k = 0; k < 3; k++)
        if (density_res[k] == 0 || mc_res[k] == 0 || mc_res[k] > 4096 || density_res[k] > 4096)
            return fail(h, MPM_ERR_ARG, "grid resolutions must be in 1..4096");
    cudaSetDevice(h->device);
    r = upload_scenes(h);
    if (r) return r;
    const SceneDev& d = h->scenes[scene].dev;
    uint32_t total = 0;
    cudaError_t ce = cudaSuccess;
    if (mc_run(density_dev, density_res, mc_res, d.gmin, d.gmax, d.scale, vertices_dev, max_vertices, &total, h->n_sms,
               h->stream, &ce))
        return fail(h, MPM_ERR_CUDA, "marching cubes: %s", cudaGetErrorString(ce));
    *vertex_count_out = total < max_vertices ? total : max_vertices;   // mcClampArgs
    if (vertices_generated_out) *vertices_generated_out = total;
    return MPM_OK;
}

extern "C" int mpm_scatter_particles(MpmHandle* h, const float* vertices, uint32_t n_vertices, uint32_t n_particles) {
    if (!h) return MPM_ERR_ARG;
    if (!vertices || n_vertices < 3 || n_vertices % 3 != 0)
        return fail(h, MPM_ERR_ARG, "vertices must be a triangle soup of 3k vertices");
    if (n_particles > h->cfg.max_particles)
        return fail(h, MPM_ERR_CAPACITY, "%u particles exceed max_particles %u", n_particles, h->cfg.max_particles);
    if (!h->own_particles) return fail(h, MPM_ERR_STATE, "particle buffer is bound to caller memory");
    cudaSetDevice(h->device);
    int r = set_count(h, n_particles);
    if (r) return r;
    ScatterArgs a{};
    a.particles = h->particles;
    a.n = n_particles;
    a.n_tris = n_vertices / 3;
    const uint8_t* u = h->scenes[0].uni;   // uniforms.meshMinCoords @176, meshMaxCoords @192
    for (int k = 0; k < 3; k++) {
        a.mmin[k] = rdf(u, 176 + 4 * k);
        a.mmax[k] = rdf(u, 192 + 4 * k);
    }
    float4* dv = nullptr;
    CK(h, cudaMalloc(&dv, (size_t)n_vertices * 16));
    a.verts = dv;
    cudaError_t e = cudaMemcpyAsync(dv, vertices, (size_t)n_vertices * 16, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_scatter(a, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(dv);
    if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, "scatter: %s", cudaGetErrorString(e));
    h->work_valid = false;
    h->records_stale = false;
    return MPM_OK;
}

extern "C" int mpm_set_schedule(MpmHandle* h, uint32_t order_mode, uint32_t tile_block) {
    if (!h) return MPM_ERR_ARG;
    if (order_mode != 0u && order_mode != 1u && order_mode != 4u && order_mode != 5u)
        return fail(h, MPM_ERR_ARG, "order_mode must be 0, 1, 4 or 5");
    if (tile_block != 0u && tile_block != 128u && tile_block != 256u)
        return fail(h, MPM_ERR_ARG, "tile_block must be 0, 128 or 256");
    h->order_mode = order_mode;
    h->tile_block = tile_block;
    destroy_graphs(h);
    return MPM_OK;
}

extern "C" int mpm_enable_kernel_timing(MpmHandle* h, int enable) {
    if (!h) return MPM_ERR_ARG;
    drain_timing(h);
    h->timing = enable != 0;
    for (int k = 0; k < K_COUNT; k++) { h->kms[k] = 0; h->kcount[k] = 0; }
    return MPM_OK;
}

extern "C" int mpm_kernel_times(MpmHandle* h, float* ms_out, uint32_t* launches_out, uint32_t n_kernels) {
    if (!h) return MPM_ERR_ARG;
    drain_timing(h);
    for (uint32_t k = 0; k < n_kernels && k < (uint32_t)K_COUNT; k++) {
        if (ms_out) ms_out[k] = (float)h->kms[k];
        if (launches_out) launches_out[k] = h->kcount[k];
    }
    return MPM_OK;
}

extern "C" const char* mpm_kernel_name(uint32_t kernel_id) {
    return kernel_id < (uint32_t)K_COUNT ? kKernelNames[kernel_id] : "unknown";
}

extern "C" uint32_t mpm_kernel_count(void) { return (uint32_t)K_COUNT; }

extern "C" int mpm_use_graphs(MpmHandle* h, int enable) {
    if (!h) return MPM_ERR_ARG;
    h->use_graphs = enable != 0;
    if (!h->use_graphs) destroy_graphs(h);
    return MPM_OK;
}

// ---------------------------------------------------------------------
// Learned plasticity: the network object, its training, and its use by a handle
// ---------------------------------------------------------------------
static int mlp_fail(MpmMlp* m, int code, const char* fmt, ...) {
    if (m) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        m->msg = buf;
    }
    return code;
}
#define MCK(m, expr)                                                                              \
    do {                                                                                          \
        cudaError_t _e = (expr);                                                                  \
        if (_e != cudaSuccess) return mlp_fail((m), MPM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Glorot-uniform weights, zero biases; the last layer starts at a tenth of that
extern "C" int mpm_mlp_init_params(uint32_t seed, float* out) {
    if (!out) return MPM_ERR_ARG;
    uint64_t st = 0x6d6c70ull ^ ((uint64_t)seed << 20);
    std::memset(out, 0, sizeof(float) * mlp::NPARAM);
    struct L { int ow, out, in; float gain; } layers[4] = {{mlp::OW1, mlp::HID, mlp::IN, 1.f},
                                                          {mlp::OW2, mlp::HID, mlp::HID, 1.f},
                                                          {mlp::OW3, mlp::HID, mlp::HID, 1.f},
                                                          {mlp::OW4, mlp::OUT, mlp::HID, 0.1f}};
    for (auto& l : layers) {
        float a = l.gain * std::sqrt(6.0f / (float)(l.in + l.out));
        for (int i = 0; i < l.out * l.in; i++) {
            double u = (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0);
            out[l.ow + i] = (float)((2.0 * u - 1.0) * a);
        }
    }
    return MPM_OK;
}

extern "C" int mpm_mlp_create(int device, uint32_t seed, MpmMlp** out) {
    if (!out) return MPM_ERR_ARG;
    MpmMlp* m = new MpmMlp();
    *out = m;
    m->device = device;
    MCK(m, cudaSetDevice(device));
    MCK(m, cudaDeviceGetAttribute(&m->n_sms, cudaDevAttrMultiProcessorCount, device));
    MCK(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    MCK(m, cudaMalloc(&m->params, mlp::NPARAM * 4));
    MCK(m, cudaMalloc(&m->adam_m, mlp::NPARAM * 4));
    MCK(m, cudaMalloc(&m->adam_v, mlp::NPARAM * 4));
    MCK(m, cudaMalloc(&m->grad, mlp::NPARAM * 4));
    MCK(m, cudaMalloc(&m->loss, 8));
    MCK(m, cudaMalloc(&m->err, 4));
    MCK(m, cudaMemset(m->adam_m, 0, mlp::NPARAM * 4));
    MCK(m, cudaMemset(m->adam_v, 0, mlp::NPARAM * 4));
    MCK(m, cudaMemset(m->err, 0, 4));
    MCK(m, configure_mlp_kernels());
    std::vector<float> p(mlp::NPARAM);
    mpm_mlp_init_params(seed, p.data());
    MCK(m, cudaMemcpy(m->params, p.data(), mlp::NPARAM * 4, cudaMemcpyHostToDevice));
    return MPM_OK;
}

extern "C" int mpm_mlp_destroy(MpmMlp* m) {
    if (!m) return MPM_ERR_ARG;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    void* bufs[] = {m->params, m->adam_m, m->adam_v, m->grad, m->loss, m->err, m->idx};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (m->stream && m->own_stream) cudaStreamDestroy(m->stream);
    delete m;
    return MPM_OK;
}

extern "C" const char* mpm_mlp_last_error(const MpmMlp* m) { return m ? m->msg.c_str() : "null network"; }

extern "C" int mpm_mlp_set_stream(MpmMlp* m, void* stream) {
    if (!m) return MPM_ERR_ARG;
    cudaSetDevice(m->device);
    MCK(m, cudaStreamSynchronize(m->stream));
    if (m->own_stream) cudaStreamDestroy(m->stream);
    if (stream) {
        m->stream = (cudaStream_t)stream;
        m->own_stream = false;
    } else {
        MCK(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
        m->own_stream = true;
    }
    return MPM_OK;
}

extern "C" int mpm_mlp_get_params(MpmMlp* m, float* host_out) {
    if (!m || !host_out) return MPM_ERR_ARG;
    cudaSetDevice(m->device);
    MCK(m, cudaStreamSynchronize(m->stream));
    MCK(m, cudaMemcpy(host_out, m->params, mlp::NPARAM * 4, cudaMemcpyDeviceToHost));
    return MPM_OK;
}

extern "C" int mpm_mlp_set_params(MpmMlp* m, const float* host_in) {
    if (!m || !host_in) return MPM_ERR_ARG;
    cudaSetDevice(m->device);
    MCK(m, cudaStreamSynchronize(m->stream));
    MCK(m, cudaMemcpy(m->params, host_in, mlp::NPARAM * 4, cudaMemcpyHostToDevice));
    MCK(m, cudaMemset(m->adam_m, 0, mlp::NPARAM * 4));
    MCK(m, cudaMemset(m->adam_v, 0, mlp::NPARAM * 4));
    m->adam_step = 0;
    return MPM_OK;
}

static int mlp_check_err(MpmMlp* m) {
    uint32_t e = 0;
    MCK(m, cudaMemcpy(&e, m->err, 4, cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(m->err, 0, 4);
        return mlp_fail(m, MPM_ERR_DEVICE_STATUS, "tensor-core wait ran out (device status 0x%x)", e);
    }
    return MPM_OK;
}

extern "C" int mpm_mlp_forward(MpmMlp* m, const float* x_dev, uint32_t n, float* y_dev) {
    if (!m || (n && (!x_dev || !y_dev))) return MPM_ERR_ARG;
    if (n == 0) return MPM_OK;
    cudaSetDevice(m->device);
    int grid = (int)std::min<uint32_t>((n + 127u) / 128u, (uint32_t)m->n_sms * MLP_CTAS_PER_SM);
    MCK(m, launch_mlp_forward(m->params, x_dev, n, y_dev, m->err, grid, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    return mlp_check_err(m);
}

extern "C" int mpm_mlp_gradient(MpmMlp* m, const float* x_dev, const float* t_dev, uint32_t n, float unc_weight,
                                float* grad_host, float* loss_host) {
    if (!m || n == 0 || !x_dev || !t_dev) return MPM_ERR_ARG;
    cudaSetDevice(m->device);
    MCK(m, cudaMemsetAsync(m->grad, 0, mlp::NPARAM * 4, m->stream));
    MCK(m, cudaMemsetAsync(m->loss, 0, 8, m->stream));
    int grid = (int)std::min<uint32_t>((n + 127u) / 128u, (uint32_t)m->n_sms);
    MCK(m, launch_mlp_train(m->params, x_dev, t_dev, nullptr, n, 1.0f / (float)n, unc_weight, m->grad, m->loss,
                            m->err, grid, m->stream));
    MCK(m, cudaStreamSynchronize(m->stream));
    int r = mlp_check_err(m);
    if (r) return r;
    if (grad_host) MCK(m, cudaMemcpy(grad_host, m->grad, mlp::NPARAM * 4, cudaMemcpyDeviceToHost));
    if (loss_host) MCK(m, cudaMemcpy(loss_host, m->loss, 4, cudaMemcpyDeviceToHost));
    return MPM_OK;
}

extern "C" int mpm_mlp_train(MpmMlp* m, const float* x_dev, const float* t_dev, uint32_t n,
                             const MpmMlpTrainConfig* cfg, float* loss_per_epoch) {
    if (!m || !cfg || n == 0 || !x_dev || !t_dev) return MPM_ERR_ARG;
    if (cfg->batch == 0 || cfg->epochs == 0) return mlp_fail(m, MPM_ERR_ARG, "batch and epochs must be > 0");
    cudaSetDevice(m->device);
    if (m->idx_cap < n) {
        if (m->idx) cudaFree(m->idx);
        m->idx = nullptr;
        MCK(m, cudaMalloc(&m->idx, (size_t)n * 4));
        m->idx_cap = n;
    }
    std::vector<uint32_t> perm(n);
    uint64_t st = 0x747261696eull ^ cfg->seed;
    const uint32_t n_batches = (n + cfg->batch - 1) / cfg->batch;
    const uint32_t total = n_batches * cfg->epochs;
    uint32_t step = 0;
    for (uint32_t ep = 0; ep < cfg->epochs; ep++) {
        for (uint32_t i = 0; i < n; i++) perm[i] = i;
        for (uint32_t i = n - 1; i > 0; i--) {
            uint32_t j = (uint32_t)(splitmix(st) % (uint64_t)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        MCK(m, cudaMemcpyAsync(m->idx, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
        MCK(m, cudaMemsetAsync(m->loss, 0, 8, m->stream));
        for (uint32_t b = 0; b < n_batches; b++) {
            uint32_t b0 = b * cfg->batch, nb = std::min(cfg->batch, n - b0);
            MCK(m, cudaMemsetAsync(m->grad, 0, mlp::NPARAM * 4, m->stream));
            int grid = (int)std::min<uint32_t>((nb + 127u) / 128u, (uint32_t)m->n_sms);
            MCK(m, launch_mlp_train(m->params, x_dev, t_dev, m->idx + b0, nb, 1.0f / (float)nb, cfg->unc_weight,
                                    m->grad, m->loss, m->err, grid, m->stream));
            // cosine decay from lr to lr_final over all steps
            float f = 0.5f * (1.0f + std::cos(3.14159265f * (float)step / (float)std::max(1u, total - 1u)));
            float lr = cfg->lr_final + (cfg->lr - cfg->lr_final) * f;
            m->adam_step++;
            MCK(m, launch_adam(m->params, m->adam_m, m->adam_v, m->grad, mlp::NPARAM, lr, m->adam_step, m->stream));
            step++;
        }
        float lsum = 0.f;
        MCK(m, cudaMemcpyAsync(&lsum, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
        MCK(m, cudaStreamSynchronize(m->stream));
        int r = mlp_check_err(m);
        if (r) return r;
        if (loss_per_epoch) loss_per_epoch[ep] = lsum / (float)n_batches;
    }
    return MPM_OK;
}

extern "C" int mpm_set_plasticity(MpmHandle* h, int mode, MpmMlp* net, float unc_threshold, float det_threshold,
                                  float audit_fraction) {
    if (!h) return MPM_ERR_ARG;
    if (mode < MPM_PLASTICITY_INLINE || mode > MPM_PLASTICITY_LEARNED) return fail(h, MPM_ERR_ARG, "bad plasticity mode %d", mode);
    if (mode == MPM_PLASTICITY_LEARNED && !net) return fail(h, MPM_ERR_ARG, "learned plasticity needs a network");
    if (net && net->device != h->device) return fail(h, MPM_ERR_ARG, "network lives on device %d, handle on %d", net->device, h->device);
    if (!(audit_fraction >= 0.f && audit_fraction <= 1.f)) return fail(h, MPM_ERR_ARG, "audit fraction must be in [0, 1]");
    cudaSetDevice(h->device);
    if (mode != MPM_PLASTICITY_INLINE && !h->plast_list)
        CK(h, cudaMalloc(&h->plast_list, (size_t)h->cfg.max_particles * 4));
    h->plast_mode = mode;
    h->mlp = net;
    h->unc_threshold = unc_threshold;
    h->det_threshold = det_threshold;
    h->audit_threshold = (uint32_t)std::min(4294967295.0, (double)audit_fraction * 4294967296.0);
    return MPM_OK;
}

extern "C" int mpm_set_pair_buffer(MpmHandle* h, float* x_dev, float* t_dev, uint32_t capacity) {
    if (!h) return MPM_ERR_ARG;
    if (capacity && (!x_dev || !t_dev)) return fail(h, MPM_ERR_ARG, "null pair buffer");
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    h->pair_x = capacity ? x_dev : nullptr;
    h->pair_t = capacity ? t_dev : nullptr;
    h->pair_cap = capacity;
    CK(h, cudaMemset(h->d_pair_count, 0, 4));
    return MPM_OK;
}

extern "C" int mpm_get_plasticity_stats(MpmHandle* h, MpmPlasticityStats* out, int reset) {
    if (!h || !out) return MPM_ERR_ARG;
    cudaSetDevice(h->device);
    CK(h, cudaStreamSynchronize(h->stream));
    PlastStats ps;
    uint32_t pairs = 0;
    CK(h, cudaMemcpy(&ps, h->d_stats, sizeof(ps), cudaMemcpyDeviceToHost));
    CK(h, cudaMemcpy(&pairs, h->d_pair_count, 4, cudaMemcpyDeviceToHost));
    out->candidates = ps.candidates;
    out->learned = ps.learned;
    out->fallback_domain = ps.fallback_domain;
    out->fallback_uncertain = ps.fallback_uncertain;
    out->fallback_det = ps.fallback_det;
    out->audited = ps.audited;
    float mx;
    std::memcpy(&mx, &ps.audit_max_err_bits, 4);
    out->audit_max_err = mx;
    out->audit_mean_err = ps.audited ? (float)(ps.audit_err_sum / (double)ps.audited) : 0.f;
    out->pairs_collected = std::min(pairs, h->pair_cap);
    if (reset) CK(h, cudaMemset(h->d_stats, 0, sizeof(PlastStats)));
    return MPM_OK;
}

// ---------------------------------------------------------------------
// Allocation-free substep: every intermediate buffer lives in one
// file-scope device array, so a call allocates no device memory.
// ---------------------------------------------------------------------
namespace {

constexpr uint32_t NA_EDGE = 8u;
constexpr size_t NA_NC = (size_t)(NA_EDGE + 2) * (NA_EDGE + 2) * (NA_EDGE + 2);
static_assert(MPM_NOALLOC_HASH_SLOTS % COMPACT_CHUNK == 0, "hash slots must be whole compaction chunks");
static_assert((MPM_NOALLOC_HASH_SLOTS & (MPM_NOALLOC_HASH_SLOTS - 1u)) == 0, "hash slots must be a power of two");
static_assert(MPM_NOALLOC_TILE_EDGE == NA_EDGE, "header and engine disagree on the tile edge");

constexpr size_t na_round(size_t v) { return (v + 255u) & ~(size_t)255u; }
constexpr size_t NA_P = MPM_NOALLOC_MAX_PARTICLES, NA_H = MPM_NOALLOC_HASH_SLOTS;
constexpr size_t NA_WORK0 = 0;                                          // particle state in, planes
constexpr size_t NA_WORK1 = NA_WORK0 + na_round(NA_P * MPM_PARTICLE_BYTES);   // particle state out, tile order
constexpr size_t NA_IDS0 = NA_WORK1 + na_round(NA_P * MPM_PARTICLE_BYTES);    // caller index per slot
constexpr size_t NA_IDS1 = NA_IDS0 + na_round(NA_P * 4);
constexpr size_t NA_SORTED = NA_IDS1 + na_round(NA_P * 4);              // input slots grouped by tile
constexpr size_t NA_BIN_SLOT = NA_SORTED + na_round(NA_P * 4);
constexpr size_t NA_BIN_RANK = NA_BIN_SLOT + na_round(NA_P * 4);
constexpr size_t NA_KEYS = NA_BIN_RANK + na_round(NA_P * 4);            // tile hash keys (u64)
constexpr size_t NA_SLOT_COUNT = NA_KEYS + na_round(NA_H * 8);
constexpr size_t NA_SLOT_OFF = NA_SLOT_COUNT + na_round(NA_H * 4);
constexpr size_t NA_SLOT_ST = NA_SLOT_OFF + na_round(NA_H * 4);
constexpr size_t NA_ST_KEY = NA_SLOT_ST + na_round(NA_H * 4);
constexpr size_t NA_ST_SLOT = NA_ST_KEY + na_round(NA_H * 8);
constexpr size_t NA_ST_BEGIN = NA_ST_SLOT + na_round(NA_H * 4);
constexpr size_t NA_ST_COUNT = NA_ST_BEGIN + na_round(NA_H * 4);
constexpr size_t NA_CHUNK_NST = NA_ST_COUNT + na_round(NA_H * 4);
constexpr size_t NA_CHUNK_NP = NA_CHUNK_NST + na_round(NA_H / COMPACT_CHUNK * 4);
constexpr size_t NA_TILES0 = NA_CHUNK_NP + na_round(NA_H / COMPACT_CHUNK * 4);  // halo sums, int4
constexpr size_t NA_TILES1 = NA_TILES0 + na_round(MPM_NOALLOC_MAX_TILES * NA_NC * 16);
constexpr size_t NA_ITER_REC = NA_TILES1 + na_round(MPM_NOALLOC_MAX_TILES * NA_NC * 16);  // PBMPM records
constexpr size_t NA_ST_NBR = NA_ITER_REC + na_round(NA_P * IR_PLANES * 16);  // tile neighbour table
constexpr size_t NA_SCENE = NA_ST_NBR + na_round(MPM_NOALLOC_MAX_TILES * 27 * 4);
constexpr size_t NA_SCENE_FIRST = NA_SCENE + na_round(sizeof(SceneDev));
constexpr size_t NA_COUNTERS = NA_SCENE_FIRST + na_round(2 * 4);
constexpr size_t NA_BYTES = NA_COUNTERS + na_round(sizeof(Counters));
static_assert(NA_BYTES <= MPM_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the declared size");

constexpr int NA_MAX_DEVICES = 64;

struct NaDevice {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of the scratch array on this device
    int n_sms = 0;
    int blocks_per_sm[K_COUNT] = {0};
};

std::mutex g_na_mutex;
NaDevice g_na_dev[NA_MAX_DEVICES];

int na_fail(char* err, size_t err_len, int code, const char* fmt, ...) {
    if (err && err_len) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, err_len, fmt, ap);
        va_end(ap);
    }
    return code;
}

}  // namespace

// Writes the call's scene record and particle range into the scratch array.
__global__ void k_na_store_scene(SceneDev sc, uint32_t n_particles, SceneDev* scene, uint32_t* scene_first) {
    *scene = sc;
    scene_first[0] = 0u;
    scene_first[1] = n_particles;
}

// The scratch itself.  A host-side use of this name refers to a host stand-in,
// not to device memory: host code passes kernels the address returned by
// cudaGetSymbolAddress for the current device instead.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MPM_NOALLOC_SCRATCH_BYTES];

extern "C" int mpm_step_noalloc(int device, void* stream, void* particles, uint32_t n_particles, int method,
                                const void* uniforms, size_t uniform_bytes, const MpmParams* params,
                                const uint32_t* collider_data, size_t collider_words, uint32_t num_indices,
                                const void* bvh_nodes, uint32_t n_nodes, uint32_t* status_out, char* err,
                                size_t err_len) {
    if (err && err_len) err[0] = '\0';
    if (!particles || n_particles == 0) return na_fail(err, err_len, MPM_ERR_ARG, "no particle buffer");
    if (n_particles > MPM_NOALLOC_MAX_PARTICLES)
        return na_fail(err, err_len, MPM_ERR_CAPACITY, "%u particles exceed the allocation-free limit of %u",
                       n_particles, MPM_NOALLOC_MAX_PARTICLES);
    if (((uintptr_t)particles & 15u) != 0) return na_fail(err, err_len, MPM_ERR_ARG, "particle buffer must be 16-byte aligned");
    if (method != MPM_METHOD_EXPLICIT && method != MPM_METHOD_PBMPM)
        return na_fail(err, err_len, MPM_ERR_ARG, "bad method %d", method);
    if (!uniforms || uniform_bytes < 544)
        return na_fail(err, err_len, MPM_ERR_ARG, "uniform block needs >= 544 bytes, got %zu", uniform_bytes);
    if (!params || params->n_iter == 0) return na_fail(err, err_len, MPM_ERR_ARG, "params missing or n_iter == 0");
    if (params->return_map != 0u)
        return na_fail(err, err_len, MPM_ERR_ARG, "return_map %u needs a handle (deferred plasticity pass)",
                       params->return_map);
    if ((collider_words && !collider_data) || (n_nodes && !bvh_nodes))
        return na_fail(err, err_len, MPM_ERR_ARG, "null collider buffer");
    if ((size_t)num_indices > collider_words)
        return na_fail(err, err_len, MPM_ERR_ARG, "num_indices %u > collider words %zu", num_indices, collider_words);
    if (device < 0 || device >= NA_MAX_DEVICES) return na_fail(err, err_len, MPM_ERR_ARG, "device %d out of range", device);

    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return na_fail(err, err_len, MPM_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    struct Restore {
        int d;
        ~Restore() { if (d >= 0) cudaSetDevice(d); }
    } restore{prev};

    // once per device, with that device current: the scratch array's device
    // address and the tile kernels' launch configuration
    NaDevice& D = g_na_dev[device];
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!D.ready) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return na_fail(err, err_len, MPM_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            e = cudaDeviceGetAttribute(&D.n_sms, cudaDevAttrMultiProcessorCount, device);
            if (e != cudaSuccess) return na_fail(err, err_len, MPM_ERR_CUDA, "SM count: %s", cudaGetErrorString(e));
            e = configure_tile_kernels<NA_EDGE>(D.blocks_per_sm);
            if (e != cudaSuccess)
                return na_fail(err, err_len, MPM_ERR_CUDA, "configure kernels: %s", cudaGetErrorString(e));
            D.base = (unsigned char*)p;
            D.ready = true;
        }
    }

    // the scene record, built exactly as a handle builds it
    SceneHost sc;
    std::memset(sc.uni, 0, sizeof(sc.uni));
    std::memcpy(sc.uni, uniforms, std::min(uniform_bytes, (size_t)MPM_UNIFORMS_BYTES));
    if (collider_words) std::memcpy(sc.uni + 348, &num_indices, 4);  // GpuMpmPipelineManager.ts:80
    sc.params = *params;
    std::memset(&sc.dev, 0, sizeof(sc.dev));
    sc.dev.col_data = collider_words ? collider_data : nullptr;
    sc.dev.bvh = n_nodes ? (const uint32_t*)bvh_nodes : nullptr;
    sc.dev.col_words = (uint32_t)collider_words;
    sc.dev.n_nodes = n_nodes;
    sc.dev.c_nidx = num_indices;
    sc.dev.p_first = 0;
    sc.dev.p_count = n_particles;
    build_scene_dev(sc);
    if (sc.dev.scale <= 0.0f || !(sc.dev.dt > 0.0f))
        return na_fail(err, err_len, MPM_ERR_ARG, "fixedPointScale and timestep must be > 0");
    if (sc.dev.res[0] <= 0 || sc.dev.res[1] <= 0 || sc.dev.res[2] <= 0)
        return na_fail(err, err_len, MPM_ERR_ARG, "grid resolution must be > 0");

    unsigned char* b = D.base;
    Ctx c{};
    c.work_in = (const float4*)(b + NA_WORK0);
    c.work_out = (float4*)(b + NA_WORK1);
    c.ids_in = (const uint32_t*)(b + NA_IDS0);
    c.ids_out = (uint32_t*)(b + NA_IDS1);
    c.sorted = (uint32_t*)(b + NA_SORTED);
    c.bin_slot = (uint32_t*)(b + NA_BIN_SLOT);
    c.bin_rank = (uint32_t*)(b + NA_BIN_RANK);
    c.keys = (unsigned long long*)(b + NA_KEYS);
    c.slot_count = (uint32_t*)(b + NA_SLOT_COUNT);
    c.slot_off = (uint32_t*)(b + NA_SLOT_OFF);
    c.slot_st = (uint32_t*)(b + NA_SLOT_ST);
    c.st_key = (unsigned long long*)(b + NA_ST_KEY);
    c.st_slot = (uint32_t*)(b + NA_ST_SLOT);
    c.st_begin = (uint32_t*)(b + NA_ST_BEGIN);
    c.st_count = (uint32_t*)(b + NA_ST_COUNT);
    c.chunk_nst = (uint32_t*)(b + NA_CHUNK_NST);
    c.chunk_np = (uint32_t*)(b + NA_CHUNK_NP);
    int4* tiles[2] = {(int4*)(b + NA_TILES0), (int4*)(b + NA_TILES1)};
    c.tiles_a = tiles[0];
    c.tiles_b = tiles[0];
    c.iter_rec = (float4*)(b + NA_ITER_REC);
    c.st_nbr = (int32_t*)(b + NA_ST_NBR);
    c.scenes = (const SceneDev*)(b + NA_SCENE);
    c.scene_first = (const uint32_t*)(b + NA_SCENE_FIRST);
    c.counters = (Counters*)(b + NA_COUNTERS);
    c.n_particles = n_particles;
    c.n_scenes = 1;
    c.cap = MPM_NOALLOC_HASH_SLOTS;
    c.max_tiles = MPM_NOALLOC_MAX_TILES;

    cudaStream_t s = (cudaStream_t)stream;
#define NA_CK(expr)                                                                                  \
    do {                                                                                             \
        cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess) return na_fail(err, err_len, MPM_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
    } while (0)
    // The array keeps the previous call's contents: start from an empty tile
    // table, zero counters and status, and the identity particle order.
    NA_CK(cudaMemsetAsync(c.keys, 0xff, NA_H * 8, s));
    NA_CK(cudaMemsetAsync(c.slot_count, 0, NA_H * 4, s));
    NA_CK(cudaMemsetAsync(c.counters, 0, sizeof(Counters), s));
    // the scene record reaches the device as a kernel argument (copied at
    // launch), so no host buffer has to outlive the call and the host does
    // not wait for the stream here
    k_na_store_scene<<<1, 1, 0, s>>>(sc.dev, n_particles, (SceneDev*)c.scenes, (uint32_t*)c.scene_first);
    NA_CK(cudaGetLastError());
    // the caller's records become the input state (slot t = particle t)
    k_work_load<<<work_grid(n_particles), 256, 0, s>>>((const float4*)particles, n_particles, (float4*)c.work_in,
                                                       (uint32_t*)c.ids_in);
    NA_CK(cudaGetLastError());
    auto run = [&](uint32_t kid) {
        int grid = std::max(1, D.n_sms * std::max(1, D.blocks_per_sm[kid]));
        return launch_kernel<NA_EDGE>(kid, c, s, grid, 0, 0, nullptr);
    };
    for (uint32_t k : {K_BIN_INSERT, K_COMPACT_A, K_COMPACT_B, K_COMPACT_C, K_BIN_SCATTER, K_TILE_NBR}) NA_CK(run(k));
    if (method == MPM_METHOD_EXPLICIT) {
        NA_CK(run(K_P2G_EXPLICIT));
        NA_CK(run(K_G2P_EXPLICIT));
    } else {
        int cur = 0;
        c.tiles_a = tiles[cur];
        NA_CK(run(K_PBMPM_FIRST));
        for (uint32_t it = 1; it < params->n_iter; it++) {
            c.tiles_b = tiles[cur];
            c.tiles_a = tiles[cur ^ 1];
            c.iter_first = it == 1 ? 1u : 0u;
            NA_CK(run(K_PBMPM_ITER));
            cur ^= 1;
        }
        c.tiles_b = tiles[cur];
        c.g2p_rm = params->n_iter > 1 ? 1u : 0u;
        NA_CK(run(K_G2P_PBMPM));
    }
    // the advanced state back into the caller's records
    k_work_store<<<work_grid(n_particles), 256, 0, s>>>(c.work_out, c.ids_out, n_particles, (float4*)particles);
    NA_CK(cudaGetLastError());
    if (status_out) {
        Counters ct;
        NA_CK(cudaMemcpyAsync(&ct, c.counters, sizeof(ct), cudaMemcpyDeviceToHost, s));
        NA_CK(cudaStreamSynchronize(s));
        *status_out = ct.status;
        if (ct.status)
            return na_fail(err, err_len, MPM_ERR_DEVICE_STATUS,
                           "device status 0x%x (0x2: more than %u occupied tiles; 0x1: tile hash full)", ct.status,
                           MPM_NOALLOC_MAX_TILES);
    }
#undef NA_CK
    return MPM_OK;
}
