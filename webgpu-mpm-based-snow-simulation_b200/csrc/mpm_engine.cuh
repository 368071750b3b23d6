// mpm_engine.cuh -- device-side data layout of the MPM step.
//
// HBM layout (all buffers allocated once by mpm_create):
//   particles   N x 192 B  reference ParticleData records in the caller's order
//                          (the boundary: loaded into, and stored back from, work)
//   work[2]     REC_PLANES x N float4   the particle state the substeps advance,
//                          plane by plane (word q of the 192-byte record of slot t
//                          at work[q * N + t]), slots in the previous substep's tile
//                          order; each substep reads one and writes the other
//   ids[2]      N x u32    caller index of each work slot
//   bin_slot    N x u32    tile hash slot of the particle in work slot t
//   bin_rank    N x u32    its rank inside that tile
//   sorted      N x u32    work slots grouped by tile (this substep's tile order)
//   keys        cap x u64  open-addressing tile hash (hash3 of the tile coord,
//                          linear probing); EMPTY = ~0
//   slot_count  cap x u32  particles per slot
//   slot_off, slot_st      per-slot particle offset and compact tile index
//   st_key/st_slot/st_begin/st_count   per compact tile
//   tiles[3]    max_tiles x (E+2)^3 x int4   per-tile halo sums
//               (mass, momentum x, y, z) in the reference i32 fixed point;
//               the PBMPM iterations write the cell's reciprocal mass of the
//               substep (f32 bits, formed by the first iteration) in place of
//               the mass, and their momentum sums
//   iter_rec    IR_PLANES x N float4         PBMPM iteration records (below)
//   st_nbr      max_tiles x 27 i32           compact index of each tile's 27
//                                            neighbours (d = 9(dz+1) + 3(dy+1) + dx+1),
//                                            built once per substep after binning
//
// A tile is E^3 grid cells (E = 8, 12, 14 or 16; 8, 12 and 16 are 2^3, 3^3 and 4^3 of
// the reference's 4^3-cell blocks).  Its P2G writes the (E+2)^3 halo region it touches; the
// grid value of a cell is the i32 sum over every tile halo that covers it
// (at most 8), formed on the fly by the G2P kernels.  Integer addition
// commutes, so the sums equal the reference's atomicAdd totals exactly.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {

constexpr uint64_t KEY_EMPTY = ~0ull;
constexpr uint32_t INVALID = 0xFFFFFFFFu;
constexpr uint32_t MAX_PROBES = 1024u;
constexpr int COMPACT_CHUNK = 4096;   // hash slots per compaction block (256 threads x 16)
constexpr int KEY_BIAS = 32768;
// PBMPM iteration record of one binned particle, stored plane by plane
// (plane q of sorted position t at iter_rec[q * n + t]):
//   0: pos.xyz, mass   1: Fe[0..3]   2: Fe[4..7]   3: Fe[8], Fe^-1[0..2]
//   4: Fe^-1[3..6]     5: Fe^-1[7..8], elasticity relaxation, 0
// Fe, Fp and the position do not change between the iterations of one
// substep, so Fe^-1 and the relaxation factor (pbmpm.wgsl:29-35) are formed
// once, by the first iteration, instead of once per iteration.
constexpr int IR_PLANES = 6;
// Float4 words of a particle record (192 B), one plane each in the work buffers.
constexpr int REC_PLANES = 12;

// status bits (mirror of MPM_STATUS_* in include/mpm.h)
constexpr uint32_t ST_HASH_FULL = 0x1u;
constexpr uint32_t ST_TILE_OVERFLOW = 0x2u;
constexpr uint32_t ST_BVH_STACK = 0x4u;
constexpr uint32_t ST_SCENE_RANGE = 0x8u;
constexpr uint32_t ST_MLP_FALLBACK = 0x10u;
constexpr uint32_t ST_MLP_TIMEOUT = 0x20u;
constexpr uint32_t ST_COPY_TIMEOUT = 0x40u;


// Per-scene parameters: the uniform fields the step reads plus the
// extension constants, laid out for a word-wise copy into shared memory.
struct SceneDev {
    float dt, scale;
    float gmin[3], gmax[3], cd[3];
    int32_t res[3];
    float cmin[3], cmax[3];
    float xf[16], xfi[16];
    float cvel[3];
    uint32_t c_nidx, c_nobj;
    float ipos[3], istr, irad;
    uint32_t iact, imode;
    float g[3], mu0, la0, xi_e, xi_p, smin, smax, inv_rho;
    uint32_t n_iter;
    float fdiv;
    uint32_t bmode;
    float rest;
    int32_t bc;
    uint32_t gaxis;
    float cmargin, csurf, cthr, cfric, cvs, blend, vexp;
    uint32_t p_first, p_count;
    uint32_t col_words, n_nodes;
    const uint32_t* col_data;
    const uint32_t* bvh;
    // per-triangle bounds in leaf order (lo, hi as float4 pairs) and whether
    // the collider transform is the identity: triangles whose bounds are
    // farther from the particle than the collider threshold and clear of
    // its path are skipped (collide)
    const float4* tbox;
    uint32_t cull, cull_pad;
    // distance field of the collider (used with the identity transform, as
    // tbox): per cell of a df_res^3 grid over the triangles' bounds, a lower
    // bound of the distance from any point of the cell to every triangle;
    // nullptr when the collider has none
    const float* dfield;
    float df_lo[3], df_rcs[3];
    uint32_t df_res, df_pad;
    // reciprocals RN(1/d) of the substep-constant divisors, rounded once on
    // the host: x / d evaluates as x * RN(1/d)
    float rdt, rcd[3], rscale, rfdiv;
    float gdiv[3];     // gravity * RN(1/force_divisor) (pbmpm.wgsl:137)
    float gdt[3];      // gravity * dt (gridUpdate.cs.wgsl:44)
    // fixed-point encodings i32((x * RN(1/dt)) * scale) and
    // i32(((f * wm) * dt) * scale): when scale = 2^k, 0 <= k < 126, scaling
    // by it is exact for every value that can reach a nonzero i32, so the
    // two products fold into one multiply by rdts = RN(1/dt) * 2^k or
    // dts = dt * 2^k with the same i32 result
    uint32_t fold;
    float rdts, dts;
    uint32_t rmap;     // return map: 0 applyPlasticity, 1 SVD clamp (deferred pass only)
    uint32_t rmap_pad;
};
static_assert(sizeof(SceneDev) % 8 == 0, "SceneDev must be 8-byte sized");

// Arguments of the volumetric ray march (mpm_raymarch.cu).
struct RaymarchArgs {
    const uint32_t* mass;   // res[0] * res[1] * res[2] u32, x fastest (calculateGridMass output)
    uint32_t res[3];
    float gmin[3], gmax[3];
    float scale;            // fixedPointScale
    float inv_vp[16];       // viewProjInvMat, column-major
    uint32_t time;
    uint32_t width, height;
    uint8_t* rgba;          // width * height * 4 (rgba8unorm)
    float* depth;           // width * height (r32float)
    float* color;           // optional width * height * 4: the stored vec4f before quantisation
};
cudaError_t launch_raymarch(const RaymarchArgs& a, cudaStream_t s);

struct Counters {
    uint32_t n_st;       // occupied tiles of the current substep
    uint32_t n_binned;   // particles placed in tiles
    uint32_t status;     // sticky status bits
    uint32_t n_plast;    // deferred plasticity candidates of the current substep
    uint32_t step;       // substeps run on this buffer (advanced at each substep's start)
    uint32_t tile_ticket;  // tile kernels: tiles claimed past each CTA's first (0 between launches)
    uint32_t tile_done;    // tile kernels: CTAs finished; the last one resets both
    uint32_t n_carry;      // particles no tile kernel advances this substep (no hash slot):
                           // copied unchanged into work slots n_binned, n_binned + 1, ...
};

struct Ctx {
    const float4* work_in;    // particle state before the substep: REC_PLANES planes of n float4
    float4* work_out;         // after the substep, slots in this substep's tile order
    const uint32_t* ids_in;   // caller index of each slot of work_in
    uint32_t* ids_out;        // caller index of each slot of work_out
    uint32_t* sorted;         // slots of work_in grouped by tile (this substep's tile order)
    uint32_t* bin_slot;
    uint32_t* bin_rank;
    unsigned long long* keys;
    uint32_t* slot_count;
    uint32_t* slot_off;
    uint32_t* slot_st;
    unsigned long long* st_key;
    uint32_t* st_slot;
    uint32_t* st_begin;
    uint32_t* st_count;
    uint32_t* chunk_nst;
    uint32_t* chunk_np;
    int4* tiles_a;            // tiles written by this pass's P2G
    int4* tiles_b;            // tiles read by this pass's G2P
    float4* iter_rec;         // PBMPM iteration records, IR_PLANES x n float4, sorted order
    int32_t* st_nbr;          // per compact tile, the compact index of its 27 neighbours (-1: none)
    uint32_t* tile_order;     // optional: the order the tile kernels claim tiles in (Morton order of
                              // the tile coordinates, per scene); nullptr: compact index order
    uint32_t order_rev;       // this launch claims tile_order from its end (alternates per launch)
    uint32_t order_mode;      // tile claim order: 0 automatic, 1 compact index order, 4 / 5 Morton
                              // buckets of 4 / 5 bits per axis (schedule knob of the autotuner)
    const int4* tiles_m;      // readback only: tiles holding the substep's mass sums (nullptr: tiles_b)
    uint32_t iter_first;      // this PBMPM iteration forms the reciprocal masses from the mass sums
    uint32_t g2p_rm;          // the final PBMPM G2P reads the reciprocal masses from the halo records
    uint32_t* plast_list;     // deferred plasticity: work_out slots the strain-bound check did not clear
    uint32_t plast_defer;     // 0: exact return map inside integrate; 1: deferred to the plasticity pass
    const SceneDev* scenes;
    const uint32_t* scene_first;  // n_scenes + 1 particle offsets
    Counters* counters;
    uint32_t n_particles;
    uint32_t n_scenes;
    uint32_t cap;             // hash capacity, power of two
    uint32_t max_tiles;
};

__host__ __device__ inline uint64_t pack_key(uint32_t scene, int sx, int sy, int sz) {
    return ((uint64_t)scene << 48) | ((uint64_t)(uint32_t)(sx + KEY_BIAS) << 32) |
           ((uint64_t)(uint32_t)(sy + KEY_BIAS) << 16) | (uint64_t)(uint32_t)(sz + KEY_BIAS);
}
__host__ __device__ inline void unpack_key(uint64_t k, uint32_t& scene, int& sx, int& sy, int& sz) {
    scene = (uint32_t)(k >> 48);
    sx = (int)((k >> 32) & 0xffff) - KEY_BIAS;
    sy = (int)((k >> 16) & 0xffff) - KEY_BIAS;
    sz = (int)(k & 0xffff) - KEY_BIAS;
}

enum KernelId : uint32_t {
    K_CLEAR_TABLE = 0,
    K_BIN_INSERT,
    K_COMPACT_A,
    K_COMPACT_B,
    K_COMPACT_C,
    K_BIN_SCATTER,
    K_P2G_EXPLICIT,
    K_G2P_EXPLICIT,
    K_PBMPM_FIRST,
    K_PBMPM_ITER,
    K_G2P_PBMPM,
    K_GRID_DENSE,
    K_TILE_NBR,
    K_PLASTICITY,
    K_TILE_ORDER,
    K_P2G_EXPLICIT_128,       // the explicit tile kernels with 128-thread CTAs (schedule knob)
    K_G2P_EXPLICIT_128,
    K_PBMPM_ITER_WIDE,        // the PBMPM tile kernels with 512-thread CTAs at tile edge 8 (few tiles)
    K_PBMPM_FIRST_WIDE,
    K_G2P_PBMPM_WIDE,
    K_P2G_EXPLICIT_WIDE,      // the explicit tile kernels with 512-thread CTAs at tile edge 8 (few tiles)
    K_G2P_EXPLICIT_WIDE,
    K_COUNT
};

}  // namespace mpm
