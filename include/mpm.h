/*
 * mpm.h -- C ABI of libmpm.so, the B200 (sm_100a) implementation of the
 * MPM snow simulation step of luoluobuli/WebGPU-MPM-based-Snow-Simulation.
 *
 * The library keeps the reference's data contracts:
 *   - particles are the 192-byte ParticleData records of
 *     src/lib/gpu/shaderPrelude/mpmOps.wgsl:1-12 (GpuMpmBufferManager.ts:22-26);
 *   - step parameters arrive as the reference's 37,376-byte uniform block
 *     (src/lib/gpu/shaderPrelude/uniforms.wgsl:8-56,
 *     src/lib/gpu/uniforms/GpuUniformsBufferManager.ts:15-182), plus an
 *     extension struct for the constants the WGSL hard-codes;
 *   - the collider is the reference's packed u32 buffer and 32-byte BVH nodes
 *     (src/lib/gpu/collider/GpuColliderBufferManager.ts:96-220,
 *     src/lib/gpu/mpm/colliderPrelude.wgsl:1-27).
 *
 * Conventions: every function returns an int status (MPM_OK = 0, negative =
 * error; mpm_last_error() gives the message).  No exception crosses the ABI.
 * A handle is not thread-safe; all device work is ordered on the handle's
 * CUDA stream and asynchronous unless stated.  Scenes: a handle advances
 * one or more independent scenes in the same launches; scene s owns the
 * particle records [first, first+count) given by mpm_set_scene_range().
 */
#ifndef MPM_H
#define MPM_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_UNIFORMS_BYTES 37376u
#define MPM_PARTICLE_BYTES 192u
#define MPM_BVH_NODE_BYTES 32u

#define MPM_OK 0
#define MPM_ERR_ARG (-1)
#define MPM_ERR_CUDA (-2)
#define MPM_ERR_CAPACITY (-3)
#define MPM_ERR_STATE (-4)
#define MPM_ERR_DEVICE_STATUS (-5)

/* Simulation methods (src/lib/gpu/GpuSimulationMethod.ts:1-4). */
#define MPM_METHOD_EXPLICIT 0
#define MPM_METHOD_PBMPM 1

/* Device status bits, sticky until mpm_clear_status(). */
#define MPM_STATUS_HASH_FULL      0x1u  /* tile hash table ran out of probes */
#define MPM_STATUS_TILE_OVERFLOW  0x2u  /* more occupied tiles than max_tiles */
#define MPM_STATUS_BVH_STACK      0x4u  /* BVH traversal dropped children (stack of 32 full) */
#define MPM_STATUS_SCENE_RANGE    0x8u  /* a particle index belongs to no scene */
#define MPM_STATUS_MLP_FALLBACK   0x10u /* learned plasticity fell back to the exact map */
#define MPM_STATUS_MLP_TIMEOUT    0x20u /* a tensor-core wait of the plasticity pass ran out */
#define MPM_STATUS_COPY_TIMEOUT   0x40u /* a halo bulk-copy wait of a tile kernel ran out */

typedef struct MpmHandle MpmHandle;

typedef struct MpmConfig {
    uint32_t max_particles;  /* capacity of the particle buffer, all scenes */
    uint32_t max_scenes;     /* 1 for a single scene */
    uint32_t max_tiles;      /* occupied grid tiles per substep (0: derived) */
    uint32_t hash_capacity;  /* tile hash slots, rounded up to a power of two (0: derived) */
    uint32_t tile_edge;      /* grid tile edge in cells: 8, 12, 14 or 16; 0: chosen at the
                              * first step (and again after the particle count changes)
                              * from the occupied tiles (mpm_get_tile_edge) */
    int32_t device;          /* CUDA device ordinal */
    void* stream;            /* cudaStream_t to order work on, or NULL for a private stream */
} MpmConfig;

/* Constants the reference hard-codes in WGSL, per scene.  mpm_default_params
 * fills the reference values (cited per field). */
typedef struct MpmParams {
    float gravity[3];            /* gridUpdate.cs.wgsl:43, pbmpm.wgsl:101: (0,0,-9.81) */
    float youngs_modulus;        /* stressTensorOps.wgsl:1: 1.4e5 */
    float poissons_ratio;        /* stressTensorOps.wgsl:2: 0.2 */
    float hardening_explicit;    /* stressTensorOps.wgsl:44: 5 */
    float hardening_pbmpm;       /* pbmpm.wgsl:35: 20 */
    float theta_c;               /* plasticityOps.wgsl:18: 2.5e-2 */
    float theta_s;               /* plasticityOps.wgsl:19: 7.5e-3 */
    float density;               /* particleToGrid.cs.wgsl:36: 400 */
    uint32_t n_iter;             /* GpuMpmPipelineManager.ts:445: 3 */
    float force_divisor;         /* pbmpm.wgsl:137: 3 */
    uint32_t boundary_mode;      /* 0 reference particle reflect; 1 adds grid sticky ground + slip walls */
    float restitution;           /* integrateParticles.wgsl:34: -0.5 */
    uint32_t bc_cells;           /* boundary_mode 1: boundary layer width, cells (2) */
    uint32_t ground_axis;        /* boundary_mode 1: sticky plane at grid min of this axis (2) */
    float collider_margin;       /* colliderPrelude.wgsl:158: 0.05 */
    float collider_surface_margin; /* colliderPrelude.wgsl:297,351: 0.05 */
    float collider_threshold;    /* colliderPrelude.wgsl:330: 0.05 */
    float collider_friction;     /* colliderPrelude.wgsl:308: 0.1 */
    float collider_vel_scale;    /* colliderPrelude.wgsl:294: 0.2 */
    float pbmpm_blend;           /* pbmpm.wgsl:26: 0.95 */
    float pbmpm_volume_exponent; /* pbmpm.wgsl:23: -0.3333333 */
    uint32_t return_map;         /* 0: applyPlasticity (plasticityOps.wgsl:7-48), the clamp of the
                                  * diagonal of R^T Fe; 1: a true-SVD clamp of the singular values,
                                  * an option of this library (applied by the deferred plasticity
                                  * pass; not available to mpm_step_noalloc) */
} MpmParams;

/* ---- lifetime ------------------------------------------------------ */
int mpm_default_params(MpmParams* out);
/* Allocates the particle and bookkeeping buffers.  Grid-tile storage and the
 * tile hash table are sized from the first substep's occupancy when
 * max_tiles / hash_capacity are 0 (again by the first step after the particle
 * count changes) and grown only inside mpm_sync (between substeps); a substep
 * itself never allocates.  Records of the same count that occupy many more tiles than the
 * previous ones can exceed the storage in the first substep after them: it
 * sets MPM_STATUS_TILE_OVERFLOW (or HASH_FULL) and leaves the particles of the
 * tiles beyond the storage unchanged, and the next mpm_sync grows it. */
int mpm_create(const MpmConfig* cfg, MpmHandle** out);
int mpm_destroy(MpmHandle* h);
const char* mpm_last_error(const MpmHandle* h);

/* ---- parameters (GpuUniformsBufferManager.ts:54-182) ---------------- */
/* Accepts the reference uniform block verbatim (n >= 544 bytes are read:
 * the fields the step uses lie below the collider-object array). */
int mpm_set_uniforms(MpmHandle* h, uint32_t scene, const void* bytes, size_t n);
int mpm_set_params(MpmHandle* h, uint32_t scene, const MpmParams* p);
/* Scene s owns particle records [first, first + count); scenes must tile
 * [0, n_particles) in increasing order. */
int mpm_set_scene_range(MpmHandle* h, uint32_t scene, uint32_t first, uint32_t count);
int mpm_set_scene_count(MpmHandle* h, uint32_t n_scenes);

/* ---- particles (GpuMpmBufferManager.ts:22-26) ---------------------- */
/* Copies n 192-byte records into the library buffer (src on host or device;
 * a host copy is enqueued on the handle's stream: asynchronous from pinned
 * memory).  The library advances its own copy of the state with the records
 * in tile order; mpm_get_particles (and mpm_particles_device_ptr, and every
 * step call on a caller-bound buffer) restores the caller's order first. */
int mpm_set_particles(MpmHandle* h, const void* src, uint32_t n, int src_is_device);
/* dst_is_device: 0 host memory, the call waits for the copy; 1 device memory;
 * 2 host memory, the copy is only enqueued on the handle's stream (dst must
 * be pinned and is valid after mpm_sync or a stream synchronisation). */
int mpm_get_particles(MpmHandle* h, void* dst, uint32_t n, int dst_is_device);
/* Zero-copy: the caller's device buffer of n records (16-byte aligned) is the
 * library's record buffer; every step call leaves it holding the advanced
 * records in the caller's order (enqueued on the handle's stream). */
int mpm_bind_particles_device(MpmHandle* h, void* dptr, uint32_t n);
/* The device record buffer in the caller's order, brought up to date on the
 * handle's stream first (read it after mpm_sync); NULL on failure. */
void* mpm_particles_device_ptr(MpmHandle* h);

/* ---- collider (GpuColliderBufferManager.ts:61-220) ------------------ */
/* data: [reordered indices (num_indices u32) | vertices f32x3 | ...];
 * nodes: n_nodes 32-byte BVH nodes.  Host pointers; copied to the device. */
int mpm_set_collider(MpmHandle* h, uint32_t scene, const uint32_t* data, size_t words,
                     uint32_t num_indices, const void* nodes, uint32_t n_nodes);
/* Host-side BVH build in the reference format (GpuColliderBufferManager.ts:222-350):
 * median split on the longest axis, leaves of <= 4 triangles, pre-order nodes.
 * nodes_out needs room for 2*n_tris+1 nodes; tri_order_out for n_tris. */
int mpm_build_bvh(const float* vertices, uint32_t n_vertices, const uint32_t* indices,
                  uint32_t n_indices, void* nodes_out, uint32_t* tri_order_out, uint32_t* n_nodes_out);
/* The same build on the GPU, node for node and bit for bit the tree of
 * mpm_build_bvh (level-synchronous: per-node bounds by block reduction, the
 * per-node stable centroid sort as one stable radix sort of (node, centroid)
 * keys per level).  Device pointers; nodes_dev needs mpm_bvh_node_count(n_tris)
 * nodes, tri_order_dev n_tris u32.  Enqueued on `stream` (a cudaStream_t, NULL
 * for the default stream) and synchronised before returning; MPM_ERR_ARG if an
 * index is >= n_vertices. */
uint32_t mpm_bvh_node_count(uint32_t n_triangles);
int mpm_build_bvh_device(const float* vertices_dev, uint32_t n_vertices, const uint32_t* indices_dev,
                         uint32_t n_indices, void* nodes_dev, uint32_t* tri_order_dev, uint32_t* n_nodes_out,
                         void* stream);
/* A device-resident collider mesh installed without a host round trip: the
 * BVH built on the GPU, the index buffer reordered into leaf order on the GPU,
 * the collider buffer laid out as mpm_set_collider's (indices | vertices). */
int mpm_set_collider_mesh_device(MpmHandle* h, uint32_t scene, const float* vertices_dev, uint32_t n_vertices,
                                 const uint32_t* indices_dev, uint32_t n_indices);

/* ---- the step (GpuMpmPipelineManager.ts:327-521) ------------------- */
/* Enqueues n_substeps substeps of `method` on the handle's stream. */
int mpm_step(MpmHandle* h, int method, uint32_t n_substeps);
/* The reference's two entry points, one substep each
 * (GpuMpmPipelineManager.ts:327 addExplicitMpmDispatches, :431 addPbmpmDispatches).
 * n_particles must equal the bound particle count. */
int mpm_add_explicit_mpm_dispatches(MpmHandle* h, uint32_t n_particles);
int mpm_add_pbmpm_dispatches(MpmHandle* h, uint32_t n_particles);
/* Waits for the stream; returns MPM_ERR_DEVICE_STATUS if a status bit is set. */
int mpm_sync(MpmHandle* h, uint32_t* status_out);
int mpm_clear_status(MpmHandle* h);

/* ---- inspection ----------------------------------------------------- */
/* Runs one substep only up to its first particle-to-grid transfer (for grid
 * parity checks); the particle buffer keeps its input values. */
int mpm_step_p2g_only(MpmHandle* h, int method);
/* Dense copy of scene `scene`'s grid, [res_z][res_y][res_x][4] i32 (mass,
 * momentum x, y, z) in the reference fixed-point encoding; cells no particle
 * reaches are 0.  apply_grid_update = 1 reproduces the explicit grid update
 * (gridUpdate.cs.wgsl:15-53), i.e. the reference buffers after a full
 * explicit substep.  Synchronous. */
int mpm_get_grid_dense(MpmHandle* h, uint32_t scene, int apply_grid_update,
                       int32_t* out_host, size_t n_cells);
/* Number of occupied tiles and binned particles of the last substep (synchronous). */
int mpm_get_counts(MpmHandle* h, uint32_t* n_tiles, uint32_t* n_binned);
/* The tile edge the substeps run with.  For a handle created with tile_edge 0
 * it is 16 until the first step picks one of 16, 12 and 8 from the occupied
 * tiles of the particles (picked again by the first step after a change of
 * the particle count): among the edges with at least two occupied tiles per
 * SM, the one whose tiles hold the fewest halo cells ((E+2)^3 per tile; a
 * smaller edge only below 9/10 of a larger one's), else the edge with the
 * most tiles.  Results do not depend on the tile edge. */
int mpm_get_tile_edge(MpmHandle* h, uint32_t* edge);
/* Per-kernel timing: when enabled, each launch of a substep is bracketed by
 * CUDA events on the handle's stream; mpm_kernel_times returns the summed
 * milliseconds and launch counts per kernel id since the last reset. */
int mpm_enable_kernel_timing(MpmHandle* h, int enable);
int mpm_kernel_times(MpmHandle* h, float* ms_out, uint32_t* launches_out, uint32_t n_kernels);
const char* mpm_kernel_name(uint32_t kernel_id);
uint32_t mpm_kernel_count(void);
/* Captures each substep into a CUDA graph (default on). */
int mpm_use_graphs(MpmHandle* h, int enable);
/* Schedule knobs (an extension; the reference dispatches fixed 4^3-block
 * workgroups, sparseGridPrelude.wgsl:1-7), set by the autotuner.  The
 * results do not depend on them.  order_mode: the order the tile kernels
 * claim tiles in -- 0 automatic (compact order up to 256 occupied tiles,
 * Morton buckets of 4 bits per axis up to 4,096, else 5), 1 compact order,
 * 4 or 5 Morton buckets of that many bits per axis.  tile_block: threads per
 * CTA of the explicit tile kernels, 0 or 256 (default) or 128. */
int mpm_set_schedule(MpmHandle* h, uint32_t order_mode, uint32_t tile_block);
/* Device self-test of the step's arithmetic helpers, on n pseudo-random
 * operand pairs: the folded fixed-point encoding i32(x * (r * 2^k)) against
 * i32((x * r) * 2^k), and the device reciprocal against the IEEE quotient
 * 1/d (ident_mismatches counts failures of either); and the saturating
 * f32->i32 conversion (cvt_mismatches: bit mask of failed cases).  Both must
 * be 0.  nan_conversion reports the hardware's raw truncating conversion of
 * a NaN. */
int mpm_selftest(int device, uint64_t n, uint64_t seed, uint64_t* ident_mismatches, uint64_t* cvt_mismatches,
                 uint64_t* nan_conversion);

/* ---- particle initialisation --------------------------------------- */
/* scatterParticles (src/lib/gpu/particleInitialize/particleScatter.cs.wgsl:47-84):
 * fills the handle's first n_particles records with positions drawn inside
 * the closed triangle mesh (rejection sampling in the box given by scene
 * 0's uniform meshMinCoords / meshMaxCoords, even-odd ray parity, at most 512
 * attempts), fBm-jittered, with hashed masses and rest state.  vertices: host
 * triangle soup, n_vertices x 4 floats (x, y, z, unused), as the reference's
 * mesh vertex buffer (GpuMeshBufferManager.ts:30-43).  Synchronous. */
int mpm_scatter_particles(MpmHandle* h, const float* vertices, uint32_t n_vertices, uint32_t n_particles);

/* ---- renderer splats ------------------------------------------------ */
/* The particle splats the reference's renderers run after the step, into the
 * caller's device buffer of u32 (res_x * res_y * res_z, x fastest), enqueued
 * on the handle's stream; accumulate = 0 clears the buffer first.
 * mpm_grid_mass: calculateGridMass (src/lib/gpu/volumetric/calculateGridMass.wgsl:8-51),
 *   on the scene's simulation grid (uniform gridResolution).
 * mpm_mc_density: calculateDensity (src/lib/gpu/marchingCubes/mcDensity.cs.wgsl:14-63),
 *   on a density grid of density_res[3] cells over the same domain (the
 *   reference uses half the simulation resolution,
 *   src/lib/gpu/marchingCubes/GpuMarchingCubesBufferManager.ts:44-48). */
int mpm_grid_mass(MpmHandle* h, uint32_t scene, uint32_t* out_dev, int accumulate);
int mpm_mc_density(MpmHandle* h, uint32_t scene, const uint32_t* density_res, uint32_t* out_dev, int accumulate);

/* ---- marching cubes --------------------------------------------------- */
/* The mesh-generation passes of GpuMarchingCubesRenderPipelineManager
 * (src/lib/gpu/marchingCubes/GpuMarchingCubesRenderPipelineManager.ts:587-633:
 * mcListBlocks, mcVertexDensity, mcGenerate, mcClampArgs) over a density grid
 * made by mpm_mc_density: vertices_dev receives 6 f32 per vertex (position,
 * normal), 3 vertices per triangle, in a deterministic order (active 8^3
 * blocks ascending, cells in block order, triangles in table order); at most
 * max_vertices are written.  *vertex_count_out = min(generated, max_vertices)
 * (the clamped draw count), *vertices_generated_out (optional) = generated.
 * The triangulation table is this library's (mpm_mc_tables): the iso-contour
 * traced around the cube with inside corners kept apart on ambiguous faces,
 * the reference's vertex and edge numbering.  Synchronises the stream. */
int mpm_marching_cubes(MpmHandle* h, uint32_t scene, const uint32_t* density_dev, const uint32_t* density_res,
                       const uint32_t* mc_res, float* vertices_dev, uint32_t max_vertices,
                       uint32_t* vertex_count_out, uint32_t* vertices_generated_out);
/* tri_out 256 x 16 edge indices (-1 padded), count_out 256 triangle counts,
 * edge_vertices_out 12 x 2 cube vertex ids; any may be NULL. */
int mpm_mc_tables(int8_t* tri_out, uint8_t* count_out, uint8_t* edge_vertices_out);

/* ---- volumetric ray march ------------------------------------------- */
/* doVolumetricRaymarch (src/lib/gpu/volumetric/volumetricRaymarch.cs.wgsl:118-226,
 * dispatched by GpuVolumetricRenderPipelineManager.addRaymarchDispatch,
 * GpuVolumetricRenderPipelineManager.ts:332-339) into headless device buffers
 * instead of the storage textures: rgba_dev width*height*4 bytes (rgba8unorm,
 * round to nearest), depth_dev width*height f32 (r32float; left unwritten
 * where the ray misses the grid, as the texture is), color_dev optional
 * width*height*4 f32 (the stored vec4f before quantisation).  mass_grid_dev is
 * the scene's calculateGridMass grid (mpm_grid_mass); the camera is the
 * uniform block's viewProjInvMat (@112) and the jitter seed its time (@12).
 * Enqueued on the handle's stream; 1 <= width, height <= 16384. */
int mpm_volumetric_raymarch(MpmHandle* h, uint32_t scene, const uint32_t* mass_grid_dev, uint32_t width,
                            uint32_t height, uint8_t* rgba_dev, float* depth_dev, float* color_dev);

/* ---- learned plasticity --------------------------------------------
 * The snow return map applyPlasticity (src/lib/gpu/shaderPrelude/
 * plasticityOps.wgsl:7-48, called from integrateParticles.wgsl) can run in
 * four ways, chosen per handle:
 *   INLINE  (default) the exact map inside the integrate kernel, as the reference;
 *   EXACT   integrate applies a strain-bound check (all Gershgorin discs of
 *           Fe^T Fe inside the elastic band, so the exact map would return
 *           its input unchanged) and lists the rest; a separate pass runs
 *           the exact map on them.  Results equal INLINE bit for bit;
 *   COLLECT as EXACT, and a sampled fraction (audit_fraction, drawn per
 *           particle and substep) of the listed particles inside the trained
 *           domain also writes a training pair (12 inputs, 10 targets) to
 *           the buffer given by mpm_set_pair_buffer;
 *   LEARNED as EXACT, but the pass runs the network (BF16 tensor cores,
 *           FP32 accumulation) and takes its answer unless the particle is
 *           outside the trained domain, the uncertainty output exceeds
 *           unc_threshold, or the determinant check fails (|ln det Fp'
 *           recomputed - ln J_p predicted| > det_threshold); those particles,
 *           and an audited fraction of the rest, take the exact map.
 * Network: 12 -> 64 -> 64 -> 64 -> 11, SiLU.  Inputs: (Fe_trial - I) * 20
 * (9, column-major), 2 ln det Fp, log2(dt) + 13.2877, (theta_c - 0.025) * 100.
 * Targets: (Fe' - Fe_trial) * 100 (9), (ln det Fp' - ln det Fp) * 100; output
 * 10 estimates the error norm of the other ten.  Parameters: MPM_MLP_PARAMS
 * FP32 values packed [W1 64x12 | b1 64 | W2 64x64 | b2 | W3 64x64 | b3 |
 * W4 11x64 | b4 11], W row-major [out][in].  No counterpart in the reference
 * (its plasticity is always the exact map). */
#define MPM_PLASTICITY_INLINE 0
#define MPM_PLASTICITY_EXACT 1
#define MPM_PLASTICITY_COLLECT 2
#define MPM_PLASTICITY_LEARNED 3
#define MPM_MLP_INPUTS 12
#define MPM_MLP_HIDDEN 64
#define MPM_MLP_OUTPUTS 11
#define MPM_MLP_TARGETS 10
#define MPM_MLP_PARAMS 9867

typedef struct MpmMlp MpmMlp;

typedef struct MpmMlpTrainConfig {
    uint32_t epochs;
    uint32_t batch;        /* pairs per Adam step */
    float lr;              /* initial learning rate, cosine-decayed to lr_final */
    float lr_final;
    float unc_weight;      /* weight of the uncertainty head's loss */
    uint32_t seed;         /* shuffling */
} MpmMlpTrainConfig;

typedef struct MpmPlasticityStats {
    uint64_t candidates;          /* particles the strain-bound check did not clear (all deferred modes) */
    uint64_t learned;             /* took the network's answer */
    uint64_t fallback_domain;     /* outside the trained domain (exact map; in COLLECT mode: no pair) */
    uint64_t fallback_uncertain;  /* exact: uncertainty above threshold */
    uint64_t fallback_det;        /* exact: determinant check failed */
    uint64_t audited;             /* exact, with the network's error recorded */
    float audit_max_err;          /* max over audited particles of max |Fe'_net - Fe'_exact| */
    float audit_mean_err;
    uint32_t pairs_collected;
    uint32_t pad;
} MpmPlasticityStats;

/* Seeded initial parameters (host only). */
int mpm_mlp_init_params(uint32_t seed, float* out);
int mpm_mlp_create(int device, uint32_t seed, MpmMlp** out);
int mpm_mlp_destroy(MpmMlp* m);
const char* mpm_mlp_last_error(const MpmMlp* m);
/* Orders the network's work on the caller's cudaStream_t (NULL: a private
 * stream, the default).  Calls still return after their work completes. */
int mpm_mlp_set_stream(MpmMlp* m, void* stream);
int mpm_mlp_get_params(MpmMlp* m, float* host_out);
int mpm_mlp_set_params(MpmMlp* m, const float* host_in);
/* Network outputs for n inputs (device arrays [n][12] -> [n][11]); synchronous. */
int mpm_mlp_forward(MpmMlp* m, const float* x_dev, uint32_t n, float* y_dev);
/* Loss and gradient of the batch loss over n pairs (device arrays
 * [n][12], [n][10]) at the current parameters; grad_host receives
 * MPM_MLP_PARAMS values.  Loss = (1/n) sum [ |y[0..9] - t|^2 +
 * unc_weight (y[10] - |y[0..9] - t|)^2 ]. */
int mpm_mlp_gradient(MpmMlp* m, const float* x_dev, const float* t_dev, uint32_t n, float unc_weight,
                     float* grad_host, float* loss_host);
/* Adam training on the GPU over n pairs; loss_per_epoch (may be NULL)
 * receives cfg->epochs mean batch losses. */
int mpm_mlp_train(MpmMlp* m, const float* x_dev, const float* t_dev, uint32_t n,
                  const MpmMlpTrainConfig* cfg, float* loss_per_epoch);
/* Selects the plasticity mode of a handle (net: required for LEARNED, must
 * outlive its use and must not train while the handle steps). */
int mpm_set_plasticity(MpmHandle* h, int mode, MpmMlp* net, float unc_threshold, float det_threshold,
                       float audit_fraction);
/* Training-pair buffer for COLLECT mode (device arrays [capacity][12],
 * [capacity][10]); resets the pair count. */
int mpm_set_pair_buffer(MpmHandle* h, float* x_dev, float* t_dev, uint32_t capacity);
int mpm_get_plasticity_stats(MpmHandle* h, MpmPlasticityStats* out, int reset);

/* ---- allocation-free substep ----------------------------------------
 * No counterpart in the reference (its TypeScript managers own every GPU
 * buffer).  For callers that cannot allocate device memory while they run:
 * a host that hands the library a fixed device-memory budget and owns every
 * allocation itself (an engine or renderer sharing the GPU through its own
 * pool), or a real-time frame loop that must not pay cudaMalloc's implicit
 * device-wide synchronisation.  The caller passes its inputs and outputs
 * (particle records, collider arrays: device pointers on `device`); every
 * intermediate buffer of the substep (the tile-ordered particle state,
 * particle bins, tile hash table, grid tile sums) lives in one static device
 * array of MPM_NOALLOC_SCRATCH_BYTES
 * that each GPU loading the library holds until the process exits.  The
 * call allocates nothing: no cudaMalloc, no cudaFree, no allocating library
 * routine.
 *
 * Limits: at most MPM_NOALLOC_MAX_PARTICLES particles (larger counts are
 * rejected with MPM_ERR_CAPACITY) and MPM_NOALLOC_MAX_TILES occupied tiles
 * of MPM_NOALLOC_TILE_EDGE^3 cells (more set status 0x2; tiles past the
 * limit are skipped).  One scene per call.
 *
 * The first call on a device sets the device up (looks up the array's
 * device address with cudaGetSymbolAddress and configures the kernels);
 * make that first call before any stream capture.  Every call shares the
 * one array and clears what must start empty, so calls whose work overlaps
 * on the GPU (different streams, or other host threads, on one device) race
 * and must be serialised by the caller.  Work is enqueued on `stream`
 * (NULL: the legacy default stream); the scene record travels as a kernel
 * argument, so with status_out NULL the call returns without waiting for the
 * GPU and the device status is not reported.  If status_out is non-NULL the
 * call waits for the stream, stores the device status bits and returns
 * MPM_ERR_DEVICE_STATUS when any is set.  The collider query tests every
 * triangle of a leaf it reaches: the per-triangle bounds a handle uses to
 * skip distant triangles would need an allocation, so this path does without
 * them (same results, slower on large meshes).  err (err_len bytes, may be
 * NULL) receives a message on failure.  The calling thread's current device
 * is restored on return. */
#define MPM_NOALLOC_MAX_PARTICLES 65536u
#define MPM_NOALLOC_MAX_TILES 512u
#define MPM_NOALLOC_TILE_EDGE 8u
#define MPM_NOALLOC_HASH_SLOTS 8192u
#define MPM_NOALLOC_SCRATCH_BYTES (50u << 20)
int mpm_step_noalloc(int device, void* stream, void* particles, uint32_t n_particles, int method,
                     const void* uniforms, size_t uniform_bytes, const MpmParams* params,
                     const uint32_t* collider_data, size_t collider_words, uint32_t num_indices,
                     const void* bvh_nodes, uint32_t n_nodes, uint32_t* status_out, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
