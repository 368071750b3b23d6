/*
 * mpm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference MPM simulation step
 * (luoluobuli/WebGPU-MPM-based-Snow-Simulation, the WGSL kernels under src/lib/gpu/mpm/ and
 * the prelude under src/lib/gpu/shaderPrelude/, scheduled by
 * src/lib/gpu/mpm/GpuMpmPipelineManager.ts:327-521).
 *
 * Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark may load this code, and only as the reference of a check or as the timed CPU
 * baseline.  The product library never links it.
 *
 * Parity status: UNPINNED.  The reference ships no golden vectors and its
 * WGSL cannot execute on a machine without a graphics stack, so this
 * restatement is checked only against hand-derived known answers
 * (tests/test_oracle_cpu.py) and against its own FP64 instantiation.
 *
 * Two instantiations are compiled from mpm_oracle.c:
 *   orf_*  : f32 arithmetic, fixed-point i32 grid (the reference encoding),
 *            the bit-exact parity oracle and the timed CPU baseline;
 *   ord_*  : f64 arithmetic, f64 grid without fixed-point quantisation,
 *            used only to state the error of the f32 paths.
 */
#ifndef MPM_ORACLE_H
#define MPM_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Size of the reference uniform block (GpuUniformsBufferManager.ts:17). */
#define OR_UNIFORMS_BYTES 37376u

/* Extension parameters: the constants the reference hard-codes in WGSL,
 * made per-scene.  Defaults (or_default_ext) are the reference values. */
typedef struct OrExt {
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
    uint32_t boundary_mode;      /* 0 = reference particle reflect; 1 = + grid sticky ground / slip walls */
    float restitution;           /* integrateParticles.wgsl:34: -0.5 */
    uint32_t bc_cells;           /* boundary_mode 1: width of the grid boundary layer, cells */
    uint32_t ground_axis;        /* boundary_mode 1: axis of the sticky ground plane (at grid min) */
    float collider_margin;       /* colliderPrelude.wgsl:158: 0.05 */
    float collider_surface_margin; /* colliderPrelude.wgsl:297,351: 0.05 */
    float collider_threshold;    /* colliderPrelude.wgsl:330: 0.05 */
    float collider_friction;     /* colliderPrelude.wgsl:308: 0.1 */
    float collider_vel_scale;    /* colliderPrelude.wgsl:294: 0.2 */
    float pbmpm_blend;           /* pbmpm.wgsl:26: 0.95 */
    float pbmpm_volume_exponent; /* pbmpm.wgsl:23: -0.3333333 */
    uint32_t return_map;         /* 0: applyPlasticity (plasticityOps.wgsl:7-48); 1: SVD clamp (library option) */
} OrExt;

/* 192-byte particle record, byte-for-byte the reference ParticleData
 * (shaderPrelude/mpmOps.wgsl:1-12; GpuMpmBufferManager.ts:24). */
typedef struct OrParticle {
    float pos[3]; float hom;
    float vel[3]; float mass;
    float Fe[12];   /* mat3x3f: 3 columns of vec3f padded to 16 bytes */
    float Fp[12];
    float dxp[3]; float pad;
    float D[12];
} OrParticle;

/* FP64 particle state for the ord_* instantiation (no padding). */
typedef struct OrParticleD {
    double pos[3], vel[3], mass;
    double Fe[9], Fp[9];   /* column-major: m[c*3 + r] */
    double dxp[3], D[9];
} OrParticleD;

/* Collider description: the reference packed u32 buffer
 * (GpuColliderBufferManager.ts:96-126,211-219) and 32-byte BVH nodes
 * (colliderPrelude.wgsl:6-11). */
typedef struct OrCollider {
    const uint32_t* data;   /* [reordered indices | vertices f32x3 | ...] */
    uint32_t data_words;
    const uint32_t* nodes;  /* 8 words per node */
    uint32_t n_nodes;
} OrCollider;

typedef struct OrCtx OrCtx;

/* status bits (sticky across calls) */
#define OR_STATUS_BLOCK_OVERFLOW   0x1u  /* more blocks than max_blocks (reference drops them) */
#define OR_STATUS_HASH_PROBE_FAIL  0x2u  /* insert or lookup ran out of probes */
#define OR_STATUS_UNBINNED         0x4u  /* a particle's own block was not allocated: the
                                            reference would read stale sorted indices */
#define OR_STATUS_BVH_STACK        0x8u  /* BVH traversal dropped children (stack full) */

void or_default_ext(OrExt* ext);

/* f32 instantiation */
OrCtx* orf_create(uint32_t hash_size, uint32_t max_blocks, uint32_t max_particles);
void orf_destroy(OrCtx* c);
uint32_t orf_status(const OrCtx* c);
void orf_set_threads(int n);
/* One substep (method 0 explicit, 1 PBMPM).  `stop_after` = 0 full step,
 * 1 stop after the first P2G (explicit) / first PBMPM P2G iteration. */
int orf_step(OrCtx* c, const uint8_t* uniforms, const OrExt* ext,
             OrParticle* particles, uint32_t n, const OrCollider* col,
             int method, int stop_after);
/* Dense copy of the current grid, [res_z][res_y][res_x][4] i32
 * (mass, momentum x, y, z); cells of unallocated blocks are 0. */
int orf_dense_grid(const OrCtx* c, const uint8_t* uniforms, int32_t* out);
uint32_t orf_n_blocks(const OrCtx* c);

/* f64 instantiation */
OrCtx* ord_create(uint32_t hash_size, uint32_t max_blocks, uint32_t max_particles);
void ord_destroy(OrCtx* c);
uint32_t ord_status(const OrCtx* c);
int ord_step(OrCtx* c, const uint8_t* uniforms, const OrExt* ext,
             OrParticleD* particles, uint32_t n, const OrCollider* col,
             int method, int stop_after);
int ord_dense_grid(const OrCtx* c, const uint8_t* uniforms, double* out);

/* Math known-answer hooks (f32 instantiation) */
uint32_t or_hash3(uint32_t x, uint32_t y, uint32_t z);
float or_expf(float x);
float or_powf(float x, float y);
int32_t or_f2i(float x);
void orf_inverse(const float* m9, float* out9);
void orf_polar(const float* m9, float* out9);
float orf_det(const float* m9);
void orf_plasticity(const OrExt* ext, float* Fe9, float* Fp9);

/* BVH build, restating GpuColliderBufferManager.ts:222-350.
 * nodes_out: 8 words per node (capacity 2*n_tris+1); tri_order_out: n_tris.
 * Returns the node count. */
uint32_t or_bvh_build(const float* vertices, uint32_t n_vertices,
                      const uint32_t* indices, uint32_t n_indices,
                      uint32_t* nodes_out, uint32_t* tri_order_out);

#ifdef __cplusplus
}
#endif
#endif
