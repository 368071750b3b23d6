// mpm_mlp.cuh -- shapes, parameter packing and pass context of the learned
// plasticity network (kernels in mpm_mlp.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_engine.cuh"

namespace mpm {
namespace mlp {

constexpr int IN = 12, HID = 64, OUT = 11;   // inputs, hidden width, outputs (10 + uncertainty)
constexpr int K1 = 16, N4 = 16;              // padded first-layer K and last-layer N
constexpr int ROWS = 128;                    // rows per tensor-core tile
// packed FP32 parameters, W row-major [out][in]
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
              OB3 = OW3 + HID * HID, OW4 = OB3 + HID, OB4 = OW4 + OUT * HID, NPARAM = OB4 + OUT;
static_assert(NPARAM == 9867, "parameter count");

}  // namespace mlp

// plasticity pass modes (after integrate; mode 0 keeps the exact map inline)
constexpr int PLAST_INLINE = 0, PLAST_EXACT = 1, PLAST_COLLECT = 2, PLAST_LEARNED = 3;
// resident CTAs per SM of the inference kernels (36 KB of shared memory and
// 64 tensor-memory columns each): one CTA's epilogue runs while another's MMAs do
constexpr unsigned MLP_CTAS_PER_SM = 6;

struct PlastStats {
    unsigned long long candidates;          // particles the strain-bound check did not clear
    unsigned long long learned;             // took the network's answer
    unsigned long long fallback_domain;     // outside the trained domain -> exact
    unsigned long long fallback_uncertain;  // uncertainty head above threshold -> exact
    unsigned long long fallback_det;        // determinant check failed -> exact
    unsigned long long audited;             // audited sample (exact applied, error recorded)
    double audit_err_sum;                   // sum over audited particles of max |Fe'_net - Fe'_exact|
    uint32_t audit_max_err_bits;            // max of the same, f32 bits
    uint32_t pad;
};

struct PlastCtx {
    const float* params;       // packed FP32 parameters (device)
    float unc_threshold;       // accept when the uncertainty output <= this (target units)
    float det_threshold;       // accept when |d ln J_p recomputed - predicted| <= this
    uint32_t audit_threshold;  // audit when hash3(pid, substep counter, seed) < this (fraction * 2^32)
    PlastStats* stats;
    float* pair_x;             // collection: [cap][12] inputs
    float* pair_t;             // collection: [cap][10] targets
    uint32_t* pair_count;
    uint32_t pair_cap;
};

cudaError_t launch_plasticity(int mode, const Ctx& c, const PlastCtx& pc, int grid, cudaStream_t s);
cudaError_t launch_mlp_forward(const float* P, const float* x, uint32_t n, float* y, uint32_t* err, int grid,
                               cudaStream_t s);
cudaError_t configure_mlp_kernels();
size_t mlp_train_smem();
cudaError_t launch_mlp_train(const float* P, const float* x, const float* t, const uint32_t* idx, uint32_t n,
                             float inv_batch, float unc_weight, float* grad, float* loss, uint32_t* err, int grid,
                             cudaStream_t s);
cudaError_t launch_adam(float* P, float* m, float* v, const float* g, uint32_t n, float lr, int step, cudaStream_t s);

}  // namespace mpm
