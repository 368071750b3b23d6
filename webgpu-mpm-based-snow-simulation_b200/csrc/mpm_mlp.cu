// mpm_mlp.cu -- learned snow plasticity: the deferred plasticity pass
// (exact, pair collection, or the BF16 tensor-core surrogate with its exact
// fallback and audit) and the network's own training kernels.
//
// Network: 12 -> 64 -> 64 -> 64 -> 11, SiLU on the hidden layers, BF16
// weights and activations, FP32 accumulation in tensor memory (tcgen05.mma,
// M = 128 rows per tile, one row per particle or training pair).  Parameters
// are kept as FP32 masters, packed [W1 64x12 | b1 | W2 64x64 | b2 | W3 64x64 |
// b3 | W4 11x64 | b4], W row-major [out][in]; every kernel rounds them to BF16
// into its shared-memory operand layout (mpm_tc.cuh).
//
// The surrogate stands in for applyPlasticity (plasticityOps.wgsl:7-48, the
// exact return map of mpm_plast.cuh).  A particle takes the network's answer
// only if it is inside the trained domain, the uncertainty head is below its
// threshold and the determinant check holds (ln det Fp' recomputed from the
// predicted Fe' agrees with the predicted ln J_p); otherwise, and for a
// deterministic audited sample, the exact map runs in the same thread.
#include <cuda_bf16.h>

#include "mpm_engine.cuh"
#include "mpm_math.cuh"
#include "mpm_mlp.cuh"
#include "mpm_plast.cuh"
#include "mpm_tc.cuh"

namespace mpm {

using namespace mlp;

namespace {

constexpr uint32_t WAIT_LIMIT = 1u << 22;   // mbarrier polls before a pass gives up

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);   // one conversion for two values, a in the low half
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void st_bf16(uint8_t* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}
// 8 consecutive K elements of row r of an R-row K-major operand
__device__ __forceinline__ void st_row8(uint8_t* base, uint32_t r, uint32_t k0, uint32_t R, const float* v) {
    uint4 q = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    *reinterpret_cast<uint4*>(base + tc::kmaj(r, k0, R)) = q;
}

// sigmoid(z) = (1 + tanh(z / 2)) / 2 with the hardware tanh (one MUFU
// operation per element instead of an exponential and a reciprocal)
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float silu_grad(float z) {
    float s = sigmoid(z);
    return s + z * s * (1.0f - s);
}

// W[out][in] (fp32, global) -> bf16 operand [rows = out (padded R) x K = in (padded KP)]
__device__ void load_w(uint8_t* dst, const float* W, int out, int in, int R, int KP) {
    for (int i = threadIdx.x; i < R * KP; i += blockDim.x) {
        int n = i / KP, k = i - n * KP;
        float v = (n < out && k < in) ? __ldg(W + n * in + k) : 0.0f;
        st_bf16(dst, tc::kmaj(n, k, R), v);
    }
}
// transposed: W^T [rows = in (padded R) x K = out (padded KP)]
__device__ void load_wt(uint8_t* dst, const float* W, int out, int in, int R, int KP) {
    for (int i = threadIdx.x; i < R * KP; i += blockDim.x) {
        int n = i / KP, k = i - n * KP;   // n = input index, k = output index
        float v = (n < in && k < out) ? __ldg(W + k * in + n) : 0.0f;
        st_bf16(dst, tc::kmaj(n, k, R), v);
    }
}

// ---------------------------------------------------------------------
// forward of one 128-row tile (inference layout)
// ---------------------------------------------------------------------
struct alignas(1024) InfSmem {
    uint8_t w1[HID * K1 * 2];
    uint8_t w2[HID * HID * 2];
    uint8_t w3[HID * HID * 2];
    uint8_t w4[N4 * HID * 2];
    uint8_t a[ROWS * HID * 2];
    float b1[HID], b2[HID], b3[HID], b4[N4];
    unsigned long long mbar;
    uint32_t tmem_slot;
};

__device__ void load_inf_weights(InfSmem& sm, const float* P) {
    load_w(sm.w1, P + OW1, HID, IN, HID, K1);
    load_w(sm.w2, P + OW2, HID, HID, HID, HID);
    load_w(sm.w3, P + OW3, HID, HID, HID, HID);
    load_w(sm.w4, P + OW4, OUT, HID, N4, HID);
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        sm.b1[i] = P[OB1 + i];
        sm.b2[i] = P[OB2 + i];
        sm.b3[i] = P[OB3 + i];
    }
    for (int i = threadIdx.x; i < N4; i += blockDim.x) sm.b4[i] = i < OUT ? P[OB4 + i] : 0.0f;
}

// Issues the K/16 MMA steps of one layer from thread 0 and waits for them.
// Returns false (on every thread) when the wait ran out.
__device__ bool run_layer(uint32_t mbar, uint32_t& phase, uint32_t tmem_d, uint32_t a_saddr, uint32_t a_rows,
                          uint32_t b_saddr, uint32_t b_rows, int M, int N, int K, bool accumulate_first) {
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc::fence_after_sync();
        const uint32_t a_lbo = a_rows * 16u, b_lbo = b_rows * 16u;
        for (int s = 0; s < K / 16; s++) {
            uint64_t ad = tc::sdesc(a_saddr + (uint32_t)s * 2u * a_lbo, a_lbo, 128u);
            uint64_t bd = tc::sdesc(b_saddr + (uint32_t)s * 2u * b_lbo, b_lbo, 128u);
            tc::mma_bf16(tmem_d, ad, bd, tc::idesc_bf16(M, N), (accumulate_first || s > 0) ? 1u : 0u);
        }
        tc::commit(mbar);
    }
    bool ok = tc::mbar_wait(mbar, phase, WAIT_LIMIT);
    phase ^= 1u;
    tc::fence_after_sync();
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// x: this thread's 12 features; y: the 16 output columns (11 used) with bias
__device__ bool tile_forward(InfSmem& sm, uint32_t tmem, uint32_t& phase, const float* x, float* y) {
    const uint32_t r = threadIdx.x, warp = threadIdx.x >> 5;
    const uint32_t mbar = tc::smem_addr(&sm.mbar);
    float v[8];
    for (int i = 0; i < 8; i++) v[i] = x[i];
    st_row8(sm.a, r, 0, ROWS, v);
    for (int i = 0; i < 8; i++) v[i] = i < 4 ? x[8 + i] : 0.0f;
    st_row8(sm.a, r, 8, ROWS, v);
    const uint32_t a_s = tc::smem_addr(sm.a);
    if (!run_layer(mbar, phase, tmem, a_s, ROWS, tc::smem_addr(sm.w1), HID, ROWS, HID, K1, false)) return false;
    const uint8_t* wl[2] = {sm.w2, sm.w3};
    const float* bl[3] = {sm.b1, sm.b2, sm.b3};
    for (int layer = 0; layer < 3; layer++) {
        // hidden activation of the layer just computed -> next A operand
        for (int c0 = 0; c0 < HID; c0 += 32) {
            float z[32];
            tc::tmem_ld32(tc::tmem_addr(tmem, warp * 32u, (uint32_t)c0), z);
            for (int h = 0; h < 4; h++) {
                for (int i = 0; i < 8; i++) v[i] = silu(z[h * 8 + i] + bl[layer][c0 + h * 8 + i]);
                st_row8(sm.a, r, (uint32_t)(c0 + h * 8), ROWS, v);
            }
        }
        if (layer < 2) {
            if (!run_layer(mbar, phase, tmem, a_s, ROWS, tc::smem_addr(wl[layer]), HID, ROWS, HID, HID, false))
                return false;
        } else {
            if (!run_layer(mbar, phase, tmem, a_s, ROWS, tc::smem_addr(sm.w4), N4, ROWS, N4, HID, false))
                return false;
        }
    }
    tc::tmem_ld16(tc::tmem_addr(tmem, warp * 32u, 0u), y);
    for (int i = 0; i < N4; i++) y[i] += sm.b4[i];
    return true;
}

__device__ __forceinline__ void warp_count(unsigned long long* dst, bool pred) {
    unsigned b = __ballot_sync(__activemask(), pred);
    if (b && (threadIdx.x & 31) == (uint32_t)(__ffs(__activemask()) - 1)) atomicAdd(dst, (unsigned long long)__popc(b));
}

// Fe and Fp of work slot t (record words 2..7; word q of slot t at w[q * n + t])
__device__ __forceinline__ void load_fe_fp(const float4* w, size_t n, uint32_t t, float* Fe, float* Fp) {
    const float4* rec = w + t;
    float4 q2 = rec[2 * n], q3 = rec[3 * n], q4 = rec[4 * n], q5 = rec[5 * n], q6 = rec[6 * n], q7 = rec[7 * n];
    Fe[0] = q2.x; Fe[1] = q2.y; Fe[2] = q2.z; Fe[3] = q3.x; Fe[4] = q3.y; Fe[5] = q3.z;
    Fe[6] = q4.x; Fe[7] = q4.y; Fe[8] = q4.z;
    Fp[0] = q5.x; Fp[1] = q5.y; Fp[2] = q5.z; Fp[3] = q6.x; Fp[4] = q6.y; Fp[5] = q6.z;
    Fp[6] = q7.x; Fp[7] = q7.y; Fp[8] = q7.z;
}
__device__ __forceinline__ void store_fe_fp(float4* w, size_t n, uint32_t t, const float* Fe, const float* Fp) {
    float4* rec = w + t;
    rec[2 * n] = make_float4(Fe[0], Fe[1], Fe[2], 0.f);
    rec[3 * n] = make_float4(Fe[3], Fe[4], Fe[5], 0.f);
    rec[4 * n] = make_float4(Fe[6], Fe[7], Fe[8], 0.f);
    rec[5 * n] = make_float4(Fp[0], Fp[1], Fp[2], 0.f);
    rec[6 * n] = make_float4(Fp[3], Fp[4], Fp[5], 0.f);
    rec[7 * n] = make_float4(Fp[6], Fp[7], Fp[8], 0.f);
}

__device__ __forceinline__ uint32_t find_scene_p(const Ctx& c, uint32_t p) {
    uint32_t lo = 0, hi = c.n_scenes;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&c.scene_first[mid]) <= p) lo = mid; else hi = mid;
    }
    return lo;
}

// network targets of an exact result
__device__ __forceinline__ void mlp_targets(const float* Fe, const float* Fp, const float* Fe2, const float* Fp2,
                                            float* t) {
    for (int i = 0; i < 9; i++) t[i] = (Fe2[i] - Fe[i]) * MLP_T_F;
    t[9] = (logf(det3(Fp2)) - logf(det3(Fp))) * MLP_T_F;
}

}  // namespace

// ---------------------------------------------------------------------
// deferred plasticity pass over the particles the strain-bound check listed
// ---------------------------------------------------------------------
// exact return map (MODE = PLAST_EXACT) or exact map plus training-pair
// collection (MODE = PLAST_COLLECT), one thread per listed particle
template <int MODE>
__global__ void __launch_bounds__(128) k_plasticity_exact(Ctx c, PlastCtx pc) {
    const uint32_t count = c.counters->n_plast;
    const uint32_t step = c.counters->step;
    {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
            // the listed work slot; sampling and scene lookup use the caller's particle index
            const uint32_t slot = c.plast_list[i];
            const uint32_t pid = c.ids_out[slot];
            const SceneDev& S = c.scenes[find_scene_p(c, pid)];
            float Fe[9], Fp[9], x[12];
            load_fe_fp(c.work_out, c.n_particles, slot, Fe, Fp);
            bool dom = mlp_features(Fe, Fp, S.dt, 1.0f - S.smin, x);
            warp_count(&pc.stats->candidates, true);
            warp_count(&pc.stats->fallback_domain, !dom);
            float Fe2[9], Fp2[9];
            for (int k = 0; k < 9; k++) { Fe2[k] = Fe[k]; Fp2[k] = Fp[k]; }
            plasticity_map(S.rmap, S.smin, S.smax, Fe2, Fp2);
            if (MODE == PLAST_COLLECT && dom && pc.pair_x && hash3(pid, step, 0xc011u) < pc.audit_threshold) {
                uint32_t slot = atomicAdd(pc.pair_count, 1u);
                if (slot < pc.pair_cap) {
                    float t[10];
                    mlp_targets(Fe, Fp, Fe2, Fp2, t);
                    for (int k = 0; k < IN; k++) pc.pair_x[(size_t)slot * IN + k] = x[k];
                    for (int k = 0; k < 10; k++) pc.pair_t[(size_t)slot * 10 + k] = t[k];
                }
            }
            store_fe_fp(c.work_out, c.n_particles, slot, Fe2, Fp2);
        }
    }
}

// learned surrogate with gating, audit and exact fallback, 128 particles per tile
__global__ void __launch_bounds__(128, MLP_CTAS_PER_SM) k_plasticity_learned(Ctx c, PlastCtx pc) {
    const uint32_t count = c.counters->n_plast;
    __shared__ InfSmem sm;
    const uint32_t warp = threadIdx.x >> 5;
    if (warp == 0) tc::tmem_alloc(&sm.tmem_slot, 64);
    if (threadIdx.x == 0) tc::mbar_init(tc::smem_addr(&sm.mbar), 1);
    load_inf_weights(sm, pc.params);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = sm.tmem_slot;
    const uint32_t step = c.counters->step;
    uint32_t phase = 0;
    const uint32_t n_tiles = (count + ROWS - 1) / ROWS;
    bool alive = true;
    for (uint32_t tile = blockIdx.x; tile < n_tiles && alive; tile += gridDim.x) {
        const uint32_t idx = tile * ROWS + threadIdx.x;
        const bool valid = idx < count;
        const uint32_t slot = valid ? c.plast_list[idx] : 0u;
        const uint32_t pid = valid ? c.ids_out[slot] : 0u;
        float Fe[9], Fp[9], x[12] = {0.f};
        bool dom = false;
        float smin = 0.f, smax = 0.f;
        uint32_t rmap = 0u;
        if (valid) {
            const SceneDev& S = c.scenes[find_scene_p(c, pid)];
            smin = S.smin;
            smax = S.smax;
            rmap = S.rmap;
            load_fe_fp(c.work_out, c.n_particles, slot, Fe, Fp);
            dom = mlp_features(Fe, Fp, S.dt, 1.0f - S.smin, x);
            if (!dom)
                for (int k = 0; k < IN; k++) x[k] = 0.f;
        }
        float y[N4];
        if (!tile_forward(sm, tmem, phase, x, y)) {
            alive = false;
            if (threadIdx.x == 0) atomicOr(&c.counters->status, ST_MLP_TIMEOUT);
            break;
        }
        if (!valid) continue;
        // decode: Fe' = Fe + y/100, Fp' = Fe'^-1 (Fe Fp)
        float Fn[9], Fni[9], F[9], Fpn[9];
        for (int k = 0; k < 9; k++) Fn[k] = Fe[k] + y[k] * MLP_T_FINV;
        inv3(Fn, Fni);
        mul3(Fe, Fp, F);
        mul3(Fni, F, Fpn);
        float jn = det3(Fn), jp = det3(Fp), jpn = det3(Fpn);
        bool det_ok = jn > 0.f && jpn > 0.f &&
                      fabsf((logf(jpn) - logf(jp)) - y[9] * MLP_T_FINV) <= pc.det_threshold;
        bool unc_ok = y[10] <= pc.unc_threshold;
        bool use = dom && det_ok && unc_ok;
        bool audit = use && hash3(pid, step, 0x5eedu) < pc.audit_threshold;
        warp_count(&pc.stats->candidates, true);
        warp_count(&pc.stats->fallback_domain, !dom);
        warp_count(&pc.stats->fallback_uncertain, dom && !unc_ok);
        warp_count(&pc.stats->fallback_det, dom && unc_ok && !det_ok);
        warp_count(&pc.stats->learned, use && !audit);
        warp_count(&pc.stats->audited, audit);
        if (!use || audit) {
            float Fe2[9], Fp2[9];
            for (int k = 0; k < 9; k++) { Fe2[k] = Fe[k]; Fp2[k] = Fp[k]; }
            plasticity_map(rmap, smin, smax, Fe2, Fp2);
            if (audit) {
                float err = 0.f;
                for (int k = 0; k < 9; k++) err = fmaxf(err, fabsf(Fn[k] - Fe2[k]));
                atomicMax(&pc.stats->audit_max_err_bits, __float_as_uint(err));
                atomicAdd(&pc.stats->audit_err_sum, (double)err);
            }
            store_fe_fp(c.work_out, c.n_particles, slot, Fe2, Fp2);
        } else {
            store_fe_fp(c.work_out, c.n_particles, slot, Fn, Fpn);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

// raw network on device arrays: x [n][12] -> y [n][11]
__global__ void __launch_bounds__(128, MLP_CTAS_PER_SM) k_mlp_forward(const float* P, const float* xin, uint32_t n, float* yout,
                                                     uint32_t* err) {
    __shared__ InfSmem sm;
    const uint32_t warp = threadIdx.x >> 5;
    if (warp == 0) tc::tmem_alloc(&sm.tmem_slot, 64);
    if (threadIdx.x == 0) tc::mbar_init(tc::smem_addr(&sm.mbar), 1);
    load_inf_weights(sm, P);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = sm.tmem_slot;
    uint32_t phase = 0;
    const uint32_t n_tiles = (n + ROWS - 1) / ROWS;
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        uint32_t idx = tile * ROWS + threadIdx.x;
        float x[12] = {0.f};
        if (idx < n)
            for (int k = 0; k < IN; k++) x[k] = xin[(size_t)idx * IN + k];
        float y[N4];
        if (!tile_forward(sm, tmem, phase, x, y)) {
            if (threadIdx.x == 0) atomicOr(err, 1u);
            break;
        }
        if (idx < n)
            for (int k = 0; k < OUT; k++) yout[(size_t)idx * OUT + k] = y[k];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------------
// training: forward + backward of 128-pair tiles, gradients accumulated in
// tensor memory over a CTA's tiles, then added to the global gradient.
// Loss of a batch of B pairs: (1/B) sum_b [ sum_{i<10} (y_i - t_i)^2
//                                           + lambda (y_10 - e_b)^2 ],
// e_b = |y[0..9] - t| (held constant).  All MMA operands are BF16 (the
// output-gradients are rounded to BF16 before their products).
// ---------------------------------------------------------------------
struct alignas(1024) TrainSmem {
    uint8_t w1[HID * K1 * 2], w2[HID * HID * 2], w3[HID * HID * 2], w4[N4 * HID * 2];
    uint8_t w2t[HID * HID * 2], w3t[HID * HID * 2], w4t[HID * N4 * 2];
    uint8_t a0[ROWS * K1 * 2], a1[ROWS * HID * 2], a2[ROWS * HID * 2], a3[ROWS * HID * 2];
    uint8_t a0t[K1 * ROWS * 2], a1t[HID * ROWS * 2], a2t[HID * ROWS * 2], a3t[HID * ROWS * 2];
    uint8_t g[ROWS * HID * 2], gt[HID * ROWS * 2];
    uint8_t g4[ROWS * N4 * 2], g4t[HID * ROWS * 2];
    float b1[HID], b2[HID], b3[HID], b4[N4];
    float db1[HID], db2[HID], db3[HID], db4[N4];
    float loss[4];
    unsigned long long mbar;
    uint32_t tmem_slot;
};

// tensor-memory columns of the training kernel
constexpr uint32_t TC_Z1 = 0, TC_Z2 = 64, TC_Z3 = 128, TC_Y = 192, TC_DW1 = 208, TC_DX = 224, TC_DW2 = 288,
                   TC_DW3 = 352, TC_DW4 = 416, TC_COLS = 512;

__global__ void __launch_bounds__(128) k_mlp_train(const float* P, const float* xin, const float* tin,
                                                   const uint32_t* idx_list, uint32_t n, float inv_batch,
                                                   float unc_weight, float* grad, float* loss_out, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t train_smem_raw[];
    const uint32_t pad = (1024u - (tc::smem_addr(train_smem_raw) & 1023u)) & 1023u;
    TrainSmem& sm = *reinterpret_cast<TrainSmem*>(train_smem_raw + pad);
    const uint32_t r = threadIdx.x, warp = threadIdx.x >> 5;
    if (warp == 0) tc::tmem_alloc(&sm.tmem_slot, TC_COLS);
    if (threadIdx.x == 0) tc::mbar_init(tc::smem_addr(&sm.mbar), 1);
    load_w(sm.w1, P + OW1, HID, IN, HID, K1);
    load_w(sm.w2, P + OW2, HID, HID, HID, HID);
    load_w(sm.w3, P + OW3, HID, HID, HID, HID);
    load_w(sm.w4, P + OW4, OUT, HID, N4, HID);
    load_wt(sm.w2t, P + OW2, HID, HID, HID, HID);
    load_wt(sm.w3t, P + OW3, HID, HID, HID, HID);
    load_wt(sm.w4t, P + OW4, OUT, HID, HID, N4);
    for (int i = threadIdx.x; i < HID; i += blockDim.x) {
        sm.b1[i] = P[OB1 + i]; sm.b2[i] = P[OB2 + i]; sm.b3[i] = P[OB3 + i];
        sm.db1[i] = 0.f; sm.db2[i] = 0.f; sm.db3[i] = 0.f;
    }
    for (int i = threadIdx.x; i < N4; i += blockDim.x) { sm.b4[i] = i < OUT ? P[OB4 + i] : 0.f; sm.db4[i] = 0.f; }
    // rows OUT.. of the last layer's transposed output-gradient stay zero
    for (int i = threadIdx.x; i < HID * ROWS * 2 / 16; i += blockDim.x) reinterpret_cast<uint4*>(sm.g4t)[i] = make_uint4(0, 0, 0, 0);
    if (threadIdx.x == 0) sm.loss[0] = 0.f;
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = sm.tmem_slot;
    const uint32_t mbar = tc::smem_addr(&sm.mbar);
    uint32_t phase = 0;
    float my_loss = 0.f;
    bool first = true, alive = true;
    const uint32_t n_tiles = (n + ROWS - 1) / ROWS;
    const uint32_t lane_base = warp * 32u;
    for (uint32_t tile = blockIdx.x; tile < n_tiles && alive; tile += gridDim.x) {
        const uint32_t i = tile * ROWS + r;
        const bool valid = i < n;
        const uint32_t src = valid ? (idx_list ? idx_list[i] : i) : 0u;
        float x[K1], t[10];
        for (int k = 0; k < K1; k++) x[k] = (valid && k < IN) ? xin[(size_t)src * IN + k] : 0.f;
        for (int k = 0; k < 10; k++) t[k] = valid ? tin[(size_t)src * 10 + k] : 0.f;
        // ---- forward
        st_row8(sm.a0, r, 0, ROWS, x);
        st_row8(sm.a0, r, 8, ROWS, x + 8);
        for (int k = 0; k < K1; k++) st_bf16(sm.a0t, tc::kmaj(k, r, K1), x[k]);
        if (!run_layer(mbar, phase, tm + TC_Z1, tc::smem_addr(sm.a0), ROWS, tc::smem_addr(sm.w1), HID, ROWS, HID, K1,
                       false)) { alive = false; break; }
        uint8_t* acts[3] = {sm.a1, sm.a2, sm.a3};
        uint8_t* actt[3] = {sm.a1t, sm.a2t, sm.a3t};
        const float* bl[3] = {sm.b1, sm.b2, sm.b3};
        const uint32_t zc[3] = {TC_Z1, TC_Z2, TC_Z3};
        for (int l = 0; l < 3 && alive; l++) {
            for (int c0 = 0; c0 < HID; c0 += 16) {
                float z[16], h[16];
                tc::tmem_ld16(tc::tmem_addr(tm, lane_base, zc[l] + c0), z);
                for (int k = 0; k < 16; k++) h[k] = silu(z[k] + bl[l][c0 + k]);
                st_row8(acts[l], r, c0, ROWS, h);
                st_row8(acts[l], r, c0 + 8, ROWS, h + 8);
                for (int k = 0; k < 16; k++) st_bf16(actt[l], tc::kmaj(c0 + k, r, HID), h[k]);
            }
            if (l < 2) {
                if (!run_layer(mbar, phase, tm + zc[l + 1], tc::smem_addr(acts[l]), ROWS,
                               tc::smem_addr(l == 0 ? sm.w2 : sm.w3), HID, ROWS, HID, HID, false)) alive = false;
            } else {
                if (!run_layer(mbar, phase, tm + TC_Y, tc::smem_addr(acts[l]), ROWS, tc::smem_addr(sm.w4), N4, ROWS,
                               N4, HID, false)) alive = false;
            }
        }
        if (!alive) break;
        // ---- loss and output gradient
        float y[N4], g4v[N4];
        tc::tmem_ld16(tc::tmem_addr(tm, lane_base, TC_Y), y);
        float se = 0.f;
        for (int k = 0; k < N4; k++) y[k] += sm.b4[k];
        for (int k = 0; k < 10; k++) se += (y[k] - t[k]) * (y[k] - t[k]);
        float e = sqrtf(se);
        for (int k = 0; k < N4; k++) g4v[k] = 0.f;
        if (valid) {
            for (int k = 0; k < 10; k++) g4v[k] = 2.f * inv_batch * (y[k] - t[k]);
            g4v[10] = 2.f * inv_batch * unc_weight * (y[10] - e);
            my_loss += inv_batch * (se + unc_weight * (y[10] - e) * (y[10] - e));
        }
        st_row8(sm.g4, r, 0, ROWS, g4v);
        st_row8(sm.g4, r, 8, ROWS, g4v + 8);
        for (int k = 0; k < N4; k++) {
            st_bf16(sm.g4t, tc::kmaj(k, r, HID), g4v[k]);
            atomicAdd(&sm.db4[k], g4v[k]);
        }
        // dW4 += g4^T a3 (M = 64 padded outputs, N = 64, K = 128 pairs); dX3 = g4 W4 (M = 128, N = 64, K = 16)
        tc::fence_smem_async();
        tc::fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after_sync();
            for (int s = 0; s < ROWS / 16; s++) {
                uint64_t ad = tc::sdesc(tc::smem_addr(sm.g4t) + s * 2u * (HID * 16u), HID * 16u, 128u);
                uint64_t bd = tc::sdesc(tc::smem_addr(sm.a3t) + s * 2u * (HID * 16u), HID * 16u, 128u);
                tc::mma_bf16(tm + TC_DW4, ad, bd, tc::idesc_bf16(64, HID), (!first || s > 0) ? 1u : 0u);
            }
            uint64_t ad = tc::sdesc(tc::smem_addr(sm.g4), ROWS * 16u, 128u);
            uint64_t bd = tc::sdesc(tc::smem_addr(sm.w4t), HID * 16u, 128u);
            tc::mma_bf16(tm + TC_DX, ad, bd, tc::idesc_bf16(ROWS, HID), 0u);
            tc::commit(mbar);
        }
        {
            bool ok = tc::mbar_wait(mbar, phase, WAIT_LIMIT);
            phase ^= 1u;
            tc::fence_after_sync();
            if (!__syncthreads_and(ok ? 1 : 0)) { alive = false; break; }
        }
        // hidden layers 3, 2, 1
        const uint8_t* wts[3] = {sm.w2t, sm.w3t, nullptr};   // W_{l+1}^T for dX_l (l = 1, 2)
        for (int l = 2; l >= 0 && alive; l--) {
            float gv[HID];
            for (int c0 = 0; c0 < HID; c0 += 16) {
                float dx[16], z[16];
                tc::tmem_ld16(tc::tmem_addr(tm, lane_base, TC_DX + c0), dx);
                tc::tmem_ld16(tc::tmem_addr(tm, lane_base, zc[l] + c0), z);
                for (int k = 0; k < 16; k++) gv[c0 + k] = valid ? dx[k] * silu_grad(z[k] + bl[l][c0 + k]) : 0.f;
            }
            for (int c0 = 0; c0 < HID; c0 += 8) st_row8(sm.g, r, c0, ROWS, gv + c0);
            float* dbl = l == 0 ? sm.db1 : (l == 1 ? sm.db2 : sm.db3);
            for (int k = 0; k < HID; k++) {
                st_bf16(sm.gt, tc::kmaj(k, r, HID), gv[k]);
                // warp-reduce the bias gradient before one shared atomic per warp
                float s = gv[k];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if ((threadIdx.x & 31) == 0) atomicAdd(&dbl[k], s);
            }
            tc::fence_smem_async();
            tc::fence_before_sync();
            __syncthreads();
            if (threadIdx.x == 0) {
                tc::fence_after_sync();
                const uint8_t* prev_t = l == 0 ? sm.a0t : (l == 1 ? sm.a1t : sm.a2t);
                const uint32_t prev_rows = l == 0 ? K1 : HID;
                const uint32_t dw = l == 0 ? TC_DW1 : (l == 1 ? TC_DW2 : TC_DW3);
                for (int s = 0; s < ROWS / 16; s++) {
                    uint64_t ad = tc::sdesc(tc::smem_addr(sm.gt) + s * 2u * (HID * 16u), HID * 16u, 128u);
                    uint64_t bd = tc::sdesc(tc::smem_addr(prev_t) + s * 2u * (prev_rows * 16u), prev_rows * 16u, 128u);
                    tc::mma_bf16(tm + dw, ad, bd, tc::idesc_bf16(64, (int)prev_rows), (!first || s > 0) ? 1u : 0u);
                }
                if (l > 0) {
                    const uint8_t* wt = wts[l - 1];
                    for (int s = 0; s < HID / 16; s++) {
                        uint64_t ad = tc::sdesc(tc::smem_addr(sm.g) + s * 2u * (ROWS * 16u), ROWS * 16u, 128u);
                        uint64_t bd = tc::sdesc(tc::smem_addr(wt) + s * 2u * (HID * 16u), HID * 16u, 128u);
                        tc::mma_bf16(tm + TC_DX, ad, bd, tc::idesc_bf16(ROWS, HID), s > 0 ? 1u : 0u);
                    }
                }
                tc::commit(mbar);
            }
            bool ok = tc::mbar_wait(mbar, phase, WAIT_LIMIT);
            phase ^= 1u;
            tc::fence_after_sync();
            if (!__syncthreads_and(ok ? 1 : 0)) alive = false;
        }
        first = false;
    }
    if (!alive && threadIdx.x == 0) atomicOr(err, 1u);
    // ---- gradients out: weights from tensor memory (M = 64 layout), biases from shared memory
    if (alive && !first) {
        const uint32_t dwc[4] = {TC_DW1, TC_DW2, TC_DW3, TC_DW4};
        const int in_dim[4] = {IN, HID, HID, HID}, out_dim[4] = {HID, HID, HID, OUT};
        const int ncols[4] = {K1, HID, HID, HID};
        const int ow[4] = {OW1, OW2, OW3, OW4};
        const uint32_t lane = threadIdx.x & 31u;
        for (int l = 0; l < 4; l++) {
            for (int c0 = 0; c0 < ncols[l]; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tc::tmem_addr(tm, lane_base, dwc[l] + c0), v);
                int o = (int)(warp * 16u + lane);
                if (lane < 16u && o < out_dim[l])
                    for (int k = 0; k < 16; k++)
                        if (c0 + k < in_dim[l]) atomicAdd(&grad[ow[l] + o * in_dim[l] + c0 + k], v[k]);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) my_loss += __shfl_xor_sync(0xffffffffu, my_loss, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sm.loss[0], my_loss);
    tc::fence_before_sync();
    __syncthreads();
    if (alive && !first) {
        for (int i = threadIdx.x; i < HID; i += blockDim.x) {
            atomicAdd(&grad[OB1 + i], sm.db1[i]);
            atomicAdd(&grad[OB2 + i], sm.db2[i]);
            atomicAdd(&grad[OB3 + i], sm.db3[i]);
        }
        for (int i = threadIdx.x; i < OUT; i += blockDim.x) atomicAdd(&grad[OB4 + i], sm.db4[i]);
        if (threadIdx.x == 0) atomicAdd(loss_out, sm.loss[0]);
    }
    if (warp == 0) tc::tmem_dealloc(tm, TC_COLS);
}

// Adam on the FP32 master parameters
__global__ void k_adam(float* P, float* m, float* v, const float* g, uint32_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1.f - b1) * gi;
        float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// ---------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------
cudaError_t launch_plasticity(int mode, const Ctx& c, const PlastCtx& pc, int grid, cudaStream_t s) {
    switch (mode) {
        case PLAST_EXACT: k_plasticity_exact<PLAST_EXACT><<<grid, 128, 0, s>>>(c, pc); break;
        case PLAST_COLLECT: k_plasticity_exact<PLAST_COLLECT><<<grid, 128, 0, s>>>(c, pc); break;
        case PLAST_LEARNED: k_plasticity_learned<<<grid, 128, 0, s>>>(c, pc); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const float* P, const float* x, uint32_t n, float* y, uint32_t* err, int grid,
                               cudaStream_t s) {
    k_mlp_forward<<<grid, 128, 0, s>>>(P, x, n, y, err);
    return cudaGetLastError();
}

size_t mlp_train_smem() { return sizeof(TrainSmem) + 1024; }

cudaError_t configure_mlp_kernels() {
    return cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_train_smem());
}

cudaError_t launch_mlp_train(const float* P, const float* x, const float* t, const uint32_t* idx, uint32_t n,
                             float inv_batch, float unc_weight, float* grad, float* loss, uint32_t* err, int grid,
                             cudaStream_t s) {
    k_mlp_train<<<grid, 128, mlp_train_smem(), s>>>(P, x, t, idx, n, inv_batch, unc_weight, grad, loss, err);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* P, float* m, float* v, const float* g, uint32_t n, float lr, int step,
                        cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    k_adam<<<(n + 255) / 256, 256, 0, s>>>(P, m, v, g, n, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace mpm
