// mpm_tc.cuh -- fifth-generation tensor core (tcgen05) helpers for sm_100a,
// written as inline PTX: tensor-memory allocation, shared-memory matrix
// descriptors, the BF16 x BF16 -> F32 MMA, commit to an mbarrier, bounded
// mbarrier waits, and tensor-memory loads.
//
// Operand layout (both A and B "K-major", no swizzle): an R x K bf16 matrix
// is stored as K/8 planes of R rows x 16 bytes; element (r, k) sits at byte
//   (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so each 8 x 8 core matrix is 128 contiguous bytes.  In the descriptor the
// leading byte offset (LBO) is the distance between the two K halves of one
// K = 16 step (R * 16 bytes) and the stride byte offset (SBO) the distance
// between 8-row groups (128 bytes).  One K = 16 step later starts 2 planes on.
//
// Accumulators: for M = 128 row i of D is tensor-memory lane i; for M = 64
// rows 16w .. 16w+15 sit in lanes 32w .. 32w+15 (w = 0..3).  Column j of D is
// column base + j.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpm {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R-row K-major operand
__host__ __device__ constexpr uint32_t kmaj(uint32_t r, uint32_t k, uint32_t R) {
    return (k >> 3) * (R * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// shared-memory matrix descriptor (sm_100 format: version 1, no swizzle)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// instruction descriptor, kind::f16: D f32, A and B bf16, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// arrive on the mbarrier once every MMA this thread issued has completed
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// waits for the phase with the given parity; false after `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// allocation by one full warp; the column base is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive f32 columns of this thread's lane (32x32b shape), waited on
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive f32 columns as two loads in flight and one wait; the wait
// names the destination registers, so no use of them moves ahead of it
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
#pragma unroll
    for (int h = 0; h < 2; h++)
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(r[16 * h + 0]), "=r"(r[16 * h + 1]), "=r"(r[16 * h + 2]), "=r"(r[16 * h + 3]),
              "=r"(r[16 * h + 4]), "=r"(r[16 * h + 5]), "=r"(r[16 * h + 6]), "=r"(r[16 * h + 7]),
              "=r"(r[16 * h + 8]), "=r"(r[16 * h + 9]), "=r"(r[16 * h + 10]), "=r"(r[16 * h + 11]),
              "=r"(r[16 * h + 12]), "=r"(r[16 * h + 13]), "=r"(r[16 * h + 14]), "=r"(r[16 * h + 15])
            : "r"(taddr + 16u * (uint32_t)h)
            : "memory");
#pragma unroll
    for (int h = 0; h < 2; h++)
        asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                     : "+r"(r[16 * h + 0]), "+r"(r[16 * h + 1]), "+r"(r[16 * h + 2]), "+r"(r[16 * h + 3]),
                       "+r"(r[16 * h + 4]), "+r"(r[16 * h + 5]), "+r"(r[16 * h + 6]), "+r"(r[16 * h + 7]),
                       "+r"(r[16 * h + 8]), "+r"(r[16 * h + 9]), "+r"(r[16 * h + 10]), "+r"(r[16 * h + 11]),
                       "+r"(r[16 * h + 12]), "+r"(r[16 * h + 13]), "+r"(r[16 * h + 14]), "+r"(r[16 * h + 15])
                     :
                     : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, uint32_t lane, uint32_t col) {
    return base + (lane << 16) + col;
}

}  // namespace tc
}  // namespace mpm
