// tcgen05.cuh -- 5th-generation tensor cores (tcgen05, sm_100a) for small per-CTA products.
//
// What the elemental kernel needs: D[M x N] = A[M x K] B[N x K]^T in FP32, with M = 128 rows of
// which only the first rows are real (the local system has 12..60 unknowns per element), both
// operands K-major in shared memory without swizzle, the accumulator in tensor memory (TMEM).
//
// Operand layout ("canonical K-major, no swizzle"): the matrix is cut into core matrices of 8
// rows x 16 bytes (8 rows x 4 FP32/TF32 values), each 128 contiguous bytes with row r % 8 at
// byte 16 (r % 8).  Core matrix (row group g = r / 8, K chunk c = k / 4) sits at byte
// (g KC + c) 128, KC = K / 4 chunks per row: the stride between row groups (SBO) is KC 128 bytes,
// the stride between the two K chunks of one MMA step (LBO) is 128 bytes, and MMA step s (K = 8
// per kind::tf32 instruction) starts 256 s bytes in.
//
// 3xTF32: x = hi + lo with hi = x rounded to TF32 and lo = x - hi (exact in FP32) rounded to TF32;
// A B^T ~ A_lo B_hi^T + A_hi B_lo^T + A_hi B_hi^T (the A_lo B_lo^T term is below FP32 rounding),
// accumulated in FP32 by the tensor core: FP32-level products from TF32 inputs.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hdgx {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, sm_100 format: start address >> 4 (bits 0-13), leading-dimension
// byte offset >> 4 (bits 16-29), stride-dimension byte offset >> 4 (bits 32-45), version 1 (bits
// 46-47), base offset 0, no swizzle (layout type 0, bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), A and B TF32 (bits 7-9,
// 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (r, k) in the canonical K-major layout with KC K chunks per row group.
__host__ __device__ constexpr int kmajor_offset(int r, int k, int KC) {
    return ((r >> 3) * KC + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
    return __uint_as_float(u);
}
// x = hi + lo, both TF32 values
__device__ __forceinline__ void split_tf32(double x, float &hi, float &lo) {
    const float f = (float)x;
    hi = to_tf32(f);
    lo = to_tf32(f - hi);
}

// ---- TMEM allocation: one warp, power-of-two column count in [32, 512] (an immediate)
template <uint32_t NCOLS>
__device__ __forceinline__ void tmem_alloc(uint32_t *slot) {
    static_assert(NCOLS >= 32 && NCOLS <= 512 && (NCOLS & (NCOLS - 1)) == 0, "TMEM columns");
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "n"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- one MMA: D (+)= A B^T, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}
// the mbarrier is arrived on once every MMA issued before by this thread has completed
__device__ __forceinline__ void commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

// ---- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
// Wait for the phase with parity `phase` to complete; false when `limit` polls pass first.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t phase, int limit) {
    const uint32_t a = smem_u32(mbar);
    for (int n = 0; n < limit; n++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ---- ordering between the generic proxy (thread stores), the async proxy (the tensor core's
// shared-memory reads) and thread synchronisation
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- TMEM -> registers: this warp's 32 lanes (lane quarter warp % 4), 16 consecutive columns
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace hdgx
