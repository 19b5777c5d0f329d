// Fifth-generation tensor core (tcgen05) building blocks for sm_100a, as
// inline PTX: shared-memory matrix descriptors, the instruction descriptor
// of a BF16 x BF16 -> FP32 MMA, tensor-memory (TMEM) allocation and loads,
// MMA issue / commit and bounded mbarrier waits.
//
// Operand layout used throughout: K-major, no swizzle. A tile of R rows
// (M or N) by K bf16 columns is stored as 8 x 8 "core matrices" (8 rows of
// 16 contiguous bytes, 128 bytes each); core matrix (rb, kb) sits at byte
// (rb * K/8 + kb) * 128, so neighbours along K are 128 bytes apart (the
// descriptor's leading byte offset) and neighbours along M/N K/8 * 128
// bytes apart (its stride byte offset). Element (r, k) is at
//   ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace oxd {
namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a K-major core-matrix tile K columns wide.
__host__ __device__ constexpr uint32_t cm_offset(uint32_t r, uint32_t k, uint32_t K) {
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (M/N) byte offsets, descriptor version 1 at bits 46-47, no swizzle.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 D, both
// operands K-major, dense: D format at bits 4-5, A / B formats at 7-9 /
// 10-12, N / 8 at 17-22, M / 16 at 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A[desc] x B[desc]^T for one K = 16 slice; one thread issues.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// Arrive on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// Whole-warp TMEM allocation of `ncols` columns (a power of two >= 32);
// the TMEM address is written to *slot in shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Shared-memory writes by threads become visible to the tensor core.
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w of the
// warpgroup reads lanes 32w..32w+31; lane = row of an M = 128 tile).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Initialises an mbarrier and makes the initialisation visible to the
// tensor core's arrivals.
__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for phase `parity` of `bar` to complete, at most `limit` polls.
// False when it gave up (the caller records an error and leaves cleanly).
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    uint32_t a = smem_addr(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

}  // namespace umma
}  // namespace oxd
