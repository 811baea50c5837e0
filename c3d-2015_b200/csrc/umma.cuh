// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a: tensor-memory
// allocation, the single-thread MMA issue with operands in shared memory, completion through
// an mbarrier, and the tensor-memory load of the FP32 accumulators.
//
// Operand layout (both operands K-major, no swizzle): 8-row x 16-byte core matrices, a core
// matrix's rows 16 bytes apart; along K the core matrices of one 8-row group are contiguous
// (leading byte offset 128), the 8-row groups are SBO bytes apart. Element (r, k) of an
// operand with KG 16-byte groups per row sits at
//     (r / 8) * SBO + (k * es / 16) * 128 + (r % 8) * 16 + (k * es) % 16,   SBO = 128 KG.
// One MMA instruction consumes 32 bytes of K per row (two core matrices): K = 16 for BF16,
// K = 8 for TF32; the next instruction's operands start 256 bytes further.
#pragma once
#include <cstdint>

namespace c3d {
namespace {

__device__ __forceinline__ uint32_t umma_smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading byte offset 128 (K direction),
// stride byte offset sbo (8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, A and B of format fmt (1 BF16, 2 TF32), both
// K-major, N = n, M = m.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt, int m, int n)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread. TF32 when tf32, else BF16 (kind::f16).
template <bool TF32>
__device__ __forceinline__ void umma_issue(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                           uint32_t idesc, uint32_t accumulate)
{
    if constexpr (TF32)
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                     : "memory");
    else
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                     : "memory");
}

// Arrives once on the mbarrier when every tcgen05 operation this thread issued before has
// completed (reads of shared memory included).
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     umma_smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Generic-proxy stores to shared memory made visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Whole warp: allocates ncols (power of two >= 32) tensor-memory columns, address to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     umma_smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}

// Whole warp.
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

// Whole warp: 16 consecutive 32-bit columns of the warp's 32 lanes (thread l: lane l).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// FP32 -> TF32, round to nearest (ties away), as a 32-bit pattern with the low 13 bits 0.
__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return r;
}

} // namespace
} // namespace c3d
