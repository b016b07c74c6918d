// nnp_tc.cuh -- sm_100a tensor-core building blocks (tcgen05 + TMEM) for the
// atomic-network layers: shared-memory operand layout, UMMA descriptors,
// MMA issue/commit, TMEM allocation and loads, bounded mbarrier waits.
//
// Operands are BF16 in the canonical K-major, non-swizzled UMMA layout:
// 8x8 "core matrices" (8 rows x 16 bytes, 128 contiguous bytes), a tile of
// R rows x K columns stored as [R/8][K/8][8][8] elements, so that
//   leading byte offset (next 8 columns of K)  = 128 B
//   stride byte offset  (next 8 rows)          = (K/8) * 128 B
// and the descriptor of the k-th 16-column slice starts 256 B * k further.
// The accumulator of an M=128 MMA is 128 TMEM lanes x N 32-bit columns:
// row r of D is lane r, so warp w of the CTA reads rows 32w..32w+31.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace nnp {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// element offset of (r, k) in a K-major canonical tile with K columns (K % 8 == 0)
__host__ __device__ __forceinline__ int kmaj(int r, int k, int K)
{
    return (((r >> 3) * (K >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

// shared-memory matrix descriptor (SWIZZLE_NONE, K-major)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3fff);
    d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
    d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
    return d;                               // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: kind::f16, A/B BF16, D FP32, both K-major, M x N
__host__ __device__ __forceinline__ uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D(tmem) (+)= A(smem) * B(smem)^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// arrive on the mbarrier once every MMA issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Waits for the phase with the given parity to complete, polling with the
// non-blocking test_wait; gives up after max_iter polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t max_iter)
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < max_iter; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation: one whole warp; the address lands in *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 8 consecutive 32-bit columns of this thread's TMEM lane (warp-collective);
// the registers are read only after tmem_wait_tie on them
__device__ __forceinline__ void tmem_ld8_raw(uint32_t taddr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

// Waits for this thread's outstanding TMEM loads, with the registers of one
// x8 load as operands, so that no use of them is scheduled before the wait
__device__ __forceinline__ void tmem_wait_tie(uint32_t (&r)[8])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
                 :
                 : "memory");
}

}  // namespace tc
}  // namespace nnp
