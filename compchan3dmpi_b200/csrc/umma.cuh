// umma.cuh -- the sm_100a tensor-core pieces the closure MLP kernels use:
// tcgen05.mma (kind::f16, BF16 x BF16 -> F32 in tensor memory) issued by one
// thread, its completion signalled through an mbarrier, tensor-memory
// allocation and the 32x32b tensor-memory loads of the epilogues.
//
// Operand tiles live in shared memory in the K-major layout without
// swizzle: an R x K BF16 tile is cut into 8 x 8 "core matrices" (8 rows of
// 16 bytes, 128 contiguous bytes); element (r, k) sits at byte
//     (r / 8) * (K * 16) + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// For one MMA of K = 16 the descriptor's leading byte offset (between the
// two 8-column core matrices along K) is 128 and its stride byte offset
// (between 8-row groups) is K * 16; step s of the K loop starts 256 * s
// bytes further in.
#pragma once
#include <cstdint>

namespace umma {

__host__ __device__ constexpr uint32_t kmaj_off(int r, int k, int K)
{
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start, leading / stride byte offsets (16-byte
// units), version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D(tmem) (+)= A(smem) * B(smem)^T for one K = 16 step
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// D = A * B^T over K (a multiple of 16): A is M(=128) x K, B is N x K, both
// K-major tiles as above; issued by the calling thread
__device__ __forceinline__ void gemm_kmajor(uint32_t d_tmem, const void *A, const void *B, int K, int N,
                                            bool accumulate)
{
    const uint32_t a0 = smem_u32(A), b0 = smem_u32(B), sbo = (uint32_t)K * 16u;
    const uint32_t id = idesc_bf16_f32(128, N);
    for (int s = 0; s < K / 16; s++)
        mma_bf16(d_tmem, sdesc(a0 + 256u * s, 128u, sbo), sdesc(b0 + 256u * s, 128u, sbo), id,
                 (accumulate || s > 0) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for phase `parity` of the barrier; false after `limit` polls (the
// caller records the error and stops issuing work)
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// generic-proxy shared-memory writes made visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// tensor-memory allocation by one whole warp; the base address lands in *dst
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive F32 columns of this thread's lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t lane_addr(uint32_t tmem_base, int warp, int col)
{
    return tmem_base + ((uint32_t)(warp * 32) << 16) + (uint32_t)col;
}

}  // namespace umma
