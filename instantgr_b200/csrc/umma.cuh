// tcgen05 (5th-generation tensor core) building blocks for sm_100a: shared
// memory matrix descriptors, the instruction descriptor of a BF16 x BF16 ->
// F32 MMA, TMEM allocation, MMA issue and commit, bounded mbarrier waits and
// TMEM loads.  Operand tiles use the canonical K-major layout without
// swizzle: 8 rows x 16 bytes per core matrix (128 contiguous bytes), the two
// 8-element K halves of a K = 16 step 128 bytes apart (leading byte offset),
// groups of 8 rows 256 bytes apart (stride byte offset).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace igr {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// element offset of (row r, k) in a 128 (or fewer) x 16 sub-tile
__device__ __forceinline__ int sub_idx(int r, int k) { return (r >> 3) * 128 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);  // start address
    d |= (uint64_t)(128 >> 4) << 16;                 // leading byte offset: K halves
    d |= (uint64_t)(256 >> 4) << 32;                 // stride byte offset: 8-row groups
    d |= (uint64_t)1 << 46;                          // descriptor version of sm_100
    return d;                                        // base offset 0, no swizzle
}

// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// one warp: allocate `cols` TMEM columns (power of two >= 32), address into *dst
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, int cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, int cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// waits for the phase of `parity` to complete; gives up after `limit_ns`
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned long long limit_ns) {
    const uint32_t a = smem_u32(bar);
    const unsigned long long t0 = now_ns();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (now_ns() - t0 > limit_ns) return false;
    }
}

// D[tmem] (+)= A * B^T for one K = 16 step; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate ? 1u : 0u), "r"(0u)
        : "memory");
}
// arrives on `bar` once every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 8 consecutive f32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = __uint_as_float(r[j]);
}

}  // namespace umma
}  // namespace igr
