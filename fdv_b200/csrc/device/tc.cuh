// Blackwell tensor-core primitives: tcgen05 MMA with TMEM accumulators,
// shared-memory matrix descriptors, mbarriers and cp.async staging.
//
// Operand tiles live in shared memory in the K-major, non-swizzled canonical
// layout: 8 rows x 16 bytes (8 bf16 along K) form one 128-byte core matrix; the
// 8 K-chunks of a 64-wide K tile follow each other (leading byte offset 128),
// and the next group of 8 rows starts 1024 bytes on (stride byte offset).  One
// tcgen05.mma of kind::f16 consumes K = 16, i.e. two chunks, so the k-th MMA of
// a 64-wide tile starts 256*k bytes into it.
//
// Every wait here is bounded by %globaltimer and reports through an error word
// instead of spinning forever.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

#include "common.cuh"

namespace fdvb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- cp.async (16-byte, L2 only); src_bytes 0 fills the chunk with zeros
__device__ __forceinline__ void cpa16(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
// 8-byte copy through L1 (both addresses 8-byte aligned)
__device__ __forceinline__ void cpa8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared-memory writes of the generic proxy (st.shared, cp.async) made visible
// to the tensor core's async proxy.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of the given parity to complete; false (and the error
// bit set) after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, unsigned *err,
                                          unsigned long long limit_ns = 1000000000ull) {
    if (mbar_test(b, parity)) return true;
    if (*(volatile unsigned *)err & kErrMmaTimeout) return false;   // an earlier wait already gave up
    const unsigned long long t0 = globaltimer();
    for (;;) {
        if (mbar_test(b, parity)) return true;
        if (globaltimer() - t0 > limit_ns) { atomicOr(err, kErrMmaTimeout); return false; }
    }
}

// ---- TMEM
// Allocation and release are warp-wide (.sync.aligned): call from one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// TMEM columns for an fp32 accumulator of n columns (a power of two >= 32).
__host__ __device__ constexpr uint32_t tmem_cols(int n) {
    return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : (n <= 256 ? 256u : 512u)));
}

// 32 lanes x 16 consecutive fp32 columns: this warp's rows (lanes 32*(warp%4)..),
// one row per thread.  Warp-wide.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- descriptors
// K-major, no swizzle: start address, leading byte offset (between the two
// 8-element K chunks of one MMA), stride byte offset (between 8-row groups),
// descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: fp32 accumulate, bf16 A and B, both K-major,
// N (multiple of 16, <= 256) in bits 17-22 as N/8, M (64 or 128) in bits 24-28 as M/16.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D (TMEM) [+]= A (smem) * B (smem)^T.  Issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The mbarrier completes one arrival when every MMA this thread issued before has finished.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Byte offset of element (r, k) of a K-major operand tile of 64-wide K
// chunks (k < 64) in the canonical layout above.
__host__ __device__ constexpr uint32_t umma_off(int r, int k) {
    return (uint32_t)(((r >> 3) * 8 + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

}  // namespace fdvb
