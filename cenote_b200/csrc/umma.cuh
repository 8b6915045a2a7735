// Fifth-generation tensor-core helpers (tcgen05, sm_100a): shared-memory
// matrix descriptors, the instruction descriptor for BF16 x BF16 -> FP32,
// TMEM allocation, MMA issue/commit, bounded mbarrier waits and TMEM loads.
//
// Encodings follow the PTX ISA's tcgen05 matrix and instruction descriptors
// (the same bit layout as CUTLASS's UMMA::SmemDescriptor / InstrDescriptor,
// cute/arch/mma_sm100_desc.hpp). Only one shared-memory layout is used: the
// no-swizzle K-major canonical layout, built from 8-row x 16-byte core
// matrices (8 rows of 8 BF16 along K). For an R x C matrix (C along K):
//     byte(r, c) = (r / 8) * SBO + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2,
// with LBO = 128 (adjacent core matrices along K) and SBO = (C / 8) * 128
// (adjacent 8-row groups). An MMA consuming K columns [k0, k0 + 16) starts at
// the matrix base + (k0 / 8) * 128.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace cn {
namespace umma {

// Byte offset of element (r, c) of an R x C K-major canonical matrix.
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t r, uint32_t c, uint32_t cols) {
    return (r / 8u) * (cols / 8u) * 128u + (c / 8u) * 128u + (r % 8u) * 16u + (c % 8u) * 2u;
}

// Shared-memory matrix descriptor, no swizzle, version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t smem_addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= uint64_t((smem_addr >> 4) & 0x3fffu);
    d |= uint64_t((lbo_bytes >> 4) & 0x3fffu) << 16;
    d |= uint64_t((sbo_bytes >> 4) & 0x3fffu) << 32;
    d |= uint64_t(1) << 46;  // descriptor version
    // base offset 0, LBO mode 0, layout type 0 (no swizzle)
    return d;
}

// Descriptor of the 16-wide K slice at k0 of an R x cols canonical matrix.
__device__ __forceinline__ uint64_t kslice_desc(uint32_t base_addr, uint32_t k0, uint32_t cols) {
    return smem_desc(base_addr + (k0 / 8u) * 128u, 128u, (cols / 8u) * 128u);
}

// Instruction descriptor for kind::f16: D F32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t m, uint32_t n) {
    return (1u << 4)           // D format F32
           | (1u << 7)         // A format BF16
           | (1u << 10)        // B format BF16
           | ((n >> 3) << 17)  // N / 8
           | ((m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// TMEM columns for this CTA (one warp, converged); the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A * B for one 16-deep K slice; issued by a single thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// Arrive on `bar` once every MMA this thread issued so far has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core's reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the phase with `parity` to complete, at most `limit` polls.
// Returns false when the bound ran out (the caller records an error and
// unwinds; nothing waits forever).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp
// w of the warpgroup reads lanes 32w..32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM address of (lane, column) relative to an allocation.
__device__ __forceinline__ uint32_t tmem_at(uint32_t base, uint32_t lane, uint32_t col) {
    return base + (lane << 16) + col;
}

}  // namespace umma
}  // namespace cn
