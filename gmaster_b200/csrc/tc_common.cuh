// sm_100a tensor-core (tcgen05 / TMEM / bulk-copy) primitives shared by the tensor-core
// kernels.  Written against the PTX ISA; every wait is bounded and reports a timeout.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace gm {
namespace tc {

// Time limit of an mbarrier wait in nanoseconds (of the global timer).
constexpr uint64_t kWaitNs = 2000000000ull;

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Suspend-time hint of one try_wait (ns): the waiting thread sleeps in hardware until the
// phase completes or the hint expires, instead of spinning on the issue slots that the
// warps sharing its scheduler need.
constexpr uint32_t kSuspendNs = 200000u;

// Wait for the phase with parity `parity` to complete.  Returns false once `limit_ns` of
// global time (kWaitNs by default) have passed without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = kWaitNs)
{
    const uint32_t addr = smem_u32(bar);
    uint64_t start = 0;
    for (uint32_t it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity), "r"(kSuspendNs)
            : "memory");
        if (done) return true;
        const uint64_t now = global_ns();
        if (it == 0) start = now;
        else if (now - start > limit_ns) return false;
    }
}

// Bulk (non-tensor) copy global -> shared, completing `bytes` on the mbarrier.
// Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes,
                                         uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Prefetch `bytes` of global memory into L2 (16-byte aligned address, size a multiple of 16).
__device__ __forceinline__ void prefetch_l2(const void *gmem_src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gmem_src), "r"(bytes) : "memory");
}

// Make generic-proxy shared-memory writes visible to the async proxy (tcgen05.mma reads).
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (bf16/f16 inputs, f32 accumulate), cta_group::1.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` when every previously issued tcgen05.mma of this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 columns of 32-bit TMEM into registers (warp-collective).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, 128-byte swizzle: 8-row groups 1024 bytes
// apart (SBO), rows of 128 bytes; start address advanced by 32 bytes per K step of 16.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// Shared-memory matrix descriptor, MN-major, 128-byte swizzle: atoms of 64 MN-elements x
// 8 K-rows (1024 bytes); `lbo` = byte stride between 64-element MN blocks, `sbo` = byte
// stride between groups of 8 K-rows.
__device__ __forceinline__ uint64_t desc_sw128_mn(uint32_t smem_addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Byte offset of element (r, k) in an MN-major SW128 image with R MN-rows (R % 64 == 0):
// K in groups of 8 (stride (R/64) 1024 bytes), MN in blocks of 64 (stride 1024 bytes).
__host__ __device__ __forceinline__ uint32_t sw128_mn_offset(uint32_t R, uint32_t r, uint32_t k)
{
    const uint32_t chunk = ((r & 63) >> 3) ^ (k & 7);
    return (k >> 3) * (R >> 6) * 1024u + (r >> 6) * 1024u + (k & 7) * 128u + chunk * 16u + (r & 7) * 2u;
}

// Instruction descriptor: kind::f16, A/B bf16 (fmt 1) or f16 (fmt 0), D f32, K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, int fmt, int a_mn = 0, int b_mn = 0)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)a_mn << 15) |
           ((uint32_t)b_mn << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row r, k) in a K-major SW128 image of R rows: K is split into
// atoms of 64 16-bit elements, each atom R x 128 bytes.
__host__ __device__ __forceinline__ uint32_t sw128_offset(uint32_t R, uint32_t r, uint32_t k)
{
    const uint32_t atom = k >> 6, kk = k & 63;
    const uint32_t chunk = (kk >> 3) ^ (r & 7);
    return atom * R * 128u + (r >> 3) * 1024u + (r & 7) * 128u + chunk * 16u + (kk & 7) * 2u;
}

// Split two floats into f16 hi + f16 lo pairs: hi + lo carries 22 significant bits for
// magnitudes in [2^-3, 2^15]; below that lo is subnormal and the absolute error is at
// most 2^-25.  Callers scale their operands by a power of two into that range.
__device__ __forceinline__ void split_f16x2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    __half2 h = __floats2half2_rn(a, b);
    float2 hf = __half22float2(h);
    __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

// Split a float into bf16 hi + bf16 lo (hi + lo carries 16 significant bits).
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

}  // namespace tc
}  // namespace gm
