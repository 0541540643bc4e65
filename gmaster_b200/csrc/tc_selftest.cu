// Self-test of the tcgen05 path: one CTA computes D[128 x N] = A[128 x K] * B[N x K]^T
// from K-major, 128-byte-swizzled bf16 operand images, exercising the bulk copy engine,
// mbarriers, TMEM allocation, tcgen05.mma / commit and tcgen05.ld exactly as the
// Legendre tensor-core kernels do.  Used by the GPU tests and as a device health check.
//
// With `skip_copies` the issuer arms the load barrier for both operand images but issues
// no copy, so the bounded wait of every thread runs out after `wait_ns`: the kernel then
// records the timeout in *err, skips the MMAs and the TMEM reads, releases its TMEM and
// returns (the error path of the Legendre kernels, exercised without a fault or hang).
#include "gm_common.cuh"
#include "tc_common.cuh"

namespace gm {

__global__ void __launch_bounds__(128) k_tc_selftest(int N, int K, int a_mn, int b_mn,
                                                     const uint8_t *__restrict__ aimg,
                                                     const uint8_t *__restrict__ bimg,
                                                     float *__restrict__ D, int *__restrict__ err,
                                                     uint64_t wait_ns, int skip_copies)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bar_load, bar_mma;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (tc::smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t *sA = smem_raw + (base - tc::smem_u32(smem_raw));
    const uint32_t a_bytes = 128u * (uint32_t)K * 2u, b_bytes = (uint32_t)N * (uint32_t)K * 2u;
    uint8_t *sB = sA + a_bytes;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)N) ncols <<= 1;
    if (tid == 0) {
        tc::mbar_init(&bar_load, 1);
        tc::mbar_init(&bar_mma, 1);
        tc::fence_mbar_init();
    }
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, ncols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = tmem_base;
    if (tid == 0) {
        tc::mbar_arrive_expect_tx(&bar_load, a_bytes + b_bytes);
        if (!skip_copies) {
            tc::bulk_g2s(sA, aimg, a_bytes, &bar_load);
            tc::bulk_g2s(sB, bimg, b_bytes, &bar_load);
        }
    }
    const bool loaded = tc::mbar_wait(&bar_load, 0, wait_ns);
    if (tid == 0) {
        if (loaded) {
            const uint32_t idesc = tc::idesc_f16(128, N, 1, a_mn, b_mn);
            for (int ks = 0; ks < K / 16; ++ks) {
                const int a = ks >> 2, kk = ks & 3;
                // K-major: atom of 64 K x rows of 128 B, +32 B per K step of 16.
                // MN-major: K groups of 8 at stride (R/64) 1024 B, two groups per K step.
                const uint64_t da = a_mn
                    ? tc::desc_sw128_mn(tc::smem_u32(sA) + ks * 2 * 2048, 1024, 2048)
                    : tc::desc_sw128(tc::smem_u32(sA) + a * 128 * 128 + kk * 32);
                const uint32_t bsbo = (uint32_t)(N >= 64 ? N / 64 : 1) * 1024u;
                const uint64_t db = b_mn
                    ? tc::desc_sw128_mn(tc::smem_u32(sB) + ks * 2 * bsbo, 1024, bsbo)
                    : tc::desc_sw128(tc::smem_u32(sB) + a * N * 128 + kk * 32);
                tc::mma_f16(taddr, da, db, idesc, ks != 0);
            }
            tc::mma_commit(&bar_mma);
        } else {
            atomicExch(err, 1);
        }
    }
    bool done = true;
    if (loaded) done = tc::mbar_wait(&bar_mma, 0, wait_ns);
    if (!done && lane == 0) atomicExch(err, 2);
    tc::tc_fence_after();
    if (loaded && done) {
        for (int c = 0; c < N; c += 16) {
            uint32_t r[16];
            tc::tmem_ld16(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, r);
            tc::tmem_ld_wait();
            float *row = D + (int64_t)(32 * warp + lane) * N + c;
#pragma unroll
            for (int i = 0; i < 16; ++i) row[i] = __uint_as_float(r[i]);
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(taddr, ncols);
}

}  // namespace gm

using namespace gm;

static int launch_selftest(int64_t N, int64_t K, int a_mn, int b_mn, const void *aimg, const void *bimg,
                           float *D, int32_t *err, uint64_t wait_ns, int skip_copies, void *stream);

extern "C" int gm_tc_selftest(int64_t N, int64_t K, int a_mn, int b_mn, const void *aimg,
                              const void *bimg, float *D, int32_t *err, void *stream)
{
    return launch_selftest(N, K, a_mn, b_mn, aimg, bimg, D, err, tc::kWaitNs, 0, stream);
}

extern "C" int gm_tc_selftest_timeout(int64_t N, int64_t K, const void *aimg, const void *bimg,
                                      float *D, int32_t *err, int64_t wait_ns, void *stream)
{
    if (wait_ns < 1000 || wait_ns > (int64_t)tc::kWaitNs) return GM_ERR_BAD_SHAPE;
    return launch_selftest(N, K, 0, 0, aimg, bimg, D, err, (uint64_t)wait_ns, 1, stream);
}

static int launch_selftest(int64_t N, int64_t K, int a_mn, int b_mn, const void *aimg, const void *bimg,
                           float *D, int32_t *err, uint64_t wait_ns, int skip_copies, void *stream)
{
    if (N < 16 || N > 256 || (N % 16) || K < 64 || (K % 64) || 128 * K * 2 + N * K * 2 > 200 * 1024)
        return GM_ERR_BAD_SHAPE;
    if (b_mn && (N % 64)) return GM_ERR_BAD_SHAPE;
    if (!aimg || !bimg || !D || !err) return GM_ERR_BAD_PTR;
    const size_t smem = (size_t)(128 * K * 2 + N * K * 2) + 1024;
    cudaError_t e = cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_error("gm_tc_selftest attr", e);
        return GM_ERR_LAUNCH;
    }
    k_tc_selftest<<<1, 128, smem, as_stream(stream)>>>((int)N, (int)K, a_mn, b_mn, (const uint8_t *)aimg,
                                                      (const uint8_t *)bimg, D, (int *)err, wait_ns,
                                                      skip_copies);
    return check_launch("gm_tc_selftest");
}
