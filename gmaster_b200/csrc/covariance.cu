// Gaussian covariance of pseudo-C_ell bandpowers in the narrow-kernel approximation
// (gmaster/covariance.py:407-575): every output block X (a pair of spectrum components of
// the two power spectra) is a signed sum of terms
//     cov_X(l1, l2) = sum_t sign_t * (A_t(l1) B_t(l2) + A_t(l2) B_t(l1)) / 2 * Xi_{k_t}(l1, l2)
// with A_t, B_t rows of the best-guess spectra and Xi_k the coupling kernels of the mask
// products.  The host builds the term list from the spins (which kernel and which spectra
// each output block takes); these kernels evaluate it.
//
// k_cov_binned fuses the assembly with the binning of both sides: one CTA per pair of
// bands (p, q) reads the (l1 in p) x (l2 in q) tile of every kernel once and reduces the
// weighted sums of all output blocks, so the unbinned (L x L) blocks are never written.
// k_cov_coupled writes the unbinned blocks (the coupled covariance).

#include "gm_common.cuh"

namespace gm {
namespace {

constexpr int kCovMaxBlocks = 16;   // 4 x 4 components (spin 2 x spin 2)
constexpr int kCovThreads = 256;

struct CovTerms {
    const double *xi;        // (nk, L, L) kernels
    const double *spec;      // (nrows, L) best-guess spectra
    const int32_t *terms;    // (nterm, 3): kernel, row of A, row of B
    const double *signs;     // (nterm,)
    const int32_t *bptr;     // (nblocks + 1,) term range of each output block
};

__device__ __forceinline__ double block_value(const CovTerms &c, int64_t L, int x, int64_t l1,
                                              int64_t l2)
{
    double s = 0.0;
    const int t1 = c.bptr[x + 1];
    for (int t = c.bptr[x]; t < t1; ++t) {
        const int64_t k = c.terms[3 * t], ra = c.terms[3 * t + 1], rb = c.terms[3 * t + 2];
        const double *A = c.spec + ra * L, *B = c.spec + rb * L;
        const double sym = 0.5 * (A[l1] * B[l2] + A[l2] * B[l1]);
        s += c.signs[t] * sym * c.xi[(k * L + l1) * L + l2];
    }
    return s;
}

__global__ void __launch_bounds__(kCovThreads) k_cov_binned(
    int64_t L, int nblocks, CovTerms c, const int32_t *__restrict__ ptr_a,
    const int32_t *__restrict__ ells_a, const double *__restrict__ w_a,
    const int32_t *__restrict__ ptr_b, const int32_t *__restrict__ ells_b,
    const double *__restrict__ w_b, int64_t nbb, double *__restrict__ out, int64_t nba)
{
    __shared__ double red[kCovThreads / 32][kCovMaxBlocks];
    const int64_t p = blockIdx.y, q = blockIdx.x;
    const int a0 = ptr_a[p], n1 = ptr_a[p + 1] - a0;
    const int b0 = ptr_b[q], n2 = ptr_b[q + 1] - b0;
    double acc[kCovMaxBlocks];
#pragma unroll
    for (int x = 0; x < kCovMaxBlocks; ++x) acc[x] = 0.0;
    const int64_t n = (int64_t)n1 * n2;
    for (int64_t e = threadIdx.x; e < n; e += kCovThreads) {
        const int64_t l1 = ells_a[a0 + (int)(e / n2)];
        const int64_t l2 = ells_b[b0 + (int)(e % n2)];
        const double w = w_a[l1] * w_b[l2];
#pragma unroll
        for (int x = 0; x < kCovMaxBlocks; ++x)
            if (x < nblocks) acc[x] += w * block_value(c, L, x, l1, l2);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int x = 0; x < kCovMaxBlocks; ++x) {
        if (x >= nblocks) break;
        double v = acc[x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][x] = v;
    }
    __syncthreads();
    if (threadIdx.x < nblocks) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kCovThreads / 32; ++w) v += red[w][threadIdx.x];
        out[((int64_t)threadIdx.x * nba + p) * nbb + q] = v;
    }
}

__global__ void __launch_bounds__(kCovThreads) k_cov_coupled(int64_t L, int nblocks, CovTerms c,
                                                             double *__restrict__ out)
{
    const int64_t l1 = blockIdx.y;
    const int64_t l2 = (int64_t)blockIdx.x * kCovThreads + threadIdx.x;
    if (l2 >= L) return;
    for (int x = 0; x < nblocks; ++x) out[((int64_t)x * L + l1) * L + l2] = block_value(c, L, x, l1, l2);
}

}  // namespace
}  // namespace gm

using namespace gm;

extern "C" int gm_cov_binned(int64_t lmax, int64_t nblocks, const double *xi, const double *spec,
                             const int32_t *terms, const double *signs, const int32_t *block_ptr,
                             int64_t nbands_a, const int32_t *ptr_a, const int32_t *ells_a,
                             const double *w_a, int64_t nbands_b, const int32_t *ptr_b,
                             const int32_t *ells_b, const double *w_b, double *out, void *stream)
{
    if (lmax < 0 || nblocks < 1 || nblocks > kCovMaxBlocks || nbands_a < 1 || nbands_b < 1 ||
        nbands_a > 65535 || nbands_b > (int64_t)INT32_MAX)
        return GM_ERR_BAD_SHAPE;
    if (!xi || !spec || !terms || !signs || !block_ptr || !ptr_a || !ells_a || !w_a || !ptr_b ||
        !ells_b || !w_b || !out)
        return GM_ERR_BAD_PTR;
    const CovTerms c{xi, spec, terms, signs, block_ptr};
    const dim3 grid((unsigned)nbands_b, (unsigned)nbands_a);
    k_cov_binned<<<grid, kCovThreads, 0, as_stream(stream)>>>(
        lmax + 1, (int)nblocks, c, ptr_a, ells_a, w_a, ptr_b, ells_b, w_b, nbands_b, out, nbands_a);
    return check_launch("gm_cov_binned");
}

extern "C" int gm_cov_coupled(int64_t lmax, int64_t nblocks, const double *xi, const double *spec,
                              const int32_t *terms, const double *signs, const int32_t *block_ptr,
                              double *out, void *stream)
{
    if (lmax < 0 || lmax + 1 > 65535 || nblocks < 1 || nblocks > kCovMaxBlocks)
        return GM_ERR_BAD_SHAPE;
    if (!xi || !spec || !terms || !signs || !block_ptr || !out) return GM_ERR_BAD_PTR;
    const CovTerms c{xi, spec, terms, signs, block_ptr};
    const int64_t L = lmax + 1;
    const dim3 grid((unsigned)((L + kCovThreads - 1) / kCovThreads), (unsigned)L);
    k_cov_coupled<<<grid, kCovThreads, 0, as_stream(stream)>>>(L, (int)nblocks, c, out);
    return check_launch("gm_cov_coupled");
}
