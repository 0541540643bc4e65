// Gauss-Legendre nodes and Wigner-d rows at those nodes, for the coupling blocks of purified
// E/B fields (gmaster/workspaces.py:593-679, 927-1061: quadrature of products of Wigner
// d-functions weighted by the mask's correlation functions).
//
// k_gl_nodes: one thread per node, Newton's iteration on P_n(x) from the three-term
// recurrence, starting from cos(pi (i + 3/4) / (n + 1/2)); the weight is
// 2 / ((1 - x^2) P_n'(x)^2).
//
// d^l_mn(beta) for l >= l0 = max(|m|, |n|) is (-1)^((n - m + mu) / 2) sin(beta/2)^mu
// cos(beta/2)^nu N_k P_k^(mu, nu)(cos beta) with k = l - l0, mu = |m - n|, nu = |m + n|,
// N_k = sqrt(k! (k + mu + nu)! / ((k + mu)! (k + nu)!)) (a table from the host) and the
// Jacobi polynomials from their three-term recurrence (DLMF 18.9.1).  k_wigner_table
// writes the (lmax + 1) x nnodes rows; k_wigner_corr accumulates sum_l d^l_mn(beta) v[l]
// for up to two vectors v without storing the rows.

#include "gm_common.cuh"

namespace gm {
namespace {

constexpr int kWigThreads = 128;

struct Jacobi {
    double x, pref;
    int mu, nu, l0;
};

__device__ __forceinline__ Jacobi jacobi_setup(double x, int m, int n)
{
    Jacobi j;
    j.x = x;
    j.mu = abs(m - n);
    j.nu = abs(m + n);
    j.l0 = max(abs(m), abs(n));
    const double sh = sqrt(fmax(0.5 * (1.0 - x), 0.0)), ch = sqrt(fmax(0.5 * (1.0 + x), 0.0));
    double p = ((((n - m + j.mu) / 2) & 1) ? -1.0 : 1.0);
    for (int i = 0; i < j.mu; ++i) p *= sh;
    for (int i = 0; i < j.nu; ++i) p *= ch;
    j.pref = p;
    return j;
}

// P_k from P_{k-1}, P_{k-2} (k >= 2)
__device__ __forceinline__ double jacobi_next(const Jacobi &j, int k, double p1, double p0)
{
    const double dk = (double)k, t = (double)(j.mu + j.nu);
    const double mu = (double)j.mu, nu = (double)j.nu;
    const double a = (2.0 * dk + t - 1.0) * ((2.0 * dk + t) * (2.0 * dk + t - 2.0) * j.x + mu * mu - nu * nu);
    const double b = 2.0 * (dk + mu - 1.0) * (dk + nu - 1.0) * (2.0 * dk + t);
    const double c = 2.0 * dk * (dk + t) * (2.0 * dk + t - 2.0);
    return (a * p1 - b * p0) / c;
}

__global__ void __launch_bounds__(kWigThreads) k_gl_nodes(int64_t n, double *__restrict__ x_out,
                                                          double *__restrict__ w_out)
{
    const int64_t i = (int64_t)blockIdx.x * kWigThreads + threadIdx.x;
    if (i >= n) return;
    const double pi = 3.141592653589793;
    double x = cos(pi * ((double)i + 0.75) / ((double)n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
        double p0 = 1.0, p1 = x;
        for (int64_t k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / (double)k;
            p0 = p1;
            p1 = p2;
        }
        // P_n = p1, P_{n-1} = p0
        dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
        const double dx = p1 / dp;
        x -= dx;
        if (fabs(dx) <= 1e-16 * fmax(fabs(x), 1e-3)) break;
    }
    {
        double p0 = 1.0, p1 = x;
        for (int64_t k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / (double)k;
            p0 = p1;
            p1 = p2;
        }
        dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
    }
    // nodes in ascending order
    const int64_t o = n - 1 - i;
    x_out[o] = x;
    w_out[o] = 2.0 / ((1.0 - x * x) * dp * dp);
}

__global__ void __launch_bounds__(kWigThreads) k_wigner_table(
    int64_t nnodes, const double *__restrict__ xs, int64_t lmax, int m, int n,
    const double *__restrict__ norm, double *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * kWigThreads + threadIdx.x;
    if (i >= nnodes) return;
    const Jacobi j = jacobi_setup(xs[i], m, n);
    for (int64_t l = 0; l < j.l0 && l <= lmax; ++l) out[l * nnodes + i] = 0.0;
    if (j.l0 > lmax) return;
    double p0 = 1.0, p1 = 0.5 * ((double)(j.mu - j.nu) + (double)(j.mu + j.nu + 2) * j.x);
    out[(int64_t)j.l0 * nnodes + i] = j.pref * norm[0] * p0;
    if (j.l0 + 1 <= lmax) out[(int64_t)(j.l0 + 1) * nnodes + i] = j.pref * norm[1] * p1;
    for (int64_t l = j.l0 + 2; l <= lmax; ++l) {
        const int k = (int)(l - j.l0);
        const double p2 = jacobi_next(j, k, p1, p0);
        p0 = p1;
        p1 = p2;
        out[l * nnodes + i] = j.pref * norm[k] * p2;
    }
}

__global__ void __launch_bounds__(kWigThreads) k_wigner_corr(
    int64_t nnodes, const double *__restrict__ xs, int64_t lmax, int m, int n,
    const double *__restrict__ norm, int nvec, const double *__restrict__ vec,
    double *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * kWigThreads + threadIdx.x;
    if (i >= nnodes) return;
    const Jacobi j = jacobi_setup(xs[i], m, n);
    const int64_t L = lmax + 1;
    double acc0 = 0.0, acc1 = 0.0;
    if (j.l0 <= lmax) {
        double p0 = 1.0, p1 = 0.5 * ((double)(j.mu - j.nu) + (double)(j.mu + j.nu + 2) * j.x);
        double d = norm[0] * p0;
        acc0 += d * vec[j.l0];
        if (nvec > 1) acc1 += d * vec[L + j.l0];
        if (j.l0 + 1 <= lmax) {
            d = norm[1] * p1;
            acc0 += d * vec[j.l0 + 1];
            if (nvec > 1) acc1 += d * vec[L + j.l0 + 1];
        }
        for (int64_t l = j.l0 + 2; l <= lmax; ++l) {
            const int k = (int)(l - j.l0);
            const double p2 = jacobi_next(j, k, p1, p0);
            p0 = p1;
            p1 = p2;
            d = norm[k] * p2;
            acc0 += d * vec[l];
            if (nvec > 1) acc1 += d * vec[L + l];
        }
    }
    out[i] = j.pref * acc0;
    if (nvec > 1) out[nnodes + i] = j.pref * acc1;
}

}  // namespace
}  // namespace gm

using namespace gm;

extern "C" int gm_gl_nodes(int64_t n, double *x, double *w, void *stream)
{
    if (n < 1 || n > (1 << 24)) return GM_ERR_BAD_SHAPE;
    if (!x || !w) return GM_ERR_BAD_PTR;
    const unsigned grid = (unsigned)((n + kWigThreads - 1) / kWigThreads);
    k_gl_nodes<<<grid, kWigThreads, 0, as_stream(stream)>>>(n, x, w);
    return check_launch("gm_gl_nodes");
}

static bool wigner_args_ok(int64_t nnodes, int64_t lmax, int m, int n)
{
    return nnodes >= 1 && nnodes <= (1 << 24) && lmax >= 0 && lmax < (1 << 24) && abs(m) <= 16 &&
           abs(n) <= 16;
}

extern "C" int gm_wigner_table(int64_t nnodes, const double *x, int64_t lmax, int m, int n,
                               const double *norm, double *out, void *stream)
{
    if (!wigner_args_ok(nnodes, lmax, m, n)) return GM_ERR_BAD_SHAPE;
    if (!x || !norm || !out) return GM_ERR_BAD_PTR;
    const unsigned grid = (unsigned)((nnodes + kWigThreads - 1) / kWigThreads);
    k_wigner_table<<<grid, kWigThreads, 0, as_stream(stream)>>>(nnodes, x, lmax, m, n, norm, out);
    return check_launch("gm_wigner_table");
}

extern "C" int gm_wigner_corr(int64_t nnodes, const double *x, int64_t lmax, int m, int n,
                              const double *norm, int64_t nvec, const double *vec, double *out,
                              void *stream)
{
    if (!wigner_args_ok(nnodes, lmax, m, n) || nvec < 1 || nvec > 2) return GM_ERR_BAD_SHAPE;
    if (!x || !norm || !vec || !out) return GM_ERR_BAD_PTR;
    const unsigned grid = (unsigned)((nnodes + kWigThreads - 1) / kWigThreads);
    k_wigner_corr<<<grid, kWigThreads, 0, as_stream(stream)>>>(nnodes, x, lmax, m, n, norm,
                                                                (int)nvec, vec, out);
    return check_launch("gm_wigner_corr");
}
