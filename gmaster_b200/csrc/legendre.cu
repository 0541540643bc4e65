// Latitudinal (Legendre / spin-weighted Wigner-d) stage, SIMT kernels for sm_100a.
//
// For each order m the rows lambda^{s'}_lm(theta) = sqrt((2l+1)/4pi) d^l_{m,s'}(theta)
// are generated on the fly by the normalised three-term recurrence in l, in double
// precision with an explicit binary exponent per lane (values below 2^-300 are
// carried exactly and emitted as zero), and contracted against the ring spectra.
// Only northern lanes are marched: the hemisphere fold
//   lambda^{s'}_lm(pi - theta) = (-1)^{l+m} lambda^{-s'}_lm(theta)
// turns the two hemispheres into the Sum / Diff right-hand sides of `rhs`.
//
// The contraction is carried in T (double for GM_FP64, float for GM_MIXED); the
// recurrence is always double.  These kernels are the plain-FP64 path and the
// narrow-batch mixed path; the tensor-core path (legendre_tc.cu) takes wide batches.
//
// Replaces gmaster/_native/cuda/march_v2.cu:155-407 (march_analysis /
// march_synthesis: float32 difference-form recurrence, SIMT FMA contraction).
#include <math.h>

#include "gm_common.cuh"

namespace gm {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;
constexpr int kWindow = 32;
// Spins 1..kMaxSpin share the polarised kernels (template SPIN = 2) with the spin passed at
// run time; the seed table holds 2 kMaxSpin + 1 variants.
constexpr int kMaxSpin = 8;

// First seed-table variant of spin s >= 1 (s' = -s; the next one is s' = +s): spin 2 keeps
// variants 1 and 2 (the tensor-core kernels read them), spin 1 takes 3 and 4, spin s >= 3
// takes 2s - 1 and 2s.
__host__ __device__ __forceinline__ int seed_variant(int s)
{
    return s == 2 ? 1 : (s == 1 ? 3 : 2 * s - 1);
}
constexpr double kBig = 2.037035976334486e90;     // 2^300
constexpr double kShrink = 2.409919865102884e-181;  // 2^-600

// Seed of one lane: value = sign * 2^f carried as v * 2^(600 k), k <= 0.
__device__ __forceinline__ void seed_lane(const double *__restrict__ sd, double lsin, double lcos,
                                          double &v, int &k)
{
    double f = sd[0];
    if (sd[2] != 0.0) f += sd[2] * lcos;
    if (sd[3] != 0.0) f += sd[3] * lsin;
    if (!(f > -1.0e300)) {
        v = 0.0;
        k = 0;
        return;
    }
    int kk = 0;
    if (f < -300.0) kk = (int)floor((f + 300.0) / 600.0);
    v = sd[1] * exp2(f - 600.0 * (double)kk);
    k = kk;
}

__device__ __forceinline__ void rescale(double &v, double &vp, int &k)
{
    if (k < 0 && fabs(v) > kBig) {
        v *= kShrink;
        vp *= kShrink;
        ++k;
    }
}

// Recurrence coefficients for target degree l (lambda_l from lambda_{l-1}, lambda_{l-2}):
//   lambda_l = alpha (x - m s'/((l-1) l)) lambda_{l-1} - beta lambda_{l-2}.
struct Coef {
    double alpha, beta, c0;  // c0 = alpha s m / ((l-1) l) for spin s >= 1, 0 for spin 0
};

__device__ __forceinline__ Coef make_coef(int l, int m, int s, int l0)
{
    Coef c;
    double dl = (double)l, dm = (double)m, ds = (double)s;
    double den = sqrt((dl * dl - dm * dm) * (dl * dl - ds * ds));
    c.alpha = sqrt((2.0 * dl + 1.0) * (2.0 * dl - 1.0)) * dl / den;
    if (l >= l0 + 2) {
        double dl1 = dl - 1.0;
        double num = sqrt((dl1 * dl1 - dm * dm) * (dl1 * dl1 - ds * ds));
        c.beta = sqrt((2.0 * dl + 1.0) / (2.0 * dl - 3.0)) * dl * num / (dl1 * den);
    } else {
        c.beta = 0.0;
    }
    // alpha (x -+ c) = fma(alpha, x, -+alpha c): one FMA per row variant in the recurrence
    c.c0 = (s != 0 && l >= 2) ? c.alpha * (ds * dm / ((dl - 1.0) * dl)) : 0.0;
    return c;
}

// Checkpoint tables of the single-precision rows (legendre_ck.cu): segment k of order m
// starts at row l0 + 128 k; per (segment, lane) the scaled pre-state (v_{l-1}, D_l) and its
// shift n (actual = stored * 2^(-64 n)).  Variant q = 0: s' = 0 (spin 0) or -2; q = 1: +2.
struct CkTab {
    const int64_t *segoff;
    const float2 *ck[2];
    const uint8_t *cn[2];
    // optional (NULL: every segment generated): per segment, bit g set when a lane of the
    // 64-lane group g has a non-zero stored state (legendre_ck.cu:gm_ck_masks)
    const unsigned long long *mask[2];
};
constexpr int kCkSeg = 128;

// Whether some lane of this CTA (lanes [j0, j0 + nl)) has a non-zero state at segment seg
// of either row variant: a CTA whose lanes all start the segment from zero gives exactly
// zero rows for its 128 rows and skips them (the decision is uniform over the CTA).
__device__ __forceinline__ bool ck_segment_active(const CkTab &tab, int nvar, int64_t seg, int64_t j0, int64_t nl,
                                                  int64_t nlanes)
{
    if (!tab.mask[0] || nlanes > 4096) return true;
    const int64_t j1 = (j0 + nl < nlanes ? j0 + nl : nlanes) - 1;
    const int g0 = (int)(j0 >> 6), g1 = (int)(j1 >> 6);
    const unsigned long long hi = g1 >= 63 ? ~0ull : ((1ull << (g1 + 1)) - 1ull);
    const unsigned long long bits = hi & ~((1ull << g0) - 1ull);
    unsigned long long mk = __ldg(tab.mask[0] + seg);
    if (nvar > 1 && tab.mask[1]) mk |= __ldg(tab.mask[1] + seg);
    return (mk & bits) != 0ull;
}

// Single-precision difference-form coefficients of row l (legendre_ck.cu): (c1, E for
// s' = -s, E for s' = +s, b); a segment's first row is the restart step (0, 0, 0, 1).
__device__ __forceinline__ float4 ck_coef(int l, int m, int s, int l0)
{
    if ((l - l0) % kCkSeg == 0) return make_float4(0.f, 0.f, 0.f, 1.f);
    const Coef c = make_coef(l, m, s, l0);
    const double e = c.alpha - c.beta - 1.0;
    return make_float4((float)c.alpha, (float)(e + c.c0), (float)(e - c.c0), (float)c.beta);
}

// One FP32 difference-form step, then the emitted value (scaled lanes: n > 0).
__device__ __forceinline__ float ck_step(float c1, float E, float b, float y, float &v, float &D, int &n,
                                         bool scaled)
{
    const float C = fmaf(c1, y, E);
    const float bD = b * D;
    D = fmaf(C, v, bD);
    v = v + D;
    if (!scaled) return v;
    const float out = v * (n == 0 ? 1.0f : (n == 1 ? 0x1p-64f : 0.0f));
    // a row grows a value by at most 2^8 (alpha <= sqrt(2m) + 1 at Nside <= 8192)
    if (n != 0 && fabsf(v) > 0x1p48f) {
        v *= 0x1p-64f;
        D *= 0x1p-64f;
        --n;
    }
    return out;
}

template <typename T, int V>
__device__ __forceinline__ T warp_reduce_scatter(T (&v)[V], int lane)
{
#pragma unroll
    for (int h = V / 2; h >= 1; h >>= 1) {
        const bool upper = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            T send = upper ? v[i] : v[i + h];
            T keep = upper ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    T r = v[0];
#pragma unroll
    for (int h = V; h < 32; h <<= 1) r += __shfl_xor_sync(0xffffffffu, r, h);
    return r;
}

__device__ __forceinline__ int64_t alm_index(int64_t lmax, int64_t l, int64_t m)
{
    return m * (2 * lmax + 1 - m) / 2 + l;
}

// ---------------------------------------------------------------- analysis

// NC components per CTA (spin 0: NC maps; spin 2: NC = 2, one (Q, U) pair).
// NV values per degree: spin 0: 2 NC; spin 2: 8.  LB degrees per reduce-scatter block.
//
// CK: the rows come from the single-precision difference form restarted from the checkpoint
// tables every 128 rows (mixed precision, spin 0 and 2) instead of the FP64 recurrence.
template <typename T, int SPIN, int NC, int R, bool CK>
__global__ void __launch_bounds__(kThreads) k_legendre_ana(
    int64_t nside, int64_t lmax, int64_t ncomp, const double *__restrict__ geom,
    const double *__restrict__ seeds, const T *__restrict__ rhs, double *__restrict__ alm,
    double scale, int spin, CkTab tab)
{
    constexpr int NV = SPIN == 0 ? 2 * NC : 8;
    constexpr int LB = 32 / NV;
    constexpr int NVAR = SPIN == 0 ? 1 : 2;
    static_assert(LB * NV == 32, "reduce-scatter width");
    static_assert(LB % 2 == 0 && kWindow % 2 == 0, "row parity is fixed by the row index");
    __shared__ Coef coef[kWindow];
    __shared__ float4 fcoef[kWindow];
    __shared__ double red[kWarps][kWindow * NV];

    const int64_t L = lmax + 1, nlanes = 2 * nside, nelem = L * (L + 1) / 2;
    const int m = blockIdx.y;
    const int64_t c0 = (int64_t)blockIdx.z * NC;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int sv = SPIN == 0 ? 0 : spin;   // the field's spin (SPIN = 2: any spin >= 1)
    const int l0 = m > sv ? m : sv;
    if (l0 > lmax) return;

    double x[R], v[NVAR][R], vp[NVAR][R];
    int kx[NVAR][R];
    float fy[R], fv[NVAR][R], fD[NVAR][R];
    int fn[NVAR][R];
    T rh[R][NC][4];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t j = (int64_t)blockIdx.x * kThreads * R + r * kThreads + threadIdx.x;
        const bool ok = j < nlanes;
        x[r] = ok ? geom[j] : 0.0;
        fy[r] = ok ? (float)(geom[j] - 1.0) : 0.0f;
        const double ls = ok ? geom[nlanes + j] : 0.0, lc = ok ? geom[2 * nlanes + j] : 0.0;
#pragma unroll
        for (int q = 0; q < NVAR; ++q) {
            // seed variants: s' = -s (lambda+), then s' = +s (lambda-, times (-1)^s)
            const int var = SPIN == 0 ? 0 : seed_variant(sv) + q;
            if (!CK && ok) {
                seed_lane(seeds + ((int64_t)var * L + m) * 4, ls, lc, v[q][r], kx[q][r]);
            } else {
                v[q][r] = 0.0;
                kx[q][r] = 0;
            }
            vp[q][r] = 0.0;
            fv[q][r] = fD[q][r] = 0.0f;
            fn[q][r] = 0;
        }
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int e = 0; e < 4; ++e)
                rh[r][c][e] = (ok && c0 + c < ncomp)
                                  ? rhs[(((int64_t)m * nlanes + j) * ncomp + c0 + c) * 4 + e]
                                  : (T)0;
    }

    // The southern ring's rows are the northern ones times (-1)^(l + m + s) (for spin s,
    // with the (-1)^s of the +s variant in its seed).  The rows of a reduce-scatter block
    // start at l0 + (an even offset: kWindow and LB are even), so that parity in unrolled
    // row s is ((l0 + m + sv) + s) & 1.  With the two hemisphere halves of the right-hand
    // side swapped once here when l0 + m + sv is odd, row s takes half s & 1, chosen at
    // compile time instead of by selects on every element.
    if ((l0 + m + sv) & 1) {
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                T t0 = rh[r][c][0], t1 = rh[r][c][1];
                rh[r][c][0] = rh[r][c][2];
                rh[r][c][1] = rh[r][c][3];
                rh[r][c][2] = t0;
                rh[r][c][3] = t1;
            }
    }
    for (int lb = l0; lb < L; lb += kWindow) {
        if (CK && (lb - l0) % kCkSeg == 0 &&
            !ck_segment_active(tab, NVAR, tab.segoff[m] + (lb - l0) / kCkSeg,
                               (int64_t)blockIdx.x * kThreads * R, (int64_t)kThreads * R, nlanes)) {
            lb += kCkSeg - kWindow;   // the segment's rows are zero on all lanes of this CTA
            continue;
        }
        if (threadIdx.x < kWindow) {
            const int l = lb + threadIdx.x;
            if (CK) fcoef[threadIdx.x] = ck_coef(l, m, sv, l0);
            else coef[threadIdx.x] = make_coef(l, m, sv, l0);
        }
        bool scaled = false;
        if (CK) {
            if ((lb - l0) % kCkSeg == 0) {
                // a new segment: the lane states restart from the checkpoint table
                const int64_t seg = tab.segoff[m] + (lb - l0) / kCkSeg;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int64_t j = (int64_t)blockIdx.x * kThreads * R + r * kThreads + threadIdx.x;
#pragma unroll
                    for (int q = 0; q < NVAR; ++q) {
                        float2 st = make_float2(0.f, 0.f);
                        int n = 0;
                        if (j < nlanes) {
                            st = __ldg(tab.ck[q] + seg * nlanes + j);
                            n = __ldg(tab.cn[q] + seg * nlanes + j);
                        }
                        fv[q][r] = st.x;
                        fD[q][r] = st.y;
                        fn[q][r] = n;
                    }
                }
            }
            int any = 0;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int q = 0; q < NVAR; ++q) any |= fn[q][r];
            scaled = __any_sync(0xffffffffu, any != 0);
        }
        __syncthreads();
#pragma unroll 1
        for (int i = 0; i < kWindow; i += LB) {
            T acc[LB * NV];
#pragma unroll
            for (int q = 0; q < LB * NV; ++q) acc[q] = (T)0;
#pragma unroll
            for (int s = 0; s < LB; ++s) {
                const int l = lb + i + s;
                if (l < L) {
                    float fval[NVAR][R];
                    if (CK) {
                        const float4 cq = fcoef[i + s];
#pragma unroll
                        for (int r = 0; r < R; ++r)
#pragma unroll
                            for (int q = 0; q < NVAR; ++q)
                                fval[q][r] = ck_step(cq.x, q == 0 ? cq.y : cq.z, cq.w, fy[r], fv[q][r],
                                                     fD[q][r], fn[q][r], scaled);
                    } else if (l > l0) {
                        const Coef cf = coef[i + s];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            if (SPIN == 0) {
                                double nv = fma(cf.alpha * x[r], v[0][r], -cf.beta * vp[0][r]);
                                vp[0][r] = v[0][r];
                                v[0][r] = nv;
                                rescale(v[0][r], vp[0][r], kx[0][r]);
                            } else {
                                // s' = -2: alpha (x - m s'/((l-1)l)) = fma(alpha, x, c0);
                                // s' = +2: fma(alpha, x, -c0)  (c0 carries alpha)
                                double nva = fma(fma(cf.alpha, x[r], cf.c0), v[0][r], -cf.beta * vp[0][r]);
                                double nvb = fma(fma(cf.alpha, x[r], -cf.c0), v[1][r], -cf.beta * vp[1][r]);
                                vp[0][r] = v[0][r];
                                v[0][r] = nva;
                                vp[1][r] = v[1][r];
                                v[1][r] = nvb;
                                rescale(v[0][r], vp[0][r], kx[0][r]);
                                rescale(v[1][r], vp[1][r], kx[1][r]);
                            }
                        }
                    }
                    const int par = s & 1;   // relative to (l0 + m + sv) & 1, see above
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (SPIN == 0) {
                            const T val = CK ? (T)fval[0][r] : (kx[0][r] == 0 ? (T)v[0][r] : (T)0);
#pragma unroll
                            for (int c = 0; c < NC; ++c) {
                                const T hr = par ? rh[r][c][2] : rh[r][c][0];
                                const T hi = par ? rh[r][c][3] : rh[r][c][1];
                                acc[s * NV + 2 * c] += val * hr;
                                acc[s * NV + 2 * c + 1] += val * hi;
                            }
                        } else {
                            T f1, f2;
                            if (CK) {
                                f1 = (T)(0.5f * (fval[0][r] + fval[NVAR - 1][r]));
                                f2 = (T)(0.5f * (fval[0][r] - fval[NVAR - 1][r]));
                            } else {
                                const double lp = kx[0][r] == 0 ? v[0][r] : 0.0;
                                const double lm = kx[NVAR - 1][r] == 0 ? v[NVAR - 1][r] : 0.0;
                                f1 = (T)(0.5 * (lp + lm));
                                f2 = (T)(0.5 * (lp - lm));
                            }
                            // same-parity side P = Sum (even) / Diff (odd); other side D
                            const T qpr = par ? rh[r][0][2] : rh[r][0][0];
                            const T qpi = par ? rh[r][0][3] : rh[r][0][1];
                            const T upr = par ? rh[r][1][2] : rh[r][1][0];
                            const T upi = par ? rh[r][1][3] : rh[r][1][1];
                            const T qdr = par ? rh[r][0][0] : rh[r][0][2];
                            const T qdi = par ? rh[r][0][1] : rh[r][0][3];
                            const T udr = par ? rh[r][1][0] : rh[r][1][2];
                            const T udi = par ? rh[r][1][1] : rh[r][1][3];
                            acc[s * NV + 0] += f1 * qpr;
                            acc[s * NV + 1] += f1 * qpi;
                            acc[s * NV + 2] += f1 * upr;
                            acc[s * NV + 3] += f1 * upi;
                            acc[s * NV + 4] += f2 * qdr;
                            acc[s * NV + 5] += f2 * qdi;
                            acc[s * NV + 6] += f2 * udr;
                            acc[s * NV + 7] += f2 * udi;
                        }
                    }
                }
            }
            const T tot = warp_reduce_scatter<T, LB * NV>(acc, lane);
            red[warp][i * NV + lane] = (double)tot;
        }
        __syncthreads();
        if (threadIdx.x < kWindow) {
            const int l = lb + threadIdx.x;
            if (l < L) {
                double sv[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) {
                    double t = 0.0;
#pragma unroll
                    for (int w = 0; w < kWarps; ++w) t += red[w][threadIdx.x * NV + q];
                    sv[q] = t;
                }
                const int64_t idx = alm_index(lmax, l, m);
                if (SPIN == 0) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        if (c0 + c < ncomp) {
                            double *a = alm + 2 * ((c0 + c) * nelem + idx);
                            atomicAdd(a, scale * sv[2 * c]);
                            atomicAdd(a + 1, scale * sv[2 * c + 1]);
                        }
                    }
                } else {
                    // E = -(a1 + i-rotated a2), B likewise (see the docstring of gm_legendre_analysis)
                    const int64_t f = c0 / 2;
                    double *e = alm + 2 * ((2 * f) * nelem + idx);
                    double *b = alm + 2 * ((2 * f + 1) * nelem + idx);
                    atomicAdd(e, -scale * (sv[0] - sv[7]));
                    atomicAdd(e + 1, -scale * (sv[1] + sv[6]));
                    atomicAdd(b, -scale * (sv[2] + sv[5]));
                    atomicAdd(b + 1, -scale * (sv[3] - sv[4]));
                }
            }
        }
    }
}

// ---------------------------------------------------------------- synthesis

template <typename T, int SPIN, int NC, int R, bool CK>
__global__ void __launch_bounds__(kThreads) k_legendre_syn(
    int64_t nside, int64_t lmax, int64_t ncomp, const double *__restrict__ geom,
    const double *__restrict__ seeds, const double *__restrict__ alm, T *__restrict__ syn,
    int spin, CkTab tab)
{
    constexpr int NVAR = SPIN == 0 ? 1 : 2;
    constexpr int NA = SPIN == 0 ? NC : 2;  // complex alm rows per degree (maps, or E and B)
    constexpr int NACC = SPIN == 0 ? 4 * NC : 16;
    __shared__ Coef coef[2][kWindow];
    __shared__ float4 fcoef[2][kWindow];
    __shared__ T aw[2][kWindow][NA][2];

    const int64_t L = lmax + 1, nlanes = 2 * nside, nelem = L * (L + 1) / 2;
    const int m = blockIdx.y;
    const int64_t c0 = (int64_t)blockIdx.z * NC;
    const int sv = SPIN == 0 ? 0 : spin;
    const int l0 = m > sv ? m : sv;

    double x[R], v[NVAR][R], vp[NVAR][R];
    int kx[NVAR][R];
    float fy[R], fv[NVAR][R], fD[NVAR][R];
    int fn[NVAR][R];
    T acc[R][NACC];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t j = (int64_t)blockIdx.x * kThreads * R + r * kThreads + threadIdx.x;
        const bool ok = j < nlanes && l0 <= lmax;
        x[r] = ok ? geom[j] : 0.0;
        fy[r] = ok ? (float)(geom[j] - 1.0) : 0.0f;
        const double ls = ok ? geom[nlanes + j] : 0.0, lc = ok ? geom[2 * nlanes + j] : 0.0;
#pragma unroll
        for (int q = 0; q < NVAR; ++q) {
            const int var = SPIN == 0 ? 0 : seed_variant(sv) + q;
            if (!CK && ok) {
                seed_lane(seeds + ((int64_t)var * L + m) * 4, ls, lc, v[q][r], kx[q][r]);
            } else {
                v[q][r] = 0.0;
                kx[q][r] = 0;
            }
            vp[q][r] = 0.0;
            fv[q][r] = fD[q][r] = 0.0f;
            fn[q][r] = 0;
        }
#pragma unroll
        for (int q = 0; q < NACC; ++q) acc[r][q] = (T)0;
    }

    int buf = 0;
    for (int lb = l0; lb < L; lb += kWindow, buf ^= 1) {
        if (CK && (lb - l0) % kCkSeg == 0 &&
            !ck_segment_active(tab, NVAR, tab.segoff[m] + (lb - l0) / kCkSeg,
                               (int64_t)blockIdx.x * kThreads * R, (int64_t)kThreads * R, nlanes)) {
            // the segment's rows are zero on all lanes of this CTA; the next window that runs
            // takes the other buffer, as it would have after this one
            lb += kCkSeg - kWindow;
            buf ^= 1;
            continue;
        }
        bool scaled = false;
        if (CK) {
            if ((lb - l0) % kCkSeg == 0) {
                // a new segment: the lane states restart from the checkpoint table
                const int64_t seg = tab.segoff[m] + (lb - l0) / kCkSeg;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int64_t j = (int64_t)blockIdx.x * kThreads * R + r * kThreads + threadIdx.x;
#pragma unroll
                    for (int q = 0; q < NVAR; ++q) {
                        float2 st = make_float2(0.f, 0.f);
                        int n = 0;
                        if (j < nlanes) {
                            st = __ldg(tab.ck[q] + seg * nlanes + j);
                            n = __ldg(tab.cn[q] + seg * nlanes + j);
                        }
                        fv[q][r] = st.x;
                        fD[q][r] = st.y;
                        fn[q][r] = n;
                    }
                }
            }
            int any = 0;
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int q = 0; q < NVAR; ++q) any |= fn[q][r];
            scaled = __any_sync(0xffffffffu, any != 0);
        }
        if (threadIdx.x < kWindow) {
            const int l = lb + threadIdx.x;
            if (CK) fcoef[buf][threadIdx.x] = ck_coef(l, m, sv, l0);
            else coef[buf][threadIdx.x] = make_coef(l, m, sv, l0);
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                T re = 0, im = 0;
                if (l < L) {
                    const int64_t row = SPIN == 0 ? c0 + a : c0 + a;  // spin 2: rows E, B of field c0/2
                    if (row < ncomp) {
                        const double *p = alm + 2 * (row * nelem + alm_index(lmax, l, m));
                        re = (T)p[0];
                        im = (T)p[1];
                    }
                }
                aw[buf][threadIdx.x][a][0] = re;
                aw[buf][threadIdx.x][a][1] = im;
            }
        }
        __syncthreads();
        const int lend = (lb + kWindow < L) ? kWindow : (int)(L - lb);
        // blocks start at l0 + multiples of kWindow (even), so row s has the parity of
        // l + m relative to (l0 + m) & 1 given by s & 1: rows go in pairs and each
        // accumulates into its half at compile time (no multiplications by zero); the
        // halves are put in true parity order before the output
#pragma unroll 2
        for (int s0 = 0; s0 < lend; s0 += 2) {
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int s = s0 + hh;
                if (s >= lend) break;
                const int l = lb + s;
                float fval[NVAR][R];
                if (CK) {
                    const float4 cq = fcoef[buf][s];
#pragma unroll
                    for (int r = 0; r < R; ++r)
#pragma unroll
                        for (int q = 0; q < NVAR; ++q)
                            fval[q][r] = ck_step(cq.x, q == 0 ? cq.y : cq.z, cq.w, fy[r], fv[q][r], fD[q][r],
                                                 fn[q][r], scaled);
                } else if (l > l0) {
                    const Coef cf = coef[buf][s];
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (SPIN == 0) {
                            double nv = fma(cf.alpha * x[r], v[0][r], -cf.beta * vp[0][r]);
                            vp[0][r] = v[0][r];
                            v[0][r] = nv;
                            rescale(v[0][r], vp[0][r], kx[0][r]);
                        } else {
                            double nva = fma(fma(cf.alpha, x[r], cf.c0), v[0][r], -cf.beta * vp[0][r]);
                            double nvb = fma(fma(cf.alpha, x[r], -cf.c0), v[1][r], -cf.beta * vp[1][r]);
                            vp[0][r] = v[0][r];
                            v[0][r] = nva;
                            vp[1][r] = v[1][r];
                            v[1][r] = nvb;
                            rescale(v[0][r], vp[0][r], kx[0][r]);
                            rescale(v[1][r], vp[1][r], kx[1][r]);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (SPIN == 0) {
                        const T val = CK ? (T)fval[0][r] : (kx[0][r] == 0 ? (T)v[0][r] : (T)0);
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            acc[r][4 * c + 2 * hh] += val * aw[buf][s][c][0];
                            acc[r][4 * c + 2 * hh + 1] += val * aw[buf][s][c][1];
                        }
                    } else {
                        T f1, f2;
                        if (CK) {
                            f1 = (T)(0.5f * (fval[0][r] + fval[NVAR - 1][r]));
                            f2 = (T)(0.5f * (fval[0][r] - fval[NVAR - 1][r]));
                        } else {
                            const double lp = kx[0][r] == 0 ? v[0][r] : 0.0;
                            const double lm = kx[NVAR - 1][r] == 0 ? v[NVAR - 1][r] : 0.0;
                            f1 = (T)(0.5 * (lp + lm));
                            f2 = (T)(0.5 * (lp - lm));
                        }
                        const T er = aw[buf][s][0][0], ei = aw[buf][s][0][1];
                        const T br = aw[buf][s][1][0], bi = aw[buf][s][1][1];
                        // per parity: [S1E re, im, S1B re, im, S2E re, im, S2B re, im]
                        T *a = &acc[r][8 * hh];
                        a[0] += f1 * er;
                        a[1] += f1 * ei;
                        a[2] += f1 * br;
                        a[3] += f1 * bi;
                        a[4] += f2 * er;
                        a[5] += f2 * ei;
                        a[6] += f2 * br;
                        a[7] += f2 * bi;
                    }
                }
            }
        }
    }

    if ((l0 + m + sv) & 1) {
        // the even rows of the blocks had odd l + m + s: swap the halves into parity order
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (SPIN == 0) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const T t0 = acc[r][4 * c], t1 = acc[r][4 * c + 1];
                    acc[r][4 * c] = acc[r][4 * c + 2];
                    acc[r][4 * c + 1] = acc[r][4 * c + 3];
                    acc[r][4 * c + 2] = t0;
                    acc[r][4 * c + 3] = t1;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const T t = acc[r][q];
                    acc[r][q] = acc[r][8 + q];
                    acc[r][8 + q] = t;
                }
            }
        }
    }

#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int64_t j = (int64_t)blockIdx.x * kThreads * R + r * kThreads + threadIdx.x;
        if (j >= nlanes) continue;
        if (SPIN == 0) {
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (c0 + c >= ncomp) continue;
                T *o = syn + (((int64_t)m * nlanes + j) * ncomp + c0 + c) * 4;
                const T er = acc[r][4 * c], ei = acc[r][4 * c + 1];
                const T orr = acc[r][4 * c + 2], oi = acc[r][4 * c + 3];
                o[0] = er + orr;
                o[1] = ei + oi;
                o[2] = er - orr;
                o[3] = ei - oi;
            }
        } else {
            const T *e = &acc[r][0];
            const T *od = &acc[r][8];
            // north: sums; south: F1 -> e - o, F2 -> o - e
            T s1e_n[2] = {e[0] + od[0], e[1] + od[1]}, s1b_n[2] = {e[2] + od[2], e[3] + od[3]};
            T s2e_n[2] = {e[4] + od[4], e[5] + od[5]}, s2b_n[2] = {e[6] + od[6], e[7] + od[7]};
            T s1e_s[2] = {e[0] - od[0], e[1] - od[1]}, s1b_s[2] = {e[2] - od[2], e[3] - od[3]};
            T s2e_s[2] = {od[4] - e[4], od[5] - e[5]}, s2b_s[2] = {od[6] - e[6], od[7] - e[7]};
            T *oq = syn + (((int64_t)m * nlanes + j) * ncomp + c0) * 4;
            T *ou = oq + 4;
            // Q~ = -(S1E + i S2B), U~ = -(S1B - i S2E)
            oq[0] = -(s1e_n[0] - s2b_n[1]);
            oq[1] = -(s1e_n[1] + s2b_n[0]);
            oq[2] = -(s1e_s[0] - s2b_s[1]);
            oq[3] = -(s1e_s[1] + s2b_s[0]);
            ou[0] = -(s1b_n[0] + s2e_n[1]);
            ou[1] = -(s1b_n[1] - s2e_n[0]);
            ou[2] = -(s1b_s[0] + s2e_s[1]);
            ou[3] = -(s1b_s[1] - s2e_s[0]);
        }
    }
}

}  // namespace gm

using namespace gm;

extern "C" int64_t gm_seed_table_len(int64_t L) { return (2 * kMaxSpin + 1) * 4 * L; }

template <typename T, int SPIN, int NC, int R>
static int launch_ana(int spin, int64_t nside, int64_t lmax, int64_t ncomp, const double *geom,
                      const double *seeds, const void *rhs, double *alm, double scale,
                      cudaStream_t s, const CkTab *tab = nullptr)
{
    const int64_t nlanes = 2 * nside;
    dim3 grid((unsigned)((nlanes + kThreads * R - 1) / (kThreads * R)), (unsigned)(lmax + 1),
              (unsigned)((ncomp + NC - 1) / NC));
    if (tab)
        k_legendre_ana<float, SPIN, NC, R, true><<<grid, kThreads, 0, s>>>(
            nside, lmax, ncomp, geom, seeds, (const float *)rhs, alm, scale, spin, *tab);
    else
        k_legendre_ana<T, SPIN, NC, R, false><<<grid, kThreads, 0, s>>>(
            nside, lmax, ncomp, geom, seeds, (const T *)rhs, alm, scale, spin, CkTab{});
    return check_launch("gm_legendre_analysis");
}

template <typename T, int SPIN, int NC, int R>
static int launch_syn(int spin, int64_t nside, int64_t lmax, int64_t ncomp, const double *geom,
                      const double *seeds, const double *alm, void *syn, cudaStream_t s,
                      const CkTab *tab = nullptr)
{
    const int64_t nlanes = 2 * nside;
    dim3 grid((unsigned)((nlanes + kThreads * R - 1) / (kThreads * R)), (unsigned)(lmax + 1),
              (unsigned)((ncomp + NC - 1) / NC));
    if (tab)
        k_legendre_syn<float, SPIN, NC, R, true><<<grid, kThreads, 0, s>>>(
            nside, lmax, ncomp, geom, seeds, alm, (float *)syn, spin, *tab);
    else
        k_legendre_syn<T, SPIN, NC, R, false><<<grid, kThreads, 0, s>>>(
            nside, lmax, ncomp, geom, seeds, alm, (T *)syn, spin, CkTab{});
    return check_launch("gm_legendre_synthesis");
}

template <typename T>
static int dispatch_ana(int spin, int64_t nside, int64_t lmax, int64_t ncomp, const double *geom,
                        const double *seeds, const void *rhs, double *alm, double scale,
                        cudaStream_t s, const CkTab *tab = nullptr)
{
    if (spin == 0) {
        if (ncomp == 1)
            return launch_ana<T, 0, 1, 4>(spin, nside, lmax, ncomp, geom, seeds, rhs, alm, scale, s, tab);
        if (ncomp == 2)
            return launch_ana<T, 0, 2, 4>(spin, nside, lmax, ncomp, geom, seeds, rhs, alm, scale, s, tab);
        return launch_ana<T, 0, 4, 2>(spin, nside, lmax, ncomp, geom, seeds, rhs, alm, scale, s, tab);
    }
    return launch_ana<T, 2, 2, 2>(spin, nside, lmax, ncomp, geom, seeds, rhs, alm, scale, s, tab);
}

template <typename T>
static int dispatch_syn(int spin, int64_t nside, int64_t lmax, int64_t ncomp, const double *geom,
                        const double *seeds, const double *alm, void *syn, cudaStream_t s,
                        const CkTab *tab = nullptr)
{
    if (spin == 0) {
        if (ncomp == 1) return launch_syn<T, 0, 1, 2>(spin, nside, lmax, ncomp, geom, seeds, alm, syn, s, tab);
        if (ncomp == 2) return launch_syn<T, 0, 2, 2>(spin, nside, lmax, ncomp, geom, seeds, alm, syn, s, tab);
        return launch_syn<T, 0, 4, 1>(spin, nside, lmax, ncomp, geom, seeds, alm, syn, s, tab);
    }
    return launch_syn<T, 2, 2, 2>(spin, nside, lmax, ncomp, geom, seeds, alm, syn, s, tab);
}

// Tile shapes the autotuner chooses from: (NC, R) = (components per CTA, lanes per thread).
// Spin 0 takes NC in {1, 2, 4, 8} (the reduce-scatter needs 2 NC to divide 32); spin 2
// handles one (Q, U) pair per CTA (NC = 2).  Index -1 selects the built-in heuristic.
// The last tile of each list (8 lanes per thread: a reduce-scatter tree per 8 rows shared by
// 64 elements of a thread instead of 32) is compiled for single precision only; the FP64
// kernels run it as the tile with 4 lanes per thread.
static const int kTiles0[][2] = {{1, 1}, {1, 2}, {1, 4}, {2, 1}, {2, 2}, {2, 4}, {4, 1}, {4, 2}, {8, 1}, {2, 8}};
static const int kTiles2[][2] = {{2, 1}, {2, 2}, {2, 4}, {2, 8}};
constexpr int kNTiles0 = sizeof(kTiles0) / sizeof(kTiles0[0]);
constexpr int kNTiles2 = sizeof(kTiles2) / sizeof(kTiles2[0]);

template <typename T>
static int tile_ana(int spin, int tile, int64_t nside, int64_t lmax, int64_t ncomp,
                    const double *geom, const double *seeds, const void *rhs, double *alm,
                    double scale, cudaStream_t s, const CkTab *tab = nullptr)
{
#define GM_ANA(SP, NC, R) return launch_ana<T, SP, NC, R>(spin, nside, lmax, ncomp, geom, seeds, rhs, alm, scale, s, tab)
    if (spin == 0) {
        switch (tile) {
        case 0: GM_ANA(0, 1, 1);
        case 1: GM_ANA(0, 1, 2);
        case 2: GM_ANA(0, 1, 4);
        case 3: GM_ANA(0, 2, 1);
        case 4: GM_ANA(0, 2, 2);
        case 5: GM_ANA(0, 2, 4);
        case 6: GM_ANA(0, 4, 1);
        case 7: GM_ANA(0, 4, 2);
        case 8: GM_ANA(0, 8, 1);
        case 9:
            if constexpr (sizeof(T) == 8) { GM_ANA(0, 2, 4); } else { GM_ANA(0, 2, 8); }
        default: return GM_ERR_BAD_SHAPE;
        }
    }
    switch (tile) {
    case 0: GM_ANA(2, 2, 1);
    case 1: GM_ANA(2, 2, 2);
    case 2: GM_ANA(2, 2, 4);
    case 3:
        if constexpr (sizeof(T) == 8) { GM_ANA(2, 2, 4); } else { GM_ANA(2, 2, 8); }
    default: return GM_ERR_BAD_SHAPE;
    }
#undef GM_ANA
}

template <typename T>
static int tile_syn(int spin, int tile, int64_t nside, int64_t lmax, int64_t ncomp,
                    const double *geom, const double *seeds, const double *alm, void *syn,
                    cudaStream_t s, const CkTab *tab = nullptr)
{
#define GM_SYN(SP, NC, R) return launch_syn<T, SP, NC, R>(spin, nside, lmax, ncomp, geom, seeds, alm, syn, s, tab)
    if (spin == 0) {
        switch (tile) {
        case 0: GM_SYN(0, 1, 1);
        case 1: GM_SYN(0, 1, 2);
        case 2: GM_SYN(0, 1, 4);
        case 3: GM_SYN(0, 2, 1);
        case 4: GM_SYN(0, 2, 2);
        case 5: GM_SYN(0, 2, 4);
        case 6: GM_SYN(0, 4, 1);
        case 7: GM_SYN(0, 4, 2);
        case 8: GM_SYN(0, 8, 1);
        case 9:
            if constexpr (sizeof(T) == 8) { GM_SYN(0, 2, 4); } else { GM_SYN(0, 2, 8); }
        default: return GM_ERR_BAD_SHAPE;
        }
    }
    switch (tile) {
    case 0: GM_SYN(2, 2, 1);
    case 1: GM_SYN(2, 2, 2);
    case 2: GM_SYN(2, 2, 4);
    case 3:
        if constexpr (sizeof(T) == 8) { GM_SYN(2, 2, 4); } else { GM_SYN(2, 2, 8); }
    default: return GM_ERR_BAD_SHAPE;
    }
#undef GM_SYN
}

extern "C" int gm_legendre_tiles(int spin, int32_t *nc_r, int capacity)
{
    if (spin < 0 || spin > kMaxSpin) return -1;
    const int n = spin == 0 ? kNTiles0 : kNTiles2;
    for (int i = 0; i < n && i < capacity; ++i) {
        nc_r[2 * i] = spin == 0 ? kTiles0[i][0] : kTiles2[i][0];
        nc_r[2 * i + 1] = spin == 0 ? kTiles0[i][1] : kTiles2[i][1];
    }
    return n;
}

extern "C" int gm_legendre_analysis_tile(int precision, int spin, int64_t nside, int64_t lmax,
                                         int64_t ncomp, const double *lane_geom, const double *seeds,
                                         const void *rhs, double *alm, double scale, int tile,
                                         void *stream)
{
    if (nside < 1 || lmax < 0 || lmax + 1 > 65535 || ncomp < 1 || ncomp > 65535)
        return GM_ERR_BAD_SHAPE;
    if (spin < 0 || spin > kMaxSpin) return GM_ERR_UNSUPPORTED;
    if (spin != 0 && (ncomp % 2)) return GM_ERR_BAD_SHAPE;
    if (tile < -1 || tile >= (spin == 0 ? kNTiles0 : kNTiles2)) return GM_ERR_BAD_SHAPE;
    if (!lane_geom || !seeds || !rhs || !alm) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        return tile < 0 ? dispatch_ana<double>(spin, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s)
                        : tile_ana<double>(spin, tile, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s);
    if (precision == GM_MIXED)
        return tile < 0 ? dispatch_ana<float>(spin, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s)
                        : tile_ana<float>(spin, tile, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s);
    return GM_ERR_UNSUPPORTED;
}

extern "C" int gm_legendre_synthesis_tile(int precision, int spin, int64_t nside, int64_t lmax,
                                          int64_t ncomp, const double *lane_geom, const double *seeds,
                                          const double *alm, void *syn, int tile, void *stream)
{
    if (nside < 1 || lmax < 0 || lmax + 1 > 65535 || ncomp < 1 || ncomp > 65535)
        return GM_ERR_BAD_SHAPE;
    if (spin < 0 || spin > kMaxSpin) return GM_ERR_UNSUPPORTED;
    if (spin != 0 && (ncomp % 2)) return GM_ERR_BAD_SHAPE;
    if (tile < -1 || tile >= (spin == 0 ? kNTiles0 : kNTiles2)) return GM_ERR_BAD_SHAPE;
    if (!lane_geom || !seeds || !alm || !syn) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        return tile < 0 ? dispatch_syn<double>(spin, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s)
                        : tile_syn<double>(spin, tile, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s);
    if (precision == GM_MIXED)
        return tile < 0 ? dispatch_syn<float>(spin, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s)
                        : tile_syn<float>(spin, tile, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s);
    return GM_ERR_UNSUPPORTED;
}

extern "C" int gm_legendre_analysis(int precision, int spin, int64_t nside, int64_t lmax,
                                    int64_t ncomp, const double *lane_geom, const double *seeds,
                                    const void *rhs, double *alm, double scale, void *stream)
{
    if (nside < 1 || lmax < 0 || lmax + 1 > 65535 || ncomp < 1 || ncomp > 65535)
        return GM_ERR_BAD_SHAPE;
    if (spin < 0 || spin > kMaxSpin) return GM_ERR_UNSUPPORTED;
    if (spin != 0 && (ncomp % 2)) return GM_ERR_BAD_SHAPE;
    if (!lane_geom || !seeds || !rhs || !alm) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        return dispatch_ana<double>(spin, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s);
    if (precision == GM_MIXED)
        return dispatch_ana<float>(spin, nside, lmax, ncomp, lane_geom, seeds, rhs, alm, scale, s);
    return GM_ERR_UNSUPPORTED;
}

extern "C" int gm_legendre_synthesis(int precision, int spin, int64_t nside, int64_t lmax,
                                     int64_t ncomp, const double *lane_geom, const double *seeds,
                                     const double *alm, void *syn, void *stream)
{
    if (nside < 1 || lmax < 0 || lmax + 1 > 65535 || ncomp < 1 || ncomp > 65535)
        return GM_ERR_BAD_SHAPE;
    if (spin < 0 || spin > kMaxSpin) return GM_ERR_UNSUPPORTED;
    if (spin != 0 && (ncomp % 2)) return GM_ERR_BAD_SHAPE;
    if (!lane_geom || !seeds || !alm || !syn) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        return dispatch_syn<double>(spin, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s);
    if (precision == GM_MIXED)
        return dispatch_syn<float>(spin, nside, lmax, ncomp, lane_geom, seeds, alm, syn, s);
    return GM_ERR_UNSUPPORTED;
}

// Mixed-precision spin-0 / spin-2 transforms with the checkpointed single-precision rows.
static int ck_args_ok(int spin, int64_t nside, int64_t lmax, int64_t ncomp, int tile)
{
    if (nside < 1 || lmax < 2 || lmax + 1 > 65535 || ncomp < 1 || ncomp > 65535) return GM_ERR_BAD_SHAPE;
    if (spin != 0 && spin != 2) return GM_ERR_UNSUPPORTED;
    if (spin == 2 && (ncomp % 2)) return GM_ERR_BAD_SHAPE;
    if (tile < -1 || tile >= (spin == 0 ? kNTiles0 : kNTiles2)) return GM_ERR_BAD_SHAPE;
    return GM_OK;
}

static CkTab ck_tab(const int64_t *segoff, const void *ck_a, const uint8_t *cn_a, const void *ck_b,
                    const uint8_t *cn_b, const uint64_t *mask_a, const uint64_t *mask_b)
{
    CkTab t;
    t.segoff = segoff;
    t.ck[0] = (const float2 *)ck_a;
    t.cn[0] = cn_a;
    t.ck[1] = (const float2 *)ck_b;
    t.cn[1] = cn_b;
    // both variants' masks or neither
    const bool masked = mask_a && (mask_b || ck_b == nullptr);
    t.mask[0] = masked ? (const unsigned long long *)mask_a : nullptr;
    t.mask[1] = masked ? (const unsigned long long *)mask_b : nullptr;
    return t;
}

extern "C" int gm_legendre_analysis_ck(int spin, int64_t nside, int64_t lmax, int64_t ncomp,
                                       const double *lane_geom, const void *rhs, double *alm,
                                       double scale, const int64_t *segoff, const void *ck_a,
                                       const uint8_t *cn_a, const void *ck_b, const uint8_t *cn_b,
                                       const uint64_t *mask_a, const uint64_t *mask_b, int tile, void *stream)
{
    const int st = ck_args_ok(spin, nside, lmax, ncomp, tile);
    if (st != GM_OK) return st;
    if (!lane_geom || !rhs || !alm || !segoff || !ck_a || !cn_a || (spin == 2 && (!ck_b || !cn_b)))
        return GM_ERR_BAD_PTR;
    const CkTab tab = ck_tab(segoff, ck_a, cn_a, spin == 2 ? ck_b : nullptr, cn_b, mask_a, spin == 2 ? mask_b : nullptr);
    cudaStream_t s = as_stream(stream);
    return tile < 0 ? dispatch_ana<float>(spin, nside, lmax, ncomp, lane_geom, nullptr, rhs, alm, scale, s, &tab)
                    : tile_ana<float>(spin, tile, nside, lmax, ncomp, lane_geom, nullptr, rhs, alm, scale, s, &tab);
}

extern "C" int gm_legendre_synthesis_ck(int spin, int64_t nside, int64_t lmax, int64_t ncomp,
                                        const double *lane_geom, const double *alm, void *syn,
                                        const int64_t *segoff, const void *ck_a, const uint8_t *cn_a,
                                        const void *ck_b, const uint8_t *cn_b, const uint64_t *mask_a,
                                        const uint64_t *mask_b, int tile, void *stream)
{
    const int st = ck_args_ok(spin, nside, lmax, ncomp, tile);
    if (st != GM_OK) return st;
    if (!lane_geom || !alm || !syn || !segoff || !ck_a || !cn_a || (spin == 2 && (!ck_b || !cn_b)))
        return GM_ERR_BAD_PTR;
    const CkTab tab = ck_tab(segoff, ck_a, cn_a, spin == 2 ? ck_b : nullptr, cn_b, mask_a, spin == 2 ? mask_b : nullptr);
    cudaStream_t s = as_stream(stream);
    return tile < 0 ? dispatch_syn<float>(spin, nside, lmax, ncomp, lane_geom, nullptr, alm, syn, s, &tab)
                    : tile_syn<float>(spin, tile, nside, lmax, ncomp, lane_geom, nullptr, alm, syn, s, &tab);
}
