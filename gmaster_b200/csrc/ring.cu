// Azimuthal (ring) stage of the HEALPix spherical-harmonic transforms, sm_100a.
//
// One CTA transforms one ring of one map component entirely in shared memory:
// a real ring of nphi = 4i samples is packed into a complex sequence of length
// h = nphi/2 (even samples real, odd samples imaginary), transformed by a
// self-sorting Stockham FFT of mixed radix (4, 2, then odd primes; a generic
// radix-p stage for large prime factors), and unpacked.  Loads and stores of
// pixels and spectra are coalesced along the ring / along m.
//
// Replaces the reference's XLA-lowered ring stage (gmaster/_sht/rings.py:251-299
// forward, :477-524 inverse: a cuFFT of the equatorial belt plus Bluestein chirp-Z
// convolutions for the polar caps) and its ring-fold residual kernel
// (gmaster/_native/cuda/march_v2.cu:426-493).
#include <math.h>

#include <type_traits>

#include "gm_common.cuh"

namespace gm {

// ---------------------------------------------------------------- twiddles

// tw64[i(i-1) + k] = exp(-2 pi i k / (4 i)), k < 2 i, followed by the float copy.
__global__ void k_twiddles(int64_t nside, double2 *tw64, float2 *tw32)
{
    int64_t i = blockIdx.y + 1;
    int64_t half = 2 * i;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < half;
         k += (int64_t)gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-(double)k / (double)half, &s, &c);  // -2 pi k / (4 i) = -pi k / (2 i)
        int64_t idx = i * (i - 1) + k;
        tw64[idx] = make_double2(c, s);
        tw32[idx] = make_float2((float)c, (float)s);
    }
}

template <typename T2> struct TwTable;
template <> struct TwTable<double2> {
    static __device__ __forceinline__ const double2 *get(const void *tw, int64_t cnt)
    {
        return reinterpret_cast<const double2 *>(tw);
    }
};
template <> struct TwTable<float2> {
    static __device__ __forceinline__ const float2 *get(const void *tw, int64_t cnt)
    {
        return reinterpret_cast<const float2 *>(reinterpret_cast<const double2 *>(tw) + cnt);
    }
};

// omega_h^e for an FFT of length h and 0 <= e < h, from the table of n = TM h: tw holds
// omega_n^k for k < n / 2, and omega_n^{k + n/2} = -omega_n^k.  TM = 2 is the ring
// transform (n = 2h, the ring's own table); TM = 1 a length-h FFT with its own table
// (h = n).  `sign` > 0 conjugates (inverse transform).
template <int TM = 2, typename T2>
__device__ __forceinline__ T2 twiddle(const T2 *__restrict__ tw, int h, int e, int sign)
{
    const int k = TM * e, half = TM * h / 2;
    T2 w;
    if (k < half) {
        w = __ldg(tw + k);
    } else {
        w = __ldg(tw + (k - half));
        w.x = -w.x;
        w.y = -w.y;
    }
    if (sign > 0) w.y = -w.y;
    return w;
}

// omega_n^k for k < n (n = 2h).
template <typename T2>
__device__ __forceinline__ T2 twiddle_n(const T2 *__restrict__ tw, int h, int k, int sign)
{
    T2 w;
    if (k < h) {
        w = __ldg(tw + k);
    } else {
        w = __ldg(tw + (k - h));
        w.x = -w.x;
        w.y = -w.y;
    }
    if (sign > 0) w.y = -w.y;
    return w;
}

// e^{sign i pi q2 / n} for 0 <= q2 < 2n from the table: omega_n^{q2/2} (times e^{-i pi / n}
// for odd q2), conjugated for sign > 0.  c1 = e^{-i pi / n}.
template <typename T2>
__device__ __forceinline__ T2 phase_pi(const T2 *__restrict__ tw, int h, int q2, T2 c1, int sign)
{
    T2 w = twiddle_n(tw, h, q2 >> 1, -1);
    if (q2 & 1) w = cmul(w, c1);
    if (sign > 0) w.y = -w.y;
    return w;
}

// ---------------------------------------------------------------- FFT core

__device__ int factorize(int h, int *rad)
{
    int n = 0;
    while (h % 4 == 0) { rad[n++] = 4; h /= 4; }
    if (h % 2 == 0) { rad[n++] = 2; h /= 2; }
    for (int p = 3; p * p <= h; p += 2)
        while (h % p == 0) { rad[n++] = p; h /= p; }
    if (h > 1) rad[n++] = h;
    return n;
}

// Multiply by sign * i.
template <typename T2>
__device__ __forceinline__ T2 mul_i(T2 z, int sign)
{
    T2 r;
    r.x = -sign * z.y;
    r.y = sign * z.x;
    return r;
}

// One Stockham stage: out[k' Lp + j + Ls v] = sum_q omega_p^{q v} omega_Lp^{q j} in[(k' + r q) Ls + j]
// with Lp = Ls p and r = h / Lp.  Butterflies (k', j) are spread over the CTA.
template <int TM, typename T2>
__device__ void stockham_stage(const T2 *__restrict__ in, T2 *__restrict__ out, int h, int p,
                               int Ls, const T2 *__restrict__ tw, int sign)
{
    const int Lp = Ls * p;
    const int r = h / Lp;
    const int nb = h / p;
    if (p == 4) {
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            int kk = b / Ls, j = b - kk * Ls;
            T2 x0 = in[kk * Ls + j];
            T2 x1 = in[(kk + r) * Ls + j];
            T2 x2 = in[(kk + 2 * r) * Ls + j];
            T2 x3 = in[(kk + 3 * r) * Ls + j];
            if (Ls > 1) {
                const int e = j * r;   // < h / 4
                x1 = cmul(x1, twiddle<TM>(tw, h, e, sign));
                x2 = cmul(x2, twiddle<TM>(tw, h, 2 * e, sign));
                x3 = cmul(x3, twiddle<TM>(tw, h, 3 * e, sign));
            }
            T2 a = cadd(x0, x2), bq = csub(x0, x2);
            T2 c = cadd(x1, x3), d = mul_i(csub(x1, x3), sign);
            T2 *o = out + kk * Lp + j;
            o[0] = cadd(a, c);
            o[Ls] = cadd(bq, d);
            o[2 * Ls] = csub(a, c);
            o[3 * Ls] = csub(bq, d);
        }
    } else if (p == 2) {
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            int kk = b / Ls, j = b - kk * Ls;
            T2 x0 = in[kk * Ls + j];
            T2 x1 = in[(kk + r) * Ls + j];
            if (Ls > 1) x1 = cmul(x1, twiddle<TM>(tw, h, j * r, sign));   // j r < h / 2
            T2 *o = out + kk * Lp + j;
            o[0] = cadd(x0, x1);
            o[Ls] = csub(x0, x1);
        }
    } else {
        // generic radix: one output (k', j, v) per thread iteration, p terms each
        for (int o = threadIdx.x; o < h; o += blockDim.x) {
            int kk = o / Lp, jp = o - kk * Lp;
            int j = jp % Ls;
            T2 acc;
            acc.x = 0;
            acc.y = 0;
            // term q: omega_Lp^{q jp} in[(kk + r q) Ls + j];  omega_Lp = omega_h^r, with
            // the exponent q jp mod Lp stepped incrementally
            int eq = 0;
            for (int q = 0; q < p; ++q) {
                T2 x = in[(kk + r * q) * Ls + j];
                T2 w = twiddle<TM>(tw, h, eq * r, sign);
                acc.x += x.x * w.x - x.y * w.y;
                acc.y += x.x * w.y + x.y * w.x;
                eq += jp;
                if (eq >= Lp) eq -= Lp;
            }
            out[o] = acc;
        }
    }
}

// In-shared-memory FFT of length h (ping-pong between a and b); returns the buffer
// holding the result.  Ends with a __syncthreads().
template <int TM = 2, typename T2>
__device__ T2 *fft_shared(T2 *a, T2 *b, int h, const T2 *__restrict__ tw, int sign)
{
    __shared__ int rad[40];
    __shared__ int nst;
    if (threadIdx.x == 0) nst = factorize(h, rad);
    __syncthreads();
    int Ls = 1;
    for (int s = 0; s < nst; ++s) {
        int p = rad[s];
        stockham_stage<TM>(a, b, h, p, Ls, tw, sign);
        __syncthreads();
        T2 *t = a;
        a = b;
        b = t;
        Ls *= p;
    }
    return a;
}

// ---------------------------------------------------------------- analysis

// Rings whose half-length h has a prime factor above 64 are transformed by Bluestein's
// chirp-z method in single precision (three power-of-two FFTs of length
// M = nextpow2(2h - 1) <= mcap), instead of a generic radix-p stage costing h p.
__host__ __device__ __forceinline__ int largest_prime_factor(int h)
{
    int p = 1;
    for (int q = 2; q * q <= h; ++q)
        while (h % q == 0) {
            p = q;
            h /= q;
        }
    return h > p ? h : p;
}

__host__ __device__ __forceinline__ int next_pow2(int x)
{
    int m = 1;
    while (m < x) m <<= 1;
    return m;
}

__host__ __device__ __forceinline__ bool use_bluestein(int h, int mcap)
{
    return largest_prime_factor(h) > 64 && next_pow2(2 * h - 1) <= mcap;
}

// Largest power-of-two FFT length of the Bluestein path: its table must exist (a ring
// length 4i with i <= nside) and three buffers of it must fit in shared memory.
static inline int bluestein_mcap(int64_t nside)
{
    int64_t m = 1;
    while (2 * m <= 4 * nside && 2 * m <= 8192) m *= 2;
    return (int)m;
}

// Rings beyond the shared-memory kernels: half-length above `hcap` (the ping-pong buffers
// would not fit), or, in single precision, a prime factor above 64 with a Bluestein length
// 2h - 1 < M above `bsmin` (8192, the shared-memory Bluestein length; 0: none) for which the
// M-point table exists (M <= 4 nside).  They are transformed by the persistent *_big kernels
// in global scratch.
__host__ __device__ __forceinline__ bool bluestein_big(int h, int nside, int bsmin)
{
    const int M = next_pow2(2 * h - 1);
    return bsmin > 0 && largest_prime_factor(h) > 64 && M > bsmin && M <= 4 * nside;
}

__host__ __device__ __forceinline__ bool ring_big(int h, int hcap, int nside, int bsmin)
{
    return h > hcap || bluestein_big(h, nside, bsmin);
}

// Load one ring of one map (times the mask) as h complex z_t = x_2t + i x_2t+1, each
// multiplied by f(t) (the Bluestein chirp, or 1).
template <typename T, typename Tin, typename T2, typename F>
__device__ __forceinline__ void load_ring(const Tin *__restrict__ x, const double *__restrict__ mask,
                                          int h, T2 *__restrict__ dst, F f)
{
    for (int t = threadIdx.x; t < h; t += blockDim.x) {
        T2 z;
        if (mask) {
            // masked field: the FP64 product map * mask, rounded once to T
            z.x = (T)((double)x[2 * t] * mask[2 * t]);
            z.y = (T)((double)x[2 * t + 1] * mask[2 * t + 1]);
        } else {
            z.x = (T)x[2 * t];
            z.y = (T)x[2 * t + 1];
        }
        dst[t] = f(t, z);
    }
}

// Unpack the half-length transform Z of one real ring into its spectrum for m < L, with
// the quadrature weight and the ring phase e^{-i m phi0}: dst[m] = w e^{-i m phi0} X[m mod n].
template <typename T, typename T2>
__device__ __forceinline__ void ring_outputs(const T2 *__restrict__ Z, int n, int64_t L,
                                             const T2 *__restrict__ tw, bool sh, T w,
                                             T2 *__restrict__ dst)
{
    const int h = n / 2;
    T2 c1;   // e^{-i pi / n}
    {
        double s1, c1d;
        sincospi(-1.0 / (double)n, &s1, &c1d);
        c1.x = (T)c1d;
        c1.y = (T)s1;
    }
    const unsigned n2 = 2u * (unsigned)n;
    for (int m = threadIdx.x; m < (int)L; m += blockDim.x) {
        const unsigned m2 = (unsigned)m % n2;           // m mod 2n
        const int k = (int)(m2 < (unsigned)n ? m2 : m2 - (unsigned)n);
        const bool conj = k > h;
        const int kk = conj ? n - k : k;                // 0..h
        // X[kk] = E + omega_n^kk O, E = (Z[kk] + conj Z[h-kk]) / 2, O = (Z[kk] - conj Z[h-kk]) / 2i
        const T2 za = Z[kk == h ? 0 : kk], zb = Z[kk == 0 ? 0 : h - kk];
        T er = (za.x + zb.x) * (T)0.5, ei = (za.y - zb.y) * (T)0.5;
        T orr = (za.y + zb.y) * (T)0.5, oi = -(za.x - zb.x) * (T)0.5;
        T2 wn = twiddle_n(tw, h, kk, -1);
        T xr = er + wn.x * orr - wn.y * oi;
        T xi = ei + wn.x * oi + wn.y * orr;
        if (conj) xi = -xi;
        T pr = 1, pi = 0;
        if (sh) {
            // e^{-i m phi0}, phi0 = pi / n
            const T2 ph = phase_pi(tw, h, (int)m2, c1, -1);
            pr = ph.x;
            pi = ph.y;
        }
        T2 g;
        g.x = w * (xr * pr - xi * pi);
        g.y = w * (xr * pi + xi * pr);
        dst[m] = g;
    }
}

// One CTA per (map component, ring), the component the fast grid index so that the CTAs of
// one ring run together and read its mask once from DRAM: mixed-radix Stockham FFT in
// shared memory.  In single precision the rings of the Bluestein path (use_bluestein with
// `mcap` > 0) are left to k_ring_analysis_bluestein.
template <typename T, typename Tin>
__global__ void __launch_bounds__(512) k_ring_analysis(int64_t nside, int64_t L,
                                                       const Tin *__restrict__ maps,
                                                       const double *__restrict__ mask,
                                                       const void *__restrict__ twall,
                                                       int64_t twcnt,
                                                       const uint8_t *__restrict__ shifted,
                                                       typename vec2<T>::type *__restrict__ out,
                                                       int mcap, int hcap, int bsmin)
{
    using T2 = typename vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t r = blockIdx.y, c = blockIdx.x;
    const int64_t nring = 4 * nside - 1, npix = 12 * nside * nside;
    const int n = (int)ring_nphi(nside, r), h = n / 2;
    if (mcap > 0 && use_bluestein(h, mcap)) return;
    if (ring_big(h, hcap, (int)nside, bsmin)) return;   // left to k_ring_analysis_big
    const int64_t off = ring_offset(nside, r);
    T2 *A = reinterpret_cast<T2 *>(smem_raw);
    T2 *B = A + hcap;
    const T2 *tw = TwTable<T2>::get(twall, twcnt) + twiddle_offset(n);
    load_ring<T>(maps + c * npix + off, mask ? mask + off : nullptr, h, A,
                 [](int, T2 z) { return z; });
    __syncthreads();
    T2 *Z = fft_shared(A, B, h, tw, -1);
    ring_outputs<T>(Z, n, L, tw, shifted[r] != 0, (T)(4.0 * M_PI / (double)npix),
                    out + (c * nring + r) * L);
}

// Bluestein path, single precision: one CTA per (block of `cpc` components, ring), the
// component block the fast grid index.
//   X_k = sum_j z_j omega_h^{jk} = c_k sum_j (z_j c_j) conj(c_{k-j}),  c_j = e^{-i pi j^2 / h}
// evaluated as a circular convolution of length M: the transform of the wrapped conjugate
// chirp once per CTA, then per component one forward and one inverse FFT.  The chirp is
// read exactly from the ring's table: c_j = omega_{2h}^{j^2 mod 2h}.
template <typename Tin>
__global__ void __launch_bounds__(512) k_ring_analysis_bluestein(int64_t nside, int64_t L,
                                                                 int64_t ncomp, int cpc, int mcap,
                                                                 int hcap, int bsmin,
                                                                 const Tin *__restrict__ maps,
                                                                 const double *__restrict__ mask,
                                                                 const void *__restrict__ twall,
                                                                 int64_t twcnt,
                                                                 const uint8_t *__restrict__ shifted,
                                                                 float2 *__restrict__ out)
{
    using T2 = float2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t r = blockIdx.y;
    const int n = (int)ring_nphi(nside, r), h = n / 2;
    if (!use_bluestein(h, mcap) || ring_big(h, hcap, (int)nside, bsmin)) return;
    const int M = next_pow2(2 * h - 1);
    const int64_t nring = 4 * nside - 1, npix = 12 * nside * nside;
    const int64_t off = ring_offset(nside, r);
    T2 *buf0 = reinterpret_cast<T2 *>(smem_raw);
    T2 *buf1 = buf0 + mcap, *buf2 = buf1 + mcap;
    const T2 *tw32 = TwTable<T2>::get(twall, twcnt);
    const T2 *tw = tw32 + twiddle_offset(n);     // omega_n^k, k < h
    const T2 *twM = tw32 + twiddle_offset(M);    // omega_M^k, k < M / 2 (M = 4i, i <= nside)
    auto chirp = [&](int j) {
        const unsigned q = ((unsigned)j * (unsigned)j) % (unsigned)n;
        return twiddle_n(tw, h, (int)q, -1);
    };
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        T2 v = make_float2(0.f, 0.f);
        if (m < h) v = chirp(m);
        else if (m > M - h) v = chirp(M - m);
        v.y = -v.y;
        buf0[m] = v;
    }
    __syncthreads();
    const T2 *FB = fft_shared<1>(buf0, buf1, M, twM, -1);
    T2 *X = (FB == buf0) ? buf1 : buf0;
    T2 *Y = buf2;
    const float invM = 1.0f / (float)M;
    const bool sh = shifted[r] != 0;
    const float w = (float)(4.0 * M_PI / (double)npix);
    const int64_t c1 = (int64_t)(blockIdx.x + 1) * cpc < ncomp ? (int64_t)(blockIdx.x + 1) * cpc : ncomp;
    for (int64_t c = (int64_t)blockIdx.x * cpc; c < c1; ++c) {
        for (int j = h + threadIdx.x; j < M; j += blockDim.x) X[j] = make_float2(0.f, 0.f);
        load_ring<float>(maps + c * npix + off, mask ? mask + off : nullptr, h, X,
                         [&](int t, T2 z) { return cmul(z, chirp(t)); });
        __syncthreads();
        T2 *FA = fft_shared<1>(X, Y, M, twM, -1);
        T2 *G = (FA == X) ? Y : X;
        for (int m = threadIdx.x; m < M; m += blockDim.x) {
            T2 v = cmul(FA[m], FB[m]);
            v.x *= invM;
            v.y *= invM;
            FA[m] = v;
        }
        __syncthreads();
        T2 *R = fft_shared<1>(FA, G, M, twM, +1);
        T2 *Z = (R == FA) ? G : FA;
        for (int k = threadIdx.x; k < h; k += blockDim.x) Z[k] = cmul(R[k], chirp(k));
        __syncthreads();
        ring_outputs<float>(Z, n, L, tw, sh, w, out + (c * nring + r) * L);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- hemisphere pack

template <typename T>
__global__ void k_pack_rhs(int64_t nside, int64_t L, int64_t ncomp,
                           const typename vec2<T>::type *__restrict__ spec, T *__restrict__ rhs)
{
    using T2 = typename vec2<T>::type;
    __shared__ T tile[32][33][4];
    const int64_t nlanes = 2 * nside, nring = 4 * nside - 1;
    const int64_t m0 = (int64_t)blockIdx.x * 32, j0 = (int64_t)blockIdx.y * 32, c = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int jj = ty; jj < 32; jj += 8) {
        int64_t j = j0 + jj, m = m0 + tx;
        T v[4] = {0, 0, 0, 0};
        if (j < nlanes && m < L) {
            T2 gn = spec[(c * nring + north_ring(j)) * L + m];
            T2 gs;
            gs.x = 0;
            gs.y = 0;
            if (j != nlanes - 1) gs = spec[(c * nring + south_ring(nside, j)) * L + m];
            v[0] = gn.x + gs.x;
            v[1] = gn.y + gs.y;
            v[2] = gn.x - gs.x;
            v[3] = gn.y - gs.y;
        }
        for (int q = 0; q < 4; ++q) tile[jj][tx][q] = v[q];
    }
    __syncthreads();
    for (int mm = ty; mm < 32; mm += 8) {
        int64_t m = m0 + mm, j = j0 + tx;
        if (j < nlanes && m < L) {
            T *o = rhs + ((m * nlanes + j) * ncomp + c) * 4;
            for (int q = 0; q < 4; ++q) o[q] = tile[tx][mm][q];
        }
    }
}

// ---------------------------------------------------------------- fold residual

// Sum over the residue class k (mod n) of the synthesised coefficients of one ring
// side (`part` 0 north, 2 south) with the alternating sign (-1)^{s t} of the ring
// shift: P_k = sum_t (-1)^{s t} c(k + t n), |k + t n| < L, c(-m) = conj c(m).
template <typename T>
__device__ __forceinline__ void residue_sums(const T *__restrict__ syn, int64_t L, int64_t nlanes,
                                             int64_t ncomp, int64_t j, int64_t c, int k, int n,
                                             bool sh, bool two_sides, T *pn, T *ps)
{
    T nr = 0, ni = 0, sr = 0, si = 0;
    // t >= 0 : m = k + t n in [0, L)
    int t = 0;
    for (int64_t m = k; m < L; m += n, ++t) {
        const T *e = syn + ((m * nlanes + j) * ncomp + c) * 4;
        T sg = (sh && (t & 1)) ? (T)-1 : (T)1;
        nr += sg * e[0];
        ni += sg * e[1];
        if (two_sides) {
            sr += sg * e[2];
            si += sg * e[3];
        }
    }
    // t < 0 : m = k - t' n (t' >= 1), order m < 0 with -m = t' n - k in (0, L)
    t = -1;
    for (int64_t mm = (int64_t)n - k; mm < L; mm += n, --t) {
        if (mm == 0) continue;
        const T *e = syn + ((mm * nlanes + j) * ncomp + c) * 4;
        T sg = (sh && (t & 1)) ? (T)-1 : (T)1;
        nr += sg * e[0];
        ni -= sg * e[1];
        if (two_sides) {
            sr += sg * e[2];
            si -= sg * e[3];
        }
    }
    pn[0] = nr;
    pn[1] = ni;
    ps[0] = sr;
    ps[1] = si;
}

template <typename T>
__global__ void __launch_bounds__(256) k_fold_residual(int64_t nside, int64_t L, int64_t ncomp,
                                                       const T *__restrict__ syn,
                                                       const T *__restrict__ rhs_map,
                                                       const uint8_t *__restrict__ shifted,
                                                       T *__restrict__ rhs_out)
{
    const int64_t j = blockIdx.x, c = blockIdx.y;
    const int64_t nlanes = 2 * nside, npix = 12 * nside * nside;
    const int n = (int)ring_nphi(nside, north_ring(j));
    const bool sh = shifted[north_ring(j)] != 0;
    const bool two = j != nlanes - 1;
    const T wn = (T)(4.0 * M_PI / (double)npix * (double)n);
    for (int k = threadIdx.x; k < n && k < L; k += blockDim.x) {
        T pn[2], ps[2];
        residue_sums(syn, L, nlanes, ncomp, j, c, k, n, sh, two, pn, ps);
        int t = 0;
        for (int64_t m = k; m < L; m += n, ++t) {
            T sg = (sh && (t & 1)) ? -wn : wn;
            T gnr = sg * pn[0], gni = sg * pn[1], gsr = sg * ps[0], gsi = sg * ps[1];
            const int64_t idx = ((m * nlanes + j) * ncomp + c) * 4;
            T *o = rhs_out + idx;
            const T *b = rhs_map + idx;
            o[0] = gnr + gsr - b[0];
            o[1] = gni + gsi - b[1];
            o[2] = gnr - gsr - b[2];
            o[3] = gni - gsi - b[3];
        }
    }
}

// ---------------------------------------------------------------- synthesis

template <typename T>
__global__ void __launch_bounds__(512) k_ring_synthesis(int64_t nside, int64_t L, int64_t ncomp,
                                                        const T *__restrict__ syn,
                                                        const void *__restrict__ twall,
                                                        int64_t twcnt,
                                                        const uint8_t *__restrict__ shifted,
                                                        double *__restrict__ maps, int hcap,
                                                        int bsmin)
{
    using T2 = typename vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int64_t r = blockIdx.x, c = blockIdx.y;
    const int64_t npix = 12 * nside * nside, nlanes = 2 * nside;
    const int n = (int)ring_nphi(nside, r), h = n / 2;
    if (ring_big(h, hcap, (int)nside, bsmin)) return;   // left to k_ring_synthesis_big
    const int64_t off = ring_offset(nside, r);
    const bool south = r >= nlanes;
    const int64_t j = south ? 4 * nside - 2 - r : r;
    const bool sh = shifted[r] != 0;
    T2 *A = reinterpret_cast<T2 *>(smem_raw);
    T2 *B = A + hcap;
    const T2 *tw = TwTable<T2>::get(twall, twcnt) + twiddle_offset(n);
    T2 cpi;   // e^{-i pi / n}
    {
        double s1, c1d;
        sincospi(-1.0 / (double)n, &s1, &c1d);
        cpi.x = (T)c1d;
        cpi.y = (T)s1;
    }
    // Fold into the n-periodic spectrum C_k = e^{i pi s k / n} P_k and build
    // Z'[k] = (C_k + C_{k+h}) + i (C_k - C_{k+h}) omega_n^{-k}, k < h.
    const T *base = syn + (south ? 2 : 0);
    for (int k = threadIdx.x; k < h; k += blockDim.x) {
        T c0[2], c1[2], dummy[2];
        residue_sums(base, L, nlanes, ncomp, j, c, k, n, sh, false, c0, dummy);
        residue_sums(base, L, nlanes, ncomp, j, c, k + h, n, sh, false, c1, dummy);
        T2 ck = make2<T2, T>(c0[0], c0[1]);
        T2 ckh = make2<T2, T>(c1[0], c1[1]);
        if (sh) {
            // e^{i pi k / n} and e^{i pi (k + h) / n}
            ck = cmul(ck, phase_pi(tw, h, k, cpi, +1));
            ckh = cmul(ckh, phase_pi(tw, h, k + h, cpi, +1));
        }
        T2 sum = cadd(ck, ckh);
        T2 dif = cmul(csub(ck, ckh), twiddle_n(tw, h, k, +1));
        T2 z;
        z.x = sum.x - dif.y;
        z.y = sum.y + dif.x;
        A[k] = z;
    }
    __syncthreads();
    T2 *Z = fft_shared(A, B, h, tw, +1);
    double *dst = maps + c * npix + off;
    for (int t = threadIdx.x; t < h; t += blockDim.x) {
        T2 z = Z[t];
        dst[2 * t] = (double)z.x;
        dst[2 * t + 1] = (double)z.y;
    }
}


// ---------------------------------------------------------------- rings beyond shared memory
//
// One persistent CTA per slot of the global scratch (three buffers of Mmax complex floats
// each) walks the rings; only the rings of ring_big are transformed, with the arithmetic of
// the shared-memory kernels: a Stockham FFT of length h, or Bluestein's method with a
// power-of-two length M.  __syncthreads orders the CTA's global-memory accesses.

__device__ __forceinline__ float2 bs_chirp(const float2 *__restrict__ tw, int h, int n, int j, int sign)
{
    const unsigned q = ((unsigned)j * (unsigned)j) % (unsigned)n;
    return twiddle_n(tw, h, (int)q, sign);   // e^{sign i pi j^2 / h}
}

// Bluestein filter: the transform of the wrapped conjugate chirp of length M; returns the
// buffer holding it (b0 or b1).
__device__ float2 *bs_filter(int h, int n, int M, const float2 *__restrict__ tw,
                             const float2 *__restrict__ twM, int sign, float2 *b0, float2 *b1)
{
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        int j = -1;
        if (m < h) j = m;
        else if (m > M - h) j = M - m;
        if (j >= 0) {
            v = bs_chirp(tw, h, n, j, sign);
            v.y = -v.y;
        }
        b0[m] = v;
    }
    __syncthreads();
    return fft_shared<1>(b0, b1, M, twM, -1);
}

// X[0, h) holds z_j c_j; zero-pads to M, convolves with the filter FB and returns the buffer
// holding the DFT sum_j z_j e^{sign 2 pi i jk / h}, k < h.
__device__ float2 *bs_apply(float2 *X, float2 *Y, const float2 *FB, int h, int n, int M,
                            const float2 *__restrict__ tw, const float2 *__restrict__ twM, int sign)
{
    for (int j = h + threadIdx.x; j < M; j += blockDim.x) X[j] = make_float2(0.f, 0.f);
    __syncthreads();
    float2 *FA = fft_shared<1>(X, Y, M, twM, -1);
    float2 *G = (FA == X) ? Y : X;
    const float invM = 1.0f / (float)M;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        float2 v = cmul(FA[m], FB[m]);
        v.x *= invM;
        v.y *= invM;
        FA[m] = v;
    }
    __syncthreads();
    float2 *R = fft_shared<1>(FA, G, M, twM, +1);
    float2 *Z = (R == FA) ? G : FA;
    for (int k = threadIdx.x; k < h; k += blockDim.x) Z[k] = cmul(R[k], bs_chirp(tw, h, n, k, sign));
    __syncthreads();
    return Z;
}

// T = float: three buffers of Mmax complex floats per slot (Bluestein rings included).
// T = double: no Bluestein path (the mixed-radix FFT takes every ring, as in the FP64
// shared-memory kernel); two buffers of 2 nside complex doubles per slot, which fit the
// same slot bytes (64 nside <= 96 nside).
template <typename T, typename Tin>
__global__ void __launch_bounds__(512) k_ring_analysis_big(int64_t nside, int64_t L, int64_t ncomp,
                                                           const Tin *__restrict__ maps,
                                                           const double *__restrict__ mask,
                                                           const void *__restrict__ twall,
                                                           int64_t twcnt,
                                                           const uint8_t *__restrict__ shifted,
                                                           typename vec2<T>::type *__restrict__ out,
                                                           int hcap, int bsmin, void *__restrict__ gscratch,
                                                           int64_t slot_bytes)
{
    using T2 = typename vec2<T>::type;
    constexpr bool kSingle = std::is_same<T, float>::value;
    const int64_t nring = 4 * nside - 1, npix = 12 * nside * nside;
    T2 *b0 = reinterpret_cast<T2 *>(static_cast<unsigned char *>(gscratch) + blockIdx.x * slot_bytes);
    const int64_t bstride = kSingle ? 4 * nside : 2 * nside;
    T2 *b1 = b0 + bstride, *b2 = b1 + bstride;
    const T2 *twT = TwTable<T2>::get(twall, twcnt);
    const T w = (T)(4.0 * M_PI / (double)npix);
    for (int64_t r = blockIdx.x; r < nring; r += gridDim.x) {
        const int n = (int)ring_nphi(nside, r), h = n / 2;
        if (!ring_big(h, hcap, (int)nside, bsmin)) continue;
        const int64_t off = ring_offset(nside, r);
        const T2 *tw = twT + twiddle_offset(n);
        const bool sh = shifted[r] != 0;
        if constexpr (kSingle) {
            const bool bs = bluestein_big(h, (int)nside, bsmin);
            const int M = bs ? next_pow2(2 * h - 1) : 0;
            const float2 *twM = bs ? twT + twiddle_offset(M) : nullptr;
            float2 *FB = nullptr, *X = b0, *Y = b1;
            if (bs) {
                FB = bs_filter(h, n, M, tw, twM, -1, b0, b1);
                X = (FB == b0) ? b1 : b0;
                Y = b2;
            }
            for (int64_t c = 0; c < ncomp; ++c) {
                float2 *Z;
                if (bs) {
                    load_ring<float>(maps + c * npix + off, mask ? mask + off : nullptr, h, X,
                                     [&](int t, float2 z) { return cmul(z, bs_chirp(tw, h, n, t, -1)); });
                    __syncthreads();
                    Z = bs_apply(X, Y, FB, h, n, M, tw, twM, -1);
                } else {
                    load_ring<float>(maps + c * npix + off, mask ? mask + off : nullptr, h, X,
                                     [](int, float2 z) { return z; });
                    __syncthreads();
                    Z = fft_shared(X, Y, h, tw, -1);
                }
                ring_outputs<float>(Z, n, L, tw, sh, w, out + (c * nring + r) * L);
                __syncthreads();
            }
        } else {
            for (int64_t c = 0; c < ncomp; ++c) {
                load_ring<T>(maps + c * npix + off, mask ? mask + off : nullptr, h, b0,
                             [](int, T2 z) { return z; });
                __syncthreads();
                T2 *Z = fft_shared(b0, b1, h, tw, -1);
                ring_outputs<T>(Z, n, L, tw, sh, w, out + (c * nring + r) * L);
                __syncthreads();
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(512) k_ring_synthesis_big(int64_t nside, int64_t L, int64_t ncomp,
                                                            const T *__restrict__ syn,
                                                            const void *__restrict__ twall,
                                                            int64_t twcnt,
                                                            const uint8_t *__restrict__ shifted,
                                                            double *__restrict__ maps, int hcap,
                                                            int bsmin, void *__restrict__ gscratch,
                                                            int64_t slot_bytes)
{
    using T2 = typename vec2<T>::type;
    constexpr bool kSingle = std::is_same<T, float>::value;
    const int64_t nring = 4 * nside - 1, npix = 12 * nside * nside, nlanes = 2 * nside;
    T2 *b0 = reinterpret_cast<T2 *>(static_cast<unsigned char *>(gscratch) + blockIdx.x * slot_bytes);
    const int64_t bstride = kSingle ? 4 * nside : 2 * nside;
    T2 *b1 = b0 + bstride, *b2 = b1 + bstride;
    const T2 *twT = TwTable<T2>::get(twall, twcnt);
    for (int64_t r = blockIdx.x; r < nring; r += gridDim.x) {
        const int n = (int)ring_nphi(nside, r), h = n / 2;
        if (!ring_big(h, hcap, (int)nside, bsmin)) continue;
        const int64_t off = ring_offset(nside, r);
        const bool south = r >= nlanes;
        const int64_t j = south ? 4 * nside - 2 - r : r;
        const bool sh = shifted[r] != 0;
        const T2 *tw = twT + twiddle_offset(n);
        T2 cpi;
        {
            double s1, c1d;
            sincospi(-1.0 / (double)n, &s1, &c1d);
            cpi = make2<T2, T>((T)c1d, (T)s1);
        }
        bool bs = false;
        int M = 0;
        const T2 *twM = nullptr;
        T2 *FB = nullptr, *X = b0, *Y = b1;
        if constexpr (kSingle) {
            bs = bluestein_big(h, (int)nside, bsmin);
            M = bs ? next_pow2(2 * h - 1) : 0;
            twM = bs ? twT + twiddle_offset(M) : nullptr;
            if (bs) {
                FB = bs_filter(h, n, M, tw, twM, +1, b0, b1);
                X = (FB == b0) ? b1 : b0;
                Y = b2;
            }
        }
        const T *base = syn + (south ? 2 : 0);
        for (int64_t c = 0; c < ncomp; ++c) {
            for (int k = threadIdx.x; k < h; k += blockDim.x) {
                T c0[2], c1[2], dummy[2];
                residue_sums(base, L, nlanes, ncomp, j, c, k, n, sh, false, c0, dummy);
                residue_sums(base, L, nlanes, ncomp, j, c, k + h, n, sh, false, c1, dummy);
                T2 ck = make2<T2, T>(c0[0], c0[1]);
                T2 ckh = make2<T2, T>(c1[0], c1[1]);
                if (sh) {
                    ck = cmul(ck, phase_pi(tw, h, k, cpi, +1));
                    ckh = cmul(ckh, phase_pi(tw, h, k + h, cpi, +1));
                }
                const T2 sum = cadd(ck, ckh);
                const T2 dif = cmul(csub(ck, ckh), twiddle_n(tw, h, k, +1));
                T2 z = make2<T2, T>(sum.x - dif.y, sum.y + dif.x);
                if constexpr (kSingle) {
                    if (bs) z = cmul(z, bs_chirp(tw, h, n, k, +1));
                }
                X[k] = z;
            }
            __syncthreads();
            T2 *Z;
            if constexpr (kSingle) Z = bs ? bs_apply(X, Y, FB, h, n, M, tw, twM, +1) : fft_shared(X, Y, h, tw, +1);
            else Z = fft_shared(X, Y, h, tw, +1);
            double *dst = maps + c * npix + off;
            for (int t = threadIdx.x; t < h; t += blockDim.x) {
                const T2 z = Z[t];
                dst[2 * t] = (double)z.x;
                dst[2 * t + 1] = (double)z.y;
            }
            __syncthreads();
        }
    }
}

}  // namespace gm

using namespace gm;

extern "C" int64_t gm_ring_twiddle_count(int64_t nside) { return nside * (nside + 1); }

extern "C" int gm_ring_twiddles(int64_t nside, void *tw, void *stream)
{
    if (nside < 1 || nside > 8192) return GM_ERR_BAD_SHAPE;
    if (!tw) return GM_ERR_BAD_PTR;
    int64_t cnt = gm_ring_twiddle_count(nside);
    double2 *t64 = reinterpret_cast<double2 *>(tw);
    float2 *t32 = reinterpret_cast<float2 *>(t64 + cnt);
    int64_t gx = (2 * nside + 255) / 256;
    if (gx > 64) gx = 64;
    k_twiddles<<<dim3((unsigned)gx, (unsigned)nside), 256, 0, as_stream(stream)>>>(nside, t64, t32);
    return check_launch("gm_ring_twiddles");
}

static size_t ring_smem_bytes(int precision, int64_t nside)
{
    size_t elem = precision == GM_FP64 ? sizeof(double2) : sizeof(float2);
    return 2 * (size_t)(2 * nside) * elem;
}

static int ring_shape_ok(int precision, int64_t nside, int64_t L, int64_t ncomp)
{
    if (nside < 1 || L < 1 || ncomp < 1 || ncomp > 65535) return 0;
    if (ring_smem_bytes(precision, nside) > 227 * 1024) return 0;
    return 1;
}

template <typename K>
static int set_smem(K kernel, size_t bytes)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes);
    if (e != cudaSuccess) {
        set_error("cudaFuncSetAttribute", e);
        return GM_ERR_LAUNCH;
    }
    return GM_OK;
}

// Shared memory of the ring kernels: ping-pong buffers of hcap complex values.
static int ring_hcap(int precision, int64_t nside, bool big)
{
    const size_t elem = precision == GM_FP64 ? sizeof(double2) : sizeof(float2);
    // 227 KB of dynamic shared memory per block, less 1 KB left to the kernels' static arrays
    const int64_t fit = (int64_t)((227 * 1024 - 1024) / (2 * elem));
    const int64_t h = 2 * nside;
    return (int)(big && h > fit ? fit : h);
}

extern "C" int64_t gm_ring_big_scratch_bytes(int64_t nside, int64_t nslots)
{
    return nside < 1 || nslots < 1 ? 0 : nslots * 3 * 4 * nside * (int64_t)sizeof(float2);
}

extern "C" int gm_ring_analysis_ws(int precision, int64_t nside, int64_t L, int64_t ncomp,
                                   const void *maps, int map_dtype_bytes, const double *mask,
                                   const void *tw, const uint8_t *shifted, void *ringspec,
                                   void *scratch, int64_t scratch_bytes, int64_t hcap_max,
                                   int64_t bs_min, void *stream)
{
    const bool big = scratch != nullptr;
    if (nside < 1 || nside > 8192 || L < 1 || ncomp < 1 || ncomp > 65535) return GM_ERR_BAD_SHAPE;
    if (!big && !ring_shape_ok(precision, nside, L, ncomp)) return GM_ERR_BAD_SHAPE;
    if (!maps || !tw || !shifted || !ringspec) return GM_ERR_BAD_PTR;
    if (map_dtype_bytes != 8 && map_dtype_bytes != 4) return GM_ERR_UNSUPPORTED;
    const int64_t nslots = big ? scratch_bytes / gm_ring_big_scratch_bytes(nside, 1) : 0;
    if (big && nslots < 1) return GM_ERR_BAD_SHAPE;
    const int64_t nring = 4 * nside - 1, cnt = gm_ring_twiddle_count(nside);
    int hcap = ring_hcap(precision, nside, big);
    if (big && hcap_max > 0 && hcap_max < hcap) hcap = (int)hcap_max;
    // single precision only: FP64 has no Bluestein path
    const int bsmin = big && precision == GM_MIXED ? (bs_min > 0 ? (int)bs_min : 8192) : 0;
    const size_t smem = 2 * (size_t)hcap * (precision == GM_FP64 ? sizeof(double2) : sizeof(float2));
    const int64_t slot = gm_ring_big_scratch_bytes(nside, 1);
    int threads = nside >= 256 ? 512 : 128;
    dim3 grid((unsigned)ncomp, (unsigned)nring);
    cudaStream_t s = as_stream(stream);
    int st;
    if (precision == GM_FP64) {
        const unsigned gbig = (unsigned)(nslots < nring ? nslots : nring);
        if (map_dtype_bytes == 8) {
            if ((st = set_smem(k_ring_analysis<double, double>, smem))) return st;
            k_ring_analysis<double, double><<<grid, threads, smem, s>>>(
                nside, L, (const double *)maps, mask, tw, cnt, shifted, (double2 *)ringspec, 0, hcap, 0);
            if (big)
                k_ring_analysis_big<double, double><<<gbig, 512, 0, s>>>(
                    nside, L, ncomp, (const double *)maps, mask, tw, cnt, shifted, (double2 *)ringspec,
                    hcap, 0, scratch, slot);
        } else {
            if ((st = set_smem(k_ring_analysis<double, float>, smem))) return st;
            k_ring_analysis<double, float><<<grid, threads, smem, s>>>(
                nside, L, (const float *)maps, mask, tw, cnt, shifted, (double2 *)ringspec, 0, hcap, 0);
            if (big)
                k_ring_analysis_big<double, float><<<gbig, 512, 0, s>>>(
                    nside, L, ncomp, (const float *)maps, mask, tw, cnt, shifted, (double2 *)ringspec,
                    hcap, 0, scratch, slot);
        }
    } else if (precision == GM_MIXED) {
        const int mcap = bluestein_mcap(nside);
        const size_t bs_smem = 3 * (size_t)mcap * sizeof(float2);
        const int cpc = 8;
        dim3 bs_grid((unsigned)((ncomp + cpc - 1) / cpc), (unsigned)nring);
        const unsigned gbig = (unsigned)(nslots < nring ? nslots : nring);
        if (map_dtype_bytes == 8) {
            if ((st = set_smem(k_ring_analysis<float, double>, smem))) return st;
            k_ring_analysis<float, double><<<grid, threads, smem, s>>>(
                nside, L, (const double *)maps, mask, tw, cnt, shifted, (float2 *)ringspec, mcap, hcap, bsmin);
            if ((st = set_smem(k_ring_analysis_bluestein<double>, bs_smem))) return st;
            k_ring_analysis_bluestein<double><<<bs_grid, 512, bs_smem, s>>>(
                nside, L, ncomp, cpc, mcap, hcap, bsmin, (const double *)maps, mask, tw, cnt, shifted,
                (float2 *)ringspec);
            if (big)
                k_ring_analysis_big<float, double><<<gbig, 512, 0, s>>>(
                    nside, L, ncomp, (const double *)maps, mask, tw, cnt, shifted, (float2 *)ringspec,
                    hcap, bsmin, scratch, slot);
        } else {
            if ((st = set_smem(k_ring_analysis<float, float>, smem))) return st;
            k_ring_analysis<float, float><<<grid, threads, smem, s>>>(
                nside, L, (const float *)maps, mask, tw, cnt, shifted, (float2 *)ringspec, mcap, hcap, bsmin);
            if ((st = set_smem(k_ring_analysis_bluestein<float>, bs_smem))) return st;
            k_ring_analysis_bluestein<float><<<bs_grid, 512, bs_smem, s>>>(
                nside, L, ncomp, cpc, mcap, hcap, bsmin, (const float *)maps, mask, tw, cnt, shifted,
                (float2 *)ringspec);
            if (big)
                k_ring_analysis_big<float, float><<<gbig, 512, 0, s>>>(
                    nside, L, ncomp, (const float *)maps, mask, tw, cnt, shifted, (float2 *)ringspec,
                    hcap, bsmin, scratch, slot);
        }
    } else {
        return GM_ERR_UNSUPPORTED;
    }
    return check_launch("gm_ring_analysis");
}

extern "C" int gm_ring_analysis(int precision, int64_t nside, int64_t L, int64_t ncomp,
                                const void *maps, int map_dtype_bytes, const double *mask,
                                const void *tw, const uint8_t *shifted, void *ringspec,
                                void *stream)
{
    return gm_ring_analysis_ws(precision, nside, L, ncomp, maps, map_dtype_bytes, mask, tw, shifted,
                               ringspec, nullptr, 0, 0, 0, stream);
}

extern "C" int gm_pack_rhs(int precision, int64_t nside, int64_t L, int64_t ncomp,
                           const void *ringspec, void *rhs, void *stream)
{
    if (nside < 1 || L < 1 || ncomp < 1 || ncomp > 65535) return GM_ERR_BAD_SHAPE;
    if (!ringspec || !rhs) return GM_ERR_BAD_PTR;
    const int64_t nlanes = 2 * nside;
    dim3 grid((unsigned)((L + 31) / 32), (unsigned)((nlanes + 31) / 32), (unsigned)ncomp);
    dim3 block(32, 8);
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        k_pack_rhs<double><<<grid, block, 0, s>>>(nside, L, ncomp, (const double2 *)ringspec,
                                                  (double *)rhs);
    else if (precision == GM_MIXED)
        k_pack_rhs<float><<<grid, block, 0, s>>>(nside, L, ncomp, (const float2 *)ringspec,
                                                 (float *)rhs);
    else
        return GM_ERR_UNSUPPORTED;
    return check_launch("gm_pack_rhs");
}

extern "C" int gm_fold_residual(int precision, int64_t nside, int64_t L, int64_t ncomp,
                                const void *syn, const void *rhs_map, const uint8_t *shifted,
                                void *rhs_out, void *stream)
{
    if (nside < 1 || L < 1 || ncomp < 1 || ncomp > 65535) return GM_ERR_BAD_SHAPE;
    if (!syn || !rhs_map || !shifted || !rhs_out) return GM_ERR_BAD_PTR;
    dim3 grid((unsigned)(2 * nside), (unsigned)ncomp);
    cudaStream_t s = as_stream(stream);
    if (precision == GM_FP64)
        k_fold_residual<double><<<grid, 256, 0, s>>>(nside, L, ncomp, (const double *)syn,
                                                     (const double *)rhs_map, shifted,
                                                     (double *)rhs_out);
    else if (precision == GM_MIXED)
        k_fold_residual<float><<<grid, 256, 0, s>>>(nside, L, ncomp, (const float *)syn,
                                                    (const float *)rhs_map, shifted,
                                                    (float *)rhs_out);
    else
        return GM_ERR_UNSUPPORTED;
    return check_launch("gm_fold_residual");
}

extern "C" int gm_ring_synthesis_ws(int precision, int64_t nside, int64_t L, int64_t ncomp,
                                    const void *syn, const void *tw, const uint8_t *shifted,
                                    double *maps, void *scratch, int64_t scratch_bytes,
                                    int64_t hcap_max, int64_t bs_min, void *stream)
{
    const bool big = scratch != nullptr;
    if (nside < 1 || nside > 8192 || L < 1 || ncomp < 1 || ncomp > 65535) return GM_ERR_BAD_SHAPE;
    if (!big && !ring_shape_ok(precision, nside, L, ncomp)) return GM_ERR_BAD_SHAPE;
    if (!syn || !tw || !shifted || !maps) return GM_ERR_BAD_PTR;
    const int64_t nslots = big ? scratch_bytes / gm_ring_big_scratch_bytes(nside, 1) : 0;
    if (big && nslots < 1) return GM_ERR_BAD_SHAPE;
    const int64_t nring = 4 * nside - 1, cnt = gm_ring_twiddle_count(nside);
    int hcap = ring_hcap(precision, nside, big);
    if (big && hcap_max > 0 && hcap_max < hcap) hcap = (int)hcap_max;
    const int bsmin = big && precision == GM_MIXED ? (bs_min > 0 ? (int)bs_min : 8192) : 0;
    const size_t smem = 2 * (size_t)hcap * (precision == GM_FP64 ? sizeof(double2) : sizeof(float2));
    const int64_t slot = gm_ring_big_scratch_bytes(nside, 1);
    const unsigned gbig = (unsigned)(nslots < nring ? nslots : nring);
    int threads = nside >= 256 ? 512 : 128;
    dim3 grid((unsigned)nring, (unsigned)ncomp);
    cudaStream_t s = as_stream(stream);
    int st;
    if (precision == GM_FP64) {
        if ((st = set_smem(k_ring_synthesis<double>, smem))) return st;
        k_ring_synthesis<double><<<grid, threads, smem, s>>>(nside, L, ncomp, (const double *)syn,
                                                             tw, cnt, shifted, maps, hcap, 0);
        if (big)
            k_ring_synthesis_big<double><<<gbig, 512, 0, s>>>(nside, L, ncomp, (const double *)syn, tw, cnt,
                                                              shifted, maps, hcap, 0, scratch, slot);
    } else if (precision == GM_MIXED) {
        if ((st = set_smem(k_ring_synthesis<float>, smem))) return st;
        k_ring_synthesis<float><<<grid, threads, smem, s>>>(nside, L, ncomp, (const float *)syn,
                                                            tw, cnt, shifted, maps, hcap, bsmin);
        if (big)
            k_ring_synthesis_big<float><<<gbig, 512, 0, s>>>(nside, L, ncomp, (const float *)syn, tw, cnt,
                                                             shifted, maps, hcap, bsmin, scratch, slot);
    } else {
        return GM_ERR_UNSUPPORTED;
    }
    return check_launch("gm_ring_synthesis");
}

extern "C" int gm_ring_synthesis(int precision, int64_t nside, int64_t L, int64_t ncomp,
                                 const void *syn, const void *tw, const uint8_t *shifted,
                                 double *maps, void *stream)
{
    return gm_ring_synthesis_ws(precision, nside, L, ncomp, syn, tw, shifted, maps, nullptr, 0, 0, 0,
                                stream);
}
