// Pseudo-C_ell, Wigner-3j coupling blocks, binning and the binned decouple (sm_100a).
//
// Replaces, from the reference (licongxu/GMaster):
//   gmaster/workspaces.py:86-95      `_compute_coupled_cell` (XLA segment_sum)
//   gmaster/workspaces.py:352-517    scalar coupling (threej closed form / GL quadrature)
//   gmaster/workspaces.py:682-924    spin-0/2 coupling by GL quadrature GEMMs
//   gmaster/_native/cuda/coupling_tt.cu:18-45  (FP32-product threej kernel, lmax < 48)
//   gmaster/workspaces.py:1570-1590, 292-310   binned MCM (cuBLAS GEMMs)
//   gmaster/workspaces.py:2146       decouple solve (cuSOLVER getrf/getrs)
#include <math.h>

#include "gm_common.cuh"

namespace gm {

__device__ __forceinline__ int64_t alm_idx(int64_t lmax, int64_t l, int64_t m)
{
    return m * (2 * lmax + 1 - m) / 2 + l;
}

// ---------------------------------------------------------------- pseudo-C_ell

constexpr int kPclLanes = 32;   // degrees per CTA (one per lane: coalesced over l)
constexpr int kPclWarps = 8;    // orders interleaved over the warps of a CTA

// grid (l-blocks of 32, pairs), 256 threads: lane = degree l, warp w sums the orders
// m = w, w + 8, ... <= l; the eight partial sums are then added in a fixed order, so the
// result does not depend on scheduling (equal inputs give bit-equal spectra).
__global__ void __launch_bounds__(kPclLanes * kPclWarps) k_pseudo_cl(int64_t lmax, int64_t n1,
                                                                     const double2 *__restrict__ a, int64_t n2,
                                                                     const double2 *__restrict__ b,
                                                                     double *__restrict__ cls)
{
    __shared__ double part[kPclWarps][kPclLanes];
    const int64_t L = lmax + 1, nelem = L * (L + 1) / 2;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t l = (int64_t)blockIdx.x * kPclLanes + lane;
    const int64_t pair = blockIdx.y, i = pair / n2, j = pair % n2;
    const double2 *ai = a + i * nelem;
    const double2 *bj = b + j * nelem;
    double s = 0.0;
    if (l < L) {
        for (int64_t m = w; m <= l; m += kPclWarps) {
            const int64_t k = alm_idx(lmax, l, m);
            const double2 x = ai[k], y = bj[k];
            const double re = x.x * y.x + x.y * y.y;
            s += m == 0 ? re : 2.0 * re;
        }
    }
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && l < L) {
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < kPclWarps; ++q) t += part[q][lane];
        cls[pair * L + l] = t / (2.0 * (double)l + 1.0);
    }
}

// ---------------------------------------------------------------- Wigner-3j coupling

// Work unit u -> (l1, l2 block) with l1 descending (longest recursions first):
// t = lmax - l1 has floor(t / 32) + 1 blocks of 32 columns l2 >= l1.
__device__ __forceinline__ bool unit_to_pair(int64_t u, int64_t lmax, int64_t &l1, int64_t &l2b)
{
    // cumulative units before t = 32 G + rr: 16 G (G + 1) + rr (G + 1)
    int64_t G = (int64_t)floor((sqrt(1.0 + (double)u / 4.0) - 1.0) / 2.0);
    if (G < 0) G = 0;
    while (16 * (G + 1) * (G + 2) <= u) ++G;
    while (G > 0 && 16 * G * (G + 1) > u) --G;
    const int64_t rem = u - 16 * G * (G + 1);
    const int64_t rr = rem / (G + 1), b = rem % (G + 1);
    const int64_t t = 32 * G + rr;
    if (t > lmax) return false;
    l1 = lmax - t;
    l2b = l1 + 32 * b;
    return true;
}

__host__ __device__ __forceinline__ int64_t total_units(int64_t lmax)
{
    // t in [0, lmax]: sum of floor(t/32) + 1
    const int64_t T = lmax + 1, G = T / 32, rr = T % 32;
    return 16 * G * (G + 1) + rr * (G + 1);
}

// Coupling sums of one pair (l1 <= l2): vals[x] = S_x(l1, l2) for x = tt, te, pp, mm,
// S_x = sum_l3 (2 l3 + 1) W_l3 / (4 pi) T_x(l1, l2, l3) (the blocks divided by 2 l2 + 1),
// with T_tt = (l1 l2 l3; 000)^2, T_te = (000)(2 -2 0), T_pp / T_mm = (2 -2 0)^2 on the
// l1 + l2 + l3 even / odd terms.
//
// Recurrences in j = l3 from j_min = l2 - l1 to j_max = l1 + l2 (Schulten & Gordon 1975,
// m3 = 0): with P(j) = (j^2 - d^2)(S^2 - j^2), d = l2 - l1, S = l1 + l2 + 1,
//   sqrt P(j+1) f_{j+1} = -sqrt P(j) f_{j-1}                    for (000)
//   sqrt P(j+1) g_{j+1} = 4 (2j+1) g_j - sqrt P(j) g_{j-1}      for (2 -2 0),
// both unnormalised from f = g = 1 at j_min and normalised by sum (2j+1) f^2 = 1.  The
// substitution f^_j = f_j s_j, g^_j = g_j s_j with s_j = prod_{i <= j} sqrt P(i) removes
// every square root and division:
//   f^_{j+1} = -P(j) f^_{j-1},   g^_{j+1} = 4 (2j+1) g^_j - P(j) g^_{j-1},
// and f^2, f g, g^2 become the hatted products over D_j = prod_{i <= j} P(i).  Each sum
// sum_j c_j X^_j / D_j is carried as A / D_j with A_j = A_{j-1} P(j) + c_j X^_j (Horner
// form); D cancels in every quotient of the results, so it is never formed.  The odd-offset
// (000) terms vanish, so the loop steps j by two.  The products grow by ~P^2 per step;
// whenever a normalising sum passes 2^512 its family is scaled down by an exact power of
// two (f^ or g^ by 2^-256, their squared sums by 2^-512).
template <bool TT, bool TE, bool PM>
__device__ __forceinline__ void coupling_sums(int64_t l1, int64_t l2, const double *__restrict__ window,
                                              int64_t nw, double (&vals)[4])
{
    constexpr bool F = TT || TE, G = TE || PM;
    const double inv4pi = 1.0 / (4.0 * M_PI);
    const int64_t d = l2 - l1, jmin = d, jmax = l1 + l2;
    const double S = (double)(l1 + l2 + 1), S2 = S * S, d2 = (double)(d * d);
    const double lo = 0x1p-256, lo2 = 0x1p-512;
    const int big = (1023 + 512) << 20;  // high word of 2^512
    const double t0 = 2.0 * (double)jmin + 1.0;
    const double w0 = (jmin < nw ? __ldg(window + jmin) : 0.0) * t0;
    double f0 = 1.0, g0 = 1.0, gm1 = 0.0, P0 = 0.0;
    double an0 = t0, att = w0, an2 = t0, ate = w0, app = w0, amm = 0.0;
    double jd = (double)jmin;
    for (int64_t j = jmin; j < jmax; j += 2) {
        const double j1 = jd + 1.0, j2 = jd + 2.0;
        const double P1 = fma(j1, j1, -d2) * fma(-j1, j1, S2);
        const double P2 = fma(j2, j2, -d2) * fma(-j2, j2, S2);
        const double t1 = 2.0 * j1 + 1.0, t2 = 2.0 * j2 + 1.0;
        const double w2 = (j + 2 < nw ? __ldg(window + j + 2) : 0.0) * t2;
        const double PP = P1 * P2;
        double f2 = 0.0, g2 = 0.0;
        if (F) {
            f2 = -P1 * f0;
            const double ff2 = f2 * f2;
            an0 = fma(an0, PP, t2 * ff2);
            if (TT) att = fma(att, PP, w2 * ff2);
        }
        if (G) {
            const double g1 = fma(4.0 * (2.0 * jd + 1.0), g0, -P0 * gm1);
            g2 = fma(4.0 * t1, g1, -P1 * g0);
            const double gg1 = g1 * g1, gg2 = g2 * g2;
            an2 = fma(fma(an2, P1, t1 * gg1), P2, t2 * gg2);
            if (PM) {
                const double w1 = (j + 1 < nw ? __ldg(window + j + 1) : 0.0) * t1;
                app = fma(app, PP, w2 * gg2);
                amm = fma(amm, P1, w1 * gg1) * P2;
            }
            if (TE) ate = fma(ate, PP, w2 * f2 * g2);
            gm1 = g1;
            g0 = g2;
        }
        f0 = f2;
        P0 = P2;
        jd = j2;
        if (F && __double2hiint(an0) > big) {
            f0 *= lo;
            an0 *= lo2;
            att *= lo2;
            ate *= lo;
        }
        if (G && __double2hiint(an2) > big) {
            g0 *= lo;
            gm1 *= lo;
            an2 *= lo2;
            app *= lo2;
            amm *= lo2;
            ate *= lo;
        }
    }
    if (TT) vals[0] = inv4pi * att / an0;
    if (TE) {
        // (000) and (2 -2 0) both carry (-1)^(l1 - l2) at l3 = l1 + l2, so the relative
        // sign of the unnormalised product is sign(f g) there.
        const double sgn = (f0 * g0) < 0.0 ? -1.0 : 1.0;
        vals[1] = sgn * inv4pi * ate / (sqrt(an0) * sqrt(an2));
    }
    if (PM) {
        vals[2] = inv4pi * app / an2;
        vals[3] = inv4pi * amm / an2;
    }
}

// Coupling sums of the blocks `which` asks for (bit x = block x); the others are zero.
// Spin-2 sums vanish unless l1, l2 >= 2.
__device__ __forceinline__ void coupling_pair(int64_t l1, int64_t l2, const double *__restrict__ window,
                                              int64_t nw, int which, double (&vals)[4])
{
    vals[0] = vals[1] = vals[2] = vals[3] = 0.0;
    const bool s2ok = l1 >= 2 && l2 >= 2;
    const int w = s2ok ? which : (which & 1);
    if (w == 1) coupling_sums<true, false, false>(l1, l2, window, nw, vals);
    else if (w == 2) coupling_sums<false, true, false>(l1, l2, window, nw, vals);
    else if (w == 4 || w == 8 || w == 12) coupling_sums<false, false, true>(l1, l2, window, nw, vals);
    else if (w != 0) coupling_sums<true, true, true>(l1, l2, window, nw, vals);
}

__global__ void __launch_bounds__(128) k_coupling(int64_t lmax, const double *__restrict__ window,
                                                  int64_t nw, int which,
                                                  double *__restrict__ blocks,
                                                  unsigned long long *__restrict__ queue)
{
    const int64_t n = lmax + 1, nn = n * n;
    const int64_t nunits = total_units(lmax);
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(queue, 1ull);
        u = __shfl_sync(0xffffffffu, u, 0);
        if ((int64_t)u >= nunits) break;
        int64_t l1, l2b;
        if (!unit_to_pair((int64_t)u, lmax, l1, l2b)) break;
        const int64_t l2 = l2b + lane;
        if (l2 <= lmax) {
            double vals[4];
            coupling_pair(l1, l2, window, nw, which, vals);
            const double c1 = 2.0 * (double)l1 + 1.0, c2 = 2.0 * (double)l2 + 1.0;
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                if (!(which & (1 << x))) continue;
                double *bx = blocks + x * nn;
                bx[l1 * n + l2] = c2 * vals[x];
                bx[l2 * n + l1] = c1 * vals[x];
            }
        }
    }
}

// Many coupling matrices of different lmax in one persistent launch.  Job j is the row
// jobs[6 j .. 6 j + 5] = (lmax, window offset, nw, which, blocks offset, first unit); units
// are numbered consecutively over the jobs (job j owns [first_j, first_{j+1}) and
// nunits in total), the jobs being ordered by decreasing lmax so the longest recursions
// go first.  Each warp takes the next unit from the shared queue, finds its job by binary
// search and computes its pair block as k_coupling does.
__global__ void __launch_bounds__(128) k_coupling_multi(int64_t njobs, const int64_t *__restrict__ jobs,
                                                        int64_t nunits,
                                                        const double *__restrict__ windows,
                                                        double *__restrict__ blocks,
                                                        unsigned long long *__restrict__ queue)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(queue, 1ull);
        u = __shfl_sync(0xffffffffu, u, 0);
        if ((int64_t)u >= nunits) break;
        int64_t lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (jobs[6 * mid + 5] <= (int64_t)u) lo = mid;
            else hi = mid - 1;
        }
        const int64_t *jb = jobs + 6 * lo;
        const int64_t lmax = jb[0], n = lmax + 1, nn = n * n;
        const int which = (int)jb[3];
        int64_t l1, l2b;
        if (!unit_to_pair((int64_t)u - jb[5], lmax, l1, l2b)) continue;
        const int64_t l2 = l2b + lane;
        if (l2 <= lmax) {
            double vals[4];
            coupling_pair(l1, l2, windows + jb[1], jb[2], which, vals);
            const double c1 = 2.0 * (double)l1 + 1.0, c2 = 2.0 * (double)l2 + 1.0;
            double *bj = blocks + jb[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                if (!(which & (1 << x))) continue;
                double *bx = bj + x * nn;
                bx[l1 * n + l2] = c2 * vals[x];
                bx[l2 * n + l1] = c1 * vals[x];
            }
        }
    }
}

// Scalar coupling sums S_tt(l1, l2) of an explicit list of pairs, written symmetrically
// into the dense (lmax+1)^2 matrix S (entries not listed are left as they are).
__global__ void k_coupling_pairs_tt(int64_t lmax, const double *__restrict__ window, int64_t nw,
                                    const int32_t *__restrict__ pairs, int64_t npairs,
                                    double *__restrict__ S)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int64_t a = pairs[2 * t], b = pairs[2 * t + 1], n = lmax + 1;
    const int64_t l1 = a < b ? a : b, l2 = a < b ? b : a;
    double vals[4];
    coupling_pair(l1, l2, window, nw, 1, vals);
    S[l1 * n + l2] = vals[0];
    S[l2 * n + l1] = vals[0];
}

// NaMaster's Toeplitz approximation of the scalar coupling (Louis et al. 2020), filled
// from the exact entries of S = M / (2 l' + 1) that it reads: the diagonal, column
// l_toeplitz, columns 0..l_exact and the dl_band sub-diagonals.  With d_l = |S_ll|, the
// correlation c_l = S(l, lt) / sqrt(d_l d_lt) and the column correlation
// e_l = S(l, le) / sqrt(d_l d_le) (zero where d vanishes), entry (r >= q) of the lower
// triangle is, by the first rule that applies:
//   le <= q <= lt and r >= n - 1 - lt + q :  e_{r - q + le} sqrt(d_q d_r)
//   1 <= r - q <= dl_band and q <= lt      :  S(q, r)
//   r == q                                  :  S(r, r)
//   r >= lt and q >= lt                     :  c_{(r - q + lt) mod n} sqrt(d_r d_q)
//   r - q <= dl_band                        :  S(q, r)
//   q <= le                                 :  S(r, q)
//   otherwise                               :  c_{(r - q + lt) mod n} sqrt(d_r d_q)
// and the matrix is symmetric; out(i, j) = T(i, j) (2 j + 1).
__global__ void k_toeplitz_fill(int64_t lmax, int64_t lt, int64_t le, int64_t dlb,
                                const double *__restrict__ S, double *__restrict__ out)
{
    const int64_t n = lmax + 1;
    const int64_t i = blockIdx.y, j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int64_t r = i > j ? i : j, q = i > j ? j : i;
    auto d = [&](int64_t l) { return fabs(S[l * n + l]); };
    auto corr = [&](int64_t l) {
        const double den = sqrt(d(l) * d(lt));
        return den > 0.0 ? S[l * n + lt] / den : 0.0;
    };
    auto pure = [&]() { return corr((r - q + lt) % n) * sqrt(d(r) * d(q)); };
    double v;
    if (q >= le && q <= lt && r >= n - 1 - lt + q) {
        const int64_t l = r - q + le;
        const double dl = d(l);
        const double e = dl > 0.0 ? S[l * n + le] / sqrt(dl * d(le)) : 0.0;
        v = e * sqrt(d(q) * d(r));
    } else if (r - q >= 1 && r - q <= dlb && q <= lt) {
        v = S[q * n + r];
    } else if (r == q) {
        v = S[r * n + r];
    } else if (r >= lt && q >= lt) {
        v = pure();
    } else if (r - q <= dlb) {
        v = S[q * n + r];
    } else if (q <= le) {
        v = S[r * n + q];
    } else {
        v = pure();
    }
    out[i * n + j] = v * (2.0 * (double)j + 1.0);
}

// ---------------------------------------------------------------- binning

// Binned block: out[b][b'] = sum_{l in b} wfl[l] sum_{l' in b'} M[l][l'] beam[l'] inv_fl[l'].
__global__ void k_bin_block(int64_t lmax, int64_t nb, const double *__restrict__ M,
                            const int32_t *__restrict__ band_ptr, const int32_t *__restrict__ band_ells,
                            const double *__restrict__ wfl, const double *__restrict__ inv_fl,
                            const double *__restrict__ beam, double *__restrict__ out)
{
    const int64_t b = blockIdx.y, bp = blockIdx.x, n = lmax + 1;
    const int i0 = band_ptr[b], i1 = band_ptr[b + 1], k0 = band_ptr[bp], k1 = band_ptr[bp + 1];
    const int nk = k1 - k0, cnt = (i1 - i0) * nk;
    double s = 0.0;
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
        const int l = band_ells[i0 + t / nk], lp = band_ells[k0 + t % nk];
        s += wfl[l] * M[(int64_t)l * n + lp] * beam[lp] * inv_fl[lp];
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b * nb + bp] = red[0];
}

// Place binned blocks into the (ncls nb)^2 matrix, band-major channel-minor.
__global__ void k_place_binned(int64_t nb, int ncls, const double *__restrict__ bb,
                               double *__restrict__ out)
{
    const int64_t N = ncls * nb;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * N) return;
    const int64_t row = idx / N, col = idx % N;
    const int64_t b = row / ncls, c1 = row % ncls, bp = col / ncls, c2 = col % ncls;
    const int64_t nb2 = nb * nb;
    double v = 0.0;
    if (ncls == 1) {
        v = bb[b * nb + bp];
    } else if (ncls == 2) {
        if (c1 == c2) v = bb[b * nb + bp];
    } else {
        if (c1 == c2) v = bb[b * nb + bp];                       // M+ on the diagonal slots
        else if (c1 + c2 == 3)                                   // M- on the anti-diagonal
            v = ((c1 == 1 || c1 == 2) ? -1.0 : 1.0) * bb[nb2 + b * nb + bp];
    }
    out[idx] = v;
}

__global__ void k_bin_cells(int64_t lmax, int64_t nb, int64_t ncls, const double *__restrict__ cls,
                            const int32_t *__restrict__ band_ptr,
                            const int32_t *__restrict__ band_ells, const double *__restrict__ wfl,
                            double *__restrict__ out)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * ncls) return;
    const int64_t c = idx / nb, b = idx % nb;
    double s = 0.0;
    for (int i = band_ptr[b]; i < band_ptr[b + 1]; ++i) {
        const int l = band_ells[i];
        s += wfl[l] * cls[c * (lmax + 1) + l];
    }
    out[c * nb + b] = s;
}

// ---------------------------------------------------------------- LU

// Single-CTA right-looking LU with partial pivoting, row-major a (n x n).
__global__ void __launch_bounds__(1024) k_lu_factor(int64_t n, double *__restrict__ a,
                                                    int32_t *__restrict__ piv,
                                                    int32_t *__restrict__ status)
{
    __shared__ double sval[32];
    __shared__ int sidx[32];
    __shared__ int pivot_row;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    if (tid == 0) *status = 0;
    for (int64_t k = 0; k < n; ++k) {
        // pivot search in column k
        double best = -1.0;
        int bi = (int)k;
        for (int64_t i = k + tid; i < n; i += blockDim.x) {
            const double v = fabs(a[i * n + k]);
            if (v > best) {
                best = v;
                bi = (int)i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sval[warp] = best;
            sidx[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = sval[0];
            int bix = sidx[0];
            for (int w = 1; w < nwarps; ++w)
                if (sval[w] > bv || (sval[w] == bv && sidx[w] < bix)) {
                    bv = sval[w];
                    bix = sidx[w];
                }
            pivot_row = bix;
            piv[k] = bix;
            if (bv == 0.0 && *status == 0) *status = (int32_t)(k + 1);
        }
        __syncthreads();
        const int64_t p = pivot_row;
        if (p != k)
            for (int64_t jj = tid; jj < n; jj += blockDim.x) {
                const double t = a[k * n + jj];
                a[k * n + jj] = a[p * n + jj];
                a[p * n + jj] = t;
            }
        __syncthreads();
        const double d = a[k * n + k];
        const double inv = d != 0.0 ? 1.0 / d : 0.0;
        for (int64_t i = k + 1 + tid; i < n; i += blockDim.x) a[i * n + k] *= inv;
        __syncthreads();
        // trailing update, one warp per row, lanes along columns
        for (int64_t i = k + 1 + warp; i < n; i += nwarps) {
            const double lik = a[i * n + k];
            if (lik != 0.0)
                for (int64_t jj = k + 1 + lane; jj < n; jj += 32) a[i * n + jj] -= lik * a[k * n + jj];
        }
        __syncthreads();
    }
}

// Blocked LU, panel step: columns [k0, k1) of the row-major (n, n) matrix, rows k0..n-1,
// one CTA.  Partial pivoting as in k_lu_factor (the pivot swap moves whole rows, all n
// columns, so the left factor and the trailing part stay consistent); the rank-1 updates
// are confined to the panel's columns.  The caller then solves for the U rows right of
// the panel (k_lu_trsm) and updates the trailing matrix with one GEMM.
__global__ void __launch_bounds__(1024) k_lu_panel(int64_t n, int64_t k0, int64_t k1,
                                                   double *__restrict__ a, int32_t *__restrict__ piv,
                                                   int32_t *__restrict__ status)
{
    __shared__ double sval[32];
    __shared__ int sidx[32];
    __shared__ int pivot_row;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int64_t k = k0; k < k1; ++k) {
        double best = -1.0;
        int bi = (int)k;
        for (int64_t i = k + tid; i < n; i += blockDim.x) {
            const double v = fabs(a[i * n + k]);
            if (v > best) {
                best = v;
                bi = (int)i;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            sval[warp] = best;
            sidx[warp] = bi;
        }
        __syncthreads();
        if (tid == 0) {
            double bv = sval[0];
            int bix = sidx[0];
            for (int w = 1; w < nwarps; ++w)
                if (sval[w] > bv || (sval[w] == bv && sidx[w] < bix)) {
                    bv = sval[w];
                    bix = sidx[w];
                }
            pivot_row = bix;
            piv[k] = bix;
            if (bv == 0.0 && *status == 0) *status = (int32_t)(k + 1);
        }
        __syncthreads();
        const int64_t p = pivot_row;
        if (p != k)
            for (int64_t jj = tid; jj < n; jj += blockDim.x) {
                const double t = a[k * n + jj];
                a[k * n + jj] = a[p * n + jj];
                a[p * n + jj] = t;
            }
        __syncthreads();
        const double d = a[k * n + k];
        const double inv = d != 0.0 ? 1.0 / d : 0.0;
        for (int64_t i = k + 1 + tid; i < n; i += blockDim.x) a[i * n + k] *= inv;
        __syncthreads();
        for (int64_t i = k + 1 + warp; i < n; i += nwarps) {
            const double lik = a[i * n + k];
            if (lik != 0.0)
                for (int64_t jj = k + 1 + lane; jj < k1; jj += 32) a[i * n + jj] -= lik * a[k * n + jj];
        }
        __syncthreads();
    }
}

// Blocked LU, U rows right of the panel: rows [k0, k1), columns [k1, n) become
// L11^-1 times themselves (L11 unit lower triangular); one thread per column.
__global__ void k_lu_trsm(int64_t n, int64_t k0, int64_t k1, double *__restrict__ a)
{
    const int64_t col = k1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n) return;
    for (int64_t i = k0 + 1; i < k1; ++i) {
        double s = a[i * n + col];
        for (int64_t j = k0; j < i; ++j) s -= a[i * n + j] * a[j * n + col];
        a[i * n + col] = s;
    }
}

// Blocked LU, trailing update: A[i][j] -= sum_{k in [k0, k1)} A[i][k] A[k][j] for i, j >= k1
// (the Schur complement of the panel).  One CTA per 64 x 64 tile of the trailing matrix;
// the panel width (<= 64) is taken in chunks of 32: the tile's rows of the left factor and
// columns of the U rows are staged in shared memory and each of the 256 threads
// accumulates a 4 x 4 block in FP64.
constexpr int kLuTile = 64;
constexpr int kLuK = 32;
__global__ void __launch_bounds__(256) k_lu_update(int64_t n, int64_t k0, int64_t k1,
                                                   double *__restrict__ a)
{
    __shared__ double sl[kLuTile][kLuK + 1];   // [row][k]
    __shared__ double su[kLuTile][kLuK + 1];   // [col][k]
    const int kw = (int)(k1 - k0);
    const int64_t r0 = k1 + (int64_t)blockIdx.y * kLuTile, c0 = k1 + (int64_t)blockIdx.x * kLuTile;
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;   // rows 4 ty + i, columns tx + 16 j
    double acc[4][4] = {};
    for (int kc = 0; kc < kw; kc += kLuK) {
        for (int e = tid; e < kLuTile * kLuK; e += 256) {
            // left factor: consecutive threads take consecutive k of a row
            const int r = e / kLuK, k = e % kLuK;
            const int64_t gr = r0 + r;
            sl[r][k] = (gr < n && kc + k < kw) ? a[gr * n + k0 + kc + k] : 0.0;
            // U rows: consecutive threads take consecutive columns of a row
            const int kk = e / kLuTile, c = e % kLuTile;
            const int64_t gc = c0 + c;
            su[c][kk] = (gc < n && kc + kk < kw) ? a[(k0 + kc + kk) * n + gc] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < kLuK; ++k) {
            double l[4], u[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) l[i] = sl[4 * ty + i][k];
#pragma unroll
            for (int j = 0; j < 4; ++j) u[j] = su[tx + 16 * j][k];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(l[i], u[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t gr = r0 + 4 * ty + i;
        if (gr >= n) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t gc = c0 + tx + 16 * j;
            if (gc < n) a[gr * n + gc] -= acc[i][j];
        }
    }
}

// One warp per right-hand-side column: P, then L (unit) forward, then U backward.
// b is (n, nrhs) row-major.
__global__ void k_lu_solve(int64_t n, const double *__restrict__ lu, const int32_t *__restrict__ piv,
                           int64_t nrhs, double *__restrict__ b)
{
    const int64_t col = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (col >= nrhs) return;
    if (lane == 0)
        for (int64_t k = 0; k < n; ++k) {
            const int64_t p = piv[k];
            if (p != k) {
                const double t = b[k * nrhs + col];
                b[k * nrhs + col] = b[p * nrhs + col];
                b[p * nrhs + col] = t;
            }
        }
    __syncwarp();
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t jj = lane; jj < i; jj += 32) s += lu[i * n + jj] * b[jj * nrhs + col];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) b[i * nrhs + col] -= s;
        __syncwarp();
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = 0.0;
        for (int64_t jj = i + 1 + lane; jj < n; jj += 32) s += lu[i * n + jj] * b[jj * nrhs + col];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) b[i * nrhs + col] = (b[i * nrhs + col] - s) / lu[i * n + i];
        __syncwarp();
    }
}

// Blocked solve for many right-hand sides: one CTA per kLuCB columns of b, held in shared
// memory.  Rows go in blocks of 32: the contributions of the rows solved so far are summed
// by all 256 threads (thread = (row, one eighth of the columns j), partials added in a fixed
// order), then the 32 x 32 diagonal block is solved by one warp per column with shuffles.
// The same arithmetic as k_lu_solve up to the order of the sums.
constexpr int kLuCB = 4;      // right-hand sides per CTA
constexpr int kLuRB = 32;     // rows per block

__device__ __forceinline__ void lu_block_sums(int64_t n, const double *__restrict__ lu, const double *x,
                                              int64_t r0, int rows, int64_t jbeg, int64_t jend,
                                              double (*part)[kLuCB])
{
    const int tid = threadIdx.x, r = tid >> 3, pt = tid & 7;
    double acc[kLuCB];
#pragma unroll
    for (int c = 0; c < kLuCB; ++c) acc[c] = 0.0;
    if (r < rows) {
        const double *row = lu + (r0 + r) * n;
        for (int64_t j = jbeg + pt; j < jend; j += 8) {
            const double l = __ldg(row + j);
#pragma unroll
            for (int c = 0; c < kLuCB; ++c) acc[c] = fma(l, x[j * kLuCB + c], acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < kLuCB; ++c)
        for (int o = 1; o < 8; o <<= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (pt == 0 && r < rows)
#pragma unroll
        for (int c = 0; c < kLuCB; ++c) part[r][c] = acc[c];
}

__global__ void __launch_bounds__(256) k_lu_solve_blk(int64_t n, const double *__restrict__ lu,
                                                      const int32_t *__restrict__ piv, int64_t nrhs,
                                                      double *__restrict__ b)
{
    extern __shared__ double xs[];                   // [n][kLuCB]
    __shared__ double part[kLuRB][kLuCB];
    __shared__ double dg[kLuRB][kLuRB + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t c0 = (int64_t)blockIdx.x * kLuCB;
    const int ncol = (int)(nrhs - c0 < kLuCB ? nrhs - c0 : kLuCB);
    for (int64_t i = tid; i < n * kLuCB; i += blockDim.x) {
        const int64_t r = i / kLuCB;
        const int c = (int)(i % kLuCB);
        xs[i] = c < ncol ? b[r * nrhs + c0 + c] : 0.0;
    }
    __syncthreads();
    if (tid < kLuCB)   // row interchanges, in order
        for (int64_t k = 0; k < n; ++k) {
            const int64_t p = piv[k];
            if (p != k) {
                const double t = xs[k * kLuCB + tid];
                xs[k * kLuCB + tid] = xs[p * kLuCB + tid];
                xs[p * kLuCB + tid] = t;
            }
        }
    const int64_t nblk = (n + kLuRB - 1) / kLuRB;
    // forward: L with unit diagonal
    for (int64_t I = 0; I < nblk; ++I) {
        const int64_t r0 = I * kLuRB;
        const int rows = (int)(n - r0 < kLuRB ? n - r0 : kLuRB);
        __syncthreads();
        lu_block_sums(n, lu, xs, r0, rows, 0, r0, part);
        for (int i = tid; i < kLuRB * kLuRB; i += blockDim.x) {
            const int rr = i / kLuRB, kk = i % kLuRB;
            dg[rr][kk] = (rr < rows && kk < rows) ? lu[(r0 + rr) * n + r0 + kk] : 0.0;
        }
        __syncthreads();
        if (warp < kLuCB) {
            const int c = warp;
            double v = lane < rows ? xs[(r0 + lane) * kLuCB + c] - part[lane][c] : 0.0;
            for (int k = 0; k < rows; ++k) {
                const double xk = __shfl_sync(0xffffffffu, v, k);
                if (lane > k) v = fma(-dg[lane][k], xk, v);
            }
            if (lane < rows) xs[(r0 + lane) * kLuCB + c] = v;
        }
    }
    // backward: U
    for (int64_t I = nblk - 1; I >= 0; --I) {
        const int64_t r0 = I * kLuRB;
        const int rows = (int)(n - r0 < kLuRB ? n - r0 : kLuRB);
        __syncthreads();
        lu_block_sums(n, lu, xs, r0, rows, r0 + rows, n, part);
        for (int i = tid; i < kLuRB * kLuRB; i += blockDim.x) {
            const int rr = i / kLuRB, kk = i % kLuRB;
            dg[rr][kk] = (rr < rows && kk < rows) ? lu[(r0 + rr) * n + r0 + kk] : 1.0;
        }
        __syncthreads();
        if (warp < kLuCB) {
            const int c = warp;
            double v = lane < rows ? xs[(r0 + lane) * kLuCB + c] - part[lane][c] : 0.0;
            for (int k = rows - 1; k >= 0; --k) {
                if (lane == k) v = v / dg[k][k];
                const double xk = __shfl_sync(0xffffffffu, v, k);
                if (lane < k) v = fma(-dg[lane][k], xk, v);
            }
            if (lane < rows) xs[(r0 + lane) * kLuCB + c] = v;
        }
    }
    __syncthreads();
    for (int64_t i = tid; i < n * kLuCB; i += blockDim.x) {
        const int64_t r = i / kLuCB;
        const int c = (int)(i % kLuCB);
        if (c < ncol) b[r * nrhs + c0 + c] = xs[i];
    }
}

}  // namespace gm

using namespace gm;

extern "C" int gm_pseudo_cl(int64_t lmax, int64_t n1, const double *alm1, int64_t n2,
                            const double *alm2, double *cls, void *stream)
{
    if (lmax < 0 || n1 < 1 || n2 < 1 || n1 * n2 > 65535) return GM_ERR_BAD_SHAPE;
    if (!alm1 || !alm2 || !cls) return GM_ERR_BAD_PTR;
    const int64_t L = lmax + 1;
    cudaStream_t s = as_stream(stream);
    dim3 grid((unsigned)((L + kPclLanes - 1) / kPclLanes), (unsigned)(n1 * n2));
    k_pseudo_cl<<<grid, kPclLanes * kPclWarps, 0, s>>>(lmax, n1, (const double2 *)alm1, n2,
                                                       (const double2 *)alm2, cls);
    return check_launch("gm_pseudo_cl");
}

extern "C" int gm_coupling_blocks(int64_t lmax, const double *window, int64_t nw, int which,
                                  double *blocks, int64_t *queue, void *stream)
{
    if (lmax < 0 || lmax > 65535 || nw < 0) return GM_ERR_BAD_SHAPE;
    if (which <= 0 || which > 15) return GM_ERR_UNSUPPORTED;
    if (!window || !blocks || !queue) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    const int64_t n = lmax + 1;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int64_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(blocks, 0, sizeof(double) * 4 * n * n, s);
    if (e != cudaSuccess) {
        set_error("gm_coupling_blocks memset", e);
        return GM_ERR_LAUNCH;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    k_coupling<<<nsm * 8, 128, 0, s>>>(lmax, window, nw, which, blocks,
                                       reinterpret_cast<unsigned long long *>(queue));
    return check_launch("gm_coupling_blocks");
}

extern "C" int64_t gm_coupling_units(int64_t lmax) { return lmax < 0 ? 0 : total_units(lmax); }

extern "C" int gm_coupling_blocks_multi(int64_t njobs, const int64_t *jobs, int64_t nunits,
                                        const double *windows, double *blocks, int64_t *queue,
                                        void *stream)
{
    if (njobs < 1 || nunits < 1) return GM_ERR_BAD_SHAPE;
    if (!jobs || !windows || !blocks || !queue) return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int64_t), s);
    if (e != cudaSuccess) {
        set_error("gm_coupling_blocks_multi memset", e);
        return GM_ERR_LAUNCH;
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    k_coupling_multi<<<nsm * 8, 128, 0, s>>>(njobs, jobs, nunits, windows, blocks,
                                             reinterpret_cast<unsigned long long *>(queue));
    return check_launch("gm_coupling_blocks_multi");
}

extern "C" int gm_coupling_pairs_tt(int64_t lmax, const double *window, int64_t nw,
                                    const int32_t *pairs, int64_t npairs, double *S, void *stream)
{
    if (lmax < 0 || nw < 0 || npairs < 0) return GM_ERR_BAD_SHAPE;
    if (npairs == 0) return GM_OK;
    if (!window || !pairs || !S) return GM_ERR_BAD_PTR;
    k_coupling_pairs_tt<<<(unsigned)((npairs + 127) / 128), 128, 0, as_stream(stream)>>>(
        lmax, window, nw, pairs, npairs, S);
    return check_launch("gm_coupling_pairs_tt");
}

extern "C" int gm_toeplitz_fill(int64_t lmax, int64_t l_toeplitz, int64_t l_exact, int64_t dl_band,
                                const double *S, double *out, void *stream)
{
    if (lmax < 1 || l_toeplitz < 1 || l_exact < 0 || dl_band < 0 || l_exact > l_toeplitz ||
        l_toeplitz >= lmax || dl_band >= lmax || lmax >= 65535)
        return GM_ERR_BAD_SHAPE;
    if (!S || !out) return GM_ERR_BAD_PTR;
    const int64_t n = lmax + 1;
    dim3 grid((unsigned)((n + 127) / 128), (unsigned)n);
    k_toeplitz_fill<<<grid, 128, 0, as_stream(stream)>>>(lmax, l_toeplitz, l_exact, dl_band, S, out);
    return check_launch("gm_toeplitz_fill");
}

// Binning operators are passed in CSR form to support any NmtBin.
extern "C" int gm_bin_coupling_csr(int64_t lmax, int64_t nbands, int ncls, const double *blocks,
                                   const int32_t *band_ptr, const int32_t *band_ells,
                                   const double *wfl, const double *inv_fl, const double *beam,
                                   double *scratch, double *out, void *stream)
{
    if (lmax < 0 || nbands < 1 || nbands > 65535 || (ncls != 1 && ncls != 2 && ncls != 4))
        return GM_ERR_BAD_SHAPE;
    if (!blocks || !band_ptr || !band_ells || !wfl || !inv_fl || !beam || !scratch || !out)
        return GM_ERR_BAD_PTR;
    cudaStream_t s = as_stream(stream);
    const int64_t n = lmax + 1, nn = n * n, nb2 = nbands * nbands;
    dim3 grid((unsigned)nbands, (unsigned)nbands);
    // block slots: tt 0, te 1, pp 2, mm 3
    if (ncls == 1) {
        k_bin_block<<<grid, 256, 0, s>>>(lmax, nbands, blocks, band_ptr, band_ells, wfl, inv_fl,
                                         beam, scratch);
    } else if (ncls == 2) {
        k_bin_block<<<grid, 256, 0, s>>>(lmax, nbands, blocks + nn, band_ptr, band_ells, wfl,
                                         inv_fl, beam, scratch);
    } else {
        k_bin_block<<<grid, 256, 0, s>>>(lmax, nbands, blocks + 2 * nn, band_ptr, band_ells, wfl,
                                         inv_fl, beam, scratch);
        k_bin_block<<<grid, 256, 0, s>>>(lmax, nbands, blocks + 3 * nn, band_ptr, band_ells, wfl,
                                         inv_fl, beam, scratch + nb2);
    }
    const int64_t N = ncls * nbands;
    k_place_binned<<<(unsigned)((N * N + 255) / 256), 256, 0, s>>>(nbands, ncls, scratch, out);
    return check_launch("gm_bin_coupling");
}

extern "C" int gm_bin_cells_csr(int64_t lmax, int64_t nbands, int64_t ncls, const double *cls,
                                const int32_t *band_ptr, const int32_t *band_ells,
                                const double *wfl, double *out, void *stream)
{
    if (lmax < 0 || nbands < 1 || ncls < 1) return GM_ERR_BAD_SHAPE;
    if (!cls || !band_ptr || !band_ells || !wfl || !out) return GM_ERR_BAD_PTR;
    const int64_t tot = nbands * ncls;
    k_bin_cells<<<(unsigned)((tot + 255) / 256), 256, 0, as_stream(stream)>>>(
        lmax, nbands, ncls, cls, band_ptr, band_ells, wfl, out);
    return check_launch("gm_bin_cells");
}

extern "C" int gm_lu_factor(int64_t n, double *a, int32_t *piv, int32_t *status, void *stream)
{
    if (n < 1 || n > 65535) return GM_ERR_BAD_SHAPE;
    if (!a || !piv || !status) return GM_ERR_BAD_PTR;
    k_lu_factor<<<1, 1024, 0, as_stream(stream)>>>(n, a, piv, status);
    return check_launch("gm_lu_factor");
}

extern "C" int gm_lu_panel(int64_t n, double *a, int64_t k0, int64_t k1, int32_t *piv,
                           int32_t *status, void *stream)
{
    if (n < 1 || n > 65535 || k0 < 0 || k1 <= k0 || k1 > n) return GM_ERR_BAD_SHAPE;
    if (!a || !piv || !status) return GM_ERR_BAD_PTR;
    k_lu_panel<<<1, 1024, 0, as_stream(stream)>>>(n, k0, k1, a, piv, status);
    return check_launch("gm_lu_panel");
}

extern "C" int gm_lu_trsm(int64_t n, double *a, int64_t k0, int64_t k1, void *stream)
{
    if (n < 1 || n > 65535 || k0 < 0 || k1 <= k0 || k1 > n) return GM_ERR_BAD_SHAPE;
    if (!a) return GM_ERR_BAD_PTR;
    if (k1 == n) return GM_OK;
    k_lu_trsm<<<(unsigned)((n - k1 + 127) / 128), 128, 0, as_stream(stream)>>>(n, k0, k1, a);
    return check_launch("gm_lu_trsm");
}

extern "C" int gm_lu_update(int64_t n, double *a, int64_t k0, int64_t k1, void *stream)
{
    if (n < 1 || k0 < 0 || k1 <= k0 || k1 - k0 > kLuTile || k1 > n) return GM_ERR_BAD_SHAPE;
    if (!a) return GM_ERR_BAD_PTR;
    if (k1 == n) return GM_OK;
    const unsigned t = (unsigned)((n - k1 + kLuTile - 1) / kLuTile);
    k_lu_update<<<dim3(t, t), 256, 0, as_stream(stream)>>>(n, k0, k1, a);
    return check_launch("gm_lu_update");
}

extern "C" int gm_lu_solve(int64_t n, const double *lu, const int32_t *piv, int64_t nrhs,
                           double *b, void *stream)
{
    if (n < 1 || nrhs < 1) return GM_ERR_BAD_SHAPE;
    if (!lu || !piv || !b) return GM_ERR_BAD_PTR;
    const size_t smem = (size_t)n * kLuCB * sizeof(double);
    if (smem <= 200 * 1024) {
        // the columns of b fit in shared memory: the blocked solve
        cudaError_t e = cudaFuncSetAttribute(k_lu_solve_blk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) {
            set_error("gm_lu_solve attr", e);
            return GM_ERR_LAUNCH;
        }
        k_lu_solve_blk<<<(unsigned)((nrhs + kLuCB - 1) / kLuCB), 256, smem, as_stream(stream)>>>(n, lu, piv,
                                                                                                nrhs, b);
        return check_launch("gm_lu_solve");
    }
    const int64_t threads = 256, warps_per = threads / 32;
    k_lu_solve<<<(unsigned)((nrhs + warps_per - 1) / warps_per), (unsigned)threads, 0,
                 as_stream(stream)>>>(n, lu, piv, nrhs, b);
    return check_launch("gm_lu_solve");
}
