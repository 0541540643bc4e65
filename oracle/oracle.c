/*
 * FP64 CPU oracle for the pseudo-C_ell MASTER hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against: it is imported by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline / --impl reference legs of bench.py, and by nothing else.  The
 * product (gmaster_b200/) never links, loads or calls it.
 *
 * Every routine restates, in plain C99 + OpenMP and in double precision, the
 * mathematics of the reference (licongxu/GMaster) for one step of the path;
 * each cites the reference file:line it follows.  It is written from the
 * definitions, not from the reference's staging: the transforms are direct sums
 * over rings (no hemisphere fold, no ring-fold residual), so the CUDA kernels'
 * algebra is checked against an independent formulation.
 *
 * Conventions (all as in the reference):
 *   - HEALPix RING geometry, gmaster/utils.py:223-249.
 *   - Ring Fourier sums F_r(m) = sum_p x_p exp(-i m phi_p),
 *     phi_p = phi0_r + 2 pi p / nphi_r (tests/test_sht.py:478-491).
 *   - Quadrature weight 4 pi / npix for every pixel (utils.py:245).
 *   - sY_lm(theta, phi) = (-1)^s sqrt((2l+1)/4pi) d^l_{m,-s}(theta) e^{i m phi}
 *     (docs/notes/latitudinal_march_maths.md eq. (1); healpix.py:117-143).
 *   - E/B from the spin +-2 coefficients: E = -(a2 + a-2)/2, B = i(a2 - a-2)/2
 *     (healpix.py:812-814), synthesis packing healpix.py:599-611.
 *   - Jacobi refinement alm <- alm - A(S(alm) - map) (healpix.py:1059-1068).
 *   - Healpy m-major packing idx = m(2 lmax + 1 - m)/2 + l (utils.py:515-521).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* Geometry (gmaster/utils.py:223-249)                                        */
/* ------------------------------------------------------------------------- */

void orc_geometry(int64_t nside, double *theta, double *phi0, int64_t *nphi,
                  int64_t *offset)
{
    int64_t nring = 4 * nside - 1;
    int64_t npix = 12 * nside * nside;
    double belt_step = (double)(8 * nside) / (double)npix;
    double cap_den = sqrt(6.0) * (double)nside;
    int64_t start = 0;
    for (int64_t r = 0; r < nring; ++r) {
        int64_t ring = r + 1;
        int64_t north = ring > 2 * nside ? 4 * nside - ring : ring;
        double th, ph;
        int64_t n;
        if (north < nside) {
            th = 2.0 * asin((double)north / cap_den);
            ph = M_PI / (double)(4 * north);
            n = 4 * north;
        } else {
            th = acos((double)(2 * nside - north) * belt_step);
            ph = (((north - nside) & 1) == 0) ? M_PI / (double)(4 * nside) : 0.0;
            n = 4 * nside;
        }
        if (north != ring) th = M_PI - th;
        theta[r] = th;
        phi0[r] = ph;
        nphi[r] = n;
        offset[r] = start;
        start += n;
    }
}

/* ------------------------------------------------------------------------- */
/* Mixed-radix complex DFT, out-of-place, sign = -1 forward, +1 backward.     */
/* Recursive decimation in time over the smallest prime factor; O(n sum p).   */
/* ------------------------------------------------------------------------- */

static int smallest_factor(int64_t n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int64_t p = 3; p * p <= n; p += 2)
        if (n % p == 0) return (int)p;
    return (int)n;
}

/* x: n complex values read with stride `stride` (interleaved re/im),
 * y: n complex values written contiguously.  tw holds exp(sign 2 pi i k / N) for the
 * top-level length N; this level uses tw[(k * tstride) mod N] with tstride = N / n. */
static void dft_rec(int64_t n, const double *x, int64_t stride, double *y, const double *tw,
                    int64_t N, int64_t tstride, double *work)
{
    if (n == 1) {
        y[0] = x[0];
        y[1] = x[1];
        return;
    }
    int p = smallest_factor(n);
    int64_t q = n / p;
    for (int r = 0; r < p; ++r)
        dft_rec(q, x + 2 * r * stride, stride * p, work + 2 * r * q, tw, N, tstride * p,
                work + 2 * n);
    for (int64_t k = 0; k < q; ++k) {
        for (int v = 0; v < p; ++v) {
            int64_t kk = k + v * q;
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; ++r) {
                int64_t e = ((r * kk) % n) * tstride;
                double c = tw[2 * e], s = tw[2 * e + 1];
                double ar = work[2 * (r * q + k)], ai = work[2 * (r * q + k) + 1];
                sr += ar * c - ai * s;
                si += ar * s + ai * c;
            }
            y[2 * kk] = sr;
            y[2 * kk + 1] = si;
        }
    }
}

/* Workspace for dft_rec: sum over recursion levels of 2n doubles < 4n doubles. */
void orc_dft(int64_t n, const double *x, double *y, int sign)
{
    double *work = (double *)malloc(sizeof(double) * 8 * (size_t)n + 64);
    double *tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int64_t k = 0; k < n; ++k) {
        double ang = sign * 2.0 * M_PI * (double)k / (double)n;
        tw[2 * k] = cos(ang);
        tw[2 * k + 1] = sin(ang);
    }
    dft_rec(n, x, 1, y, tw, n, 1, work);
    free(work);
    free(tw);
}

/* ------------------------------------------------------------------------- */
/* Ring stage                                                                 */
/* ------------------------------------------------------------------------- */

/* F[r][m] = sum_p x_p exp(-i m phi_p) for m in [-(mneg), L), complex interleaved.
 * Rows hold (mneg + L) entries; entry j is order m = j - mneg.
 * Input map is complex (interleaved) so spin fields Q+iU fit; real maps have im 0. */
void orc_ring_analysis(int64_t nside, int64_t L, int64_t mneg, const double *phi0,
                       const double *mapc, double *F)
{
    int64_t nring = 4 * nside - 1;
    double *theta = malloc(sizeof(double) * nring), *phi0_c = malloc(sizeof(double) * nring);
    int64_t *nphi = malloc(sizeof(int64_t) * nring), *off = malloc(sizeof(int64_t) * nring);
    orc_geometry(nside, theta, phi0_c, nphi, off);
    int64_t width = mneg + L;
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nring; ++r) {
        int64_t n = nphi[r];
        double *d = malloc(sizeof(double) * 2 * n);
        orc_dft(n, mapc + 2 * off[r], d, -1);
        for (int64_t j = 0; j < width; ++j) {
            int64_t m = j - mneg;
            int64_t k = ((m % n) + n) % n;
            double ang = -(double)m * phi0[r];
            double c = cos(ang), s = sin(ang);
            double ar = d[2 * k], ai = d[2 * k + 1];
            F[2 * (r * width + j)] = ar * c - ai * s;
            F[2 * (r * width + j) + 1] = ar * s + ai * c;
        }
        free(d);
    }
    free(theta); free(phi0_c); free(nphi); free(off);
}

/* map_p = sum_{m=-mneg}^{L-1} C[r][m] exp(i m phi_p) (complex output). */
void orc_ring_synthesis(int64_t nside, int64_t L, int64_t mneg, const double *phi0,
                        const double *C, double *mapc)
{
    int64_t nring = 4 * nside - 1;
    double *theta = malloc(sizeof(double) * nring), *phi0_c = malloc(sizeof(double) * nring);
    int64_t *nphi = malloc(sizeof(int64_t) * nring), *off = malloc(sizeof(int64_t) * nring);
    orc_geometry(nside, theta, phi0_c, nphi, off);
    int64_t width = mneg + L;
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nring; ++r) {
        int64_t n = nphi[r];
        double *s = calloc(2 * n, sizeof(double));
        double *d = malloc(sizeof(double) * 2 * n);
        for (int64_t j = 0; j < width; ++j) {
            int64_t m = j - mneg;
            int64_t k = ((m % n) + n) % n;
            double ang = (double)m * phi0[r];
            double c = cos(ang), sn = sin(ang);
            double ar = C[2 * (r * width + j)], ai = C[2 * (r * width + j) + 1];
            s[2 * k] += ar * c - ai * sn;
            s[2 * k + 1] += ar * sn + ai * c;
        }
        orc_dft(n, s, d, +1);
        memcpy(mapc + 2 * off[r], d, sizeof(double) * 2 * n);
        free(s); free(d);
    }
    free(theta); free(phi0_c); free(nphi); free(off);
}

/* ------------------------------------------------------------------------- */
/* Spin-weighted Legendre rows                                                */
/* lam[l] = sqrt((2l+1)/4pi) d^l_{m,sp}(theta) for l in [0, lmax], |m| <= l.  */
/* Normalised three-term recurrence in l (Edmonds 4.1.23 / DLMF 18.9.2 in     */
/* normalised form, the recurrence the reference marches,                     */
/* docs/notes/latitudinal_march_maths.md §2), seeded at l0 = max(|m|, |sp|)    */
/* from the closed form d^j_{m' j} / d^j_{j m'} with an explicit binary        */
/* exponent so that sin^m underflow is carried exactly                         */
/* (latitudinal_march_maths.md §3).                                            */
/* ------------------------------------------------------------------------- */

#define ORC_SCALE_BITS 600

/* log2 of sqrt(binomial(2j, j + k)) */
static double log2_sqrt_binom(int64_t two_j, int64_t k)
{
    return 0.5 * (lgamma((double)two_j + 1.0) - lgamma((double)k + 1.0) -
                  lgamma((double)(two_j - k) + 1.0)) / log(2.0);
}

void orc_lambda_row(int64_t lmax, int64_t m, int64_t sp, double theta, double *lam)
{
    for (int64_t l = 0; l <= lmax; ++l) lam[l] = 0.0;
    if (m < 0) {
        /* d^l_{m,sp} = (-1)^(m - sp) d^l_{-m,-sp} */
        orc_lambda_row(lmax, -m, -sp, theta, lam);
        if (((-m) - sp) & 1)  /* (m - sp) parity */
            for (int64_t l = 0; l <= lmax; ++l) lam[l] = -lam[l];
        return;
    }
    int64_t am = m, as = sp < 0 ? -sp : sp;
    int64_t l0 = am > as ? am : as;
    if (l0 > lmax) return;
    double ch = cos(0.5 * theta), sh = sin(0.5 * theta);
    double lc = ch > 0 ? log2(ch) : -HUGE_VAL, ls = sh > 0 ? log2(sh) : -HUGE_VAL;
    double lg, sign = 1.0;
    int64_t pc, ps;
    if (am >= as) {
        /* d^m_{m,sp} = (-1)^(m - sp) sqrt(C(2m, m+sp)) cos^{m+sp} sin^{m-sp} */
        pc = am + sp; ps = am - sp;
        lg = log2_sqrt_binom(2 * am, am + sp);
        if ((am - sp) & 1) sign = -1.0;
    } else if (sp > 0) {
        /* d^s_{m,s} = sqrt(C(2s, s+m)) cos^{s+m} sin^{s-m} */
        pc = as + am; ps = as - am;
        lg = log2_sqrt_binom(2 * as, as + am);
    } else {
        /* d^s_{m,-s} = (-1)^(m+s) sqrt(C(2s, s-m)) cos^{s-m} sin^{s+m} */
        pc = as - am; ps = as + am;
        lg = log2_sqrt_binom(2 * as, as - am);
        if ((am + as) & 1) sign = -1.0;
    }
    double f = lg + 0.5 * log2((2.0 * l0 + 1.0) / (4.0 * M_PI));
    if (pc) f += pc * lc;
    if (ps) f += ps * ls;
    if (!(f > -1e300)) return;  /* exactly zero (pole) */
    /* value = sign * 2^f, carried as v * 2^(S*k) */
    int64_t k = 0;
    if (f < -(double)ORC_SCALE_BITS / 2) {
        k = (int64_t)floor((f + ORC_SCALE_BITS / 2) / ORC_SCALE_BITS);
    }
    double v_cur = sign * exp2(f - (double)(ORC_SCALE_BITS * k));
    double v_prev = 0.0;
    double x = cos(theta);
    const double big = exp2(ORC_SCALE_BITS / 2), shrink = exp2(-ORC_SCALE_BITS);
    if (k == 0) lam[l0] = v_cur;
    double msp = (double)m * (double)sp;
    for (int64_t l = l0; l < lmax; ++l) {
        double dl = (double)l, dl1 = dl + 1.0;
        double den = sqrt((dl1 * dl1 - (double)(m * m)) * (dl1 * dl1 - (double)(sp * sp)));
        double alpha = sqrt((2 * dl + 3) * (2 * dl + 1)) * dl1 / den;
        double c = (l == 0) ? 0.0 : msp / (dl * dl1);
        double beta = 0.0;
        if (l > l0) {
            double num = sqrt((dl * dl - (double)(m * m)) * (dl * dl - (double)(sp * sp)));
            beta = sqrt((2 * dl + 3) / (2 * dl - 1)) * dl1 * num / (dl * den);
        }
        double v_next = alpha * (x - c) * v_cur - beta * v_prev;
        v_prev = v_cur;
        v_cur = v_next;
        if (k < 0 && fabs(v_cur) > big) {
            v_cur *= shrink;
            v_prev *= shrink;
            ++k;
        }
        if (k == 0) lam[l + 1] = v_cur;
    }
}

/* Same row from the Jacobi closed form (DLMF 18.9.2 over n with alpha = m + s',
 * beta = |m - s'|, the form of workspaces.py:608-679 and
 * latitudinal_march_maths.md §1), evaluated in long double.  Used only to pin
 * orc_lambda_row at moderate lmax (range of long double). */
void orc_lambda_row_jacobi(int64_t lmax, int64_t m, int64_t sp, double theta, double *lam)
{
    /* d^l_{m, sp} with first index m: a = |m - sp|, b = |m + sp| (Edmonds 4.1.23) */
    for (int64_t l = 0; l <= lmax; ++l) lam[l] = 0.0;
    int64_t a = m - sp; if (a < 0) a = -a;
    int64_t b = m + sp; if (b < 0) b = -b;
    int64_t M = (a + b) / 2;
    if (M > lmax) return;
    long double th = theta;
    long double sh = sinl(th / 2), ch = cosl(th / 2), x = cosl(th);
    /* xi = 1 if sp >= m else (-1)^(sp - m) */
    long double xi = 1.0L;
    if (sp < m && ((m - sp) & 1)) xi = -1.0L;
    long double pref = xi * powl(sh, (long double)a) * powl(ch, (long double)b);
    long double pprev = 0.0L, pcur = 0.0L;
    for (int64_t l = M; l <= lmax; ++l) {
        int64_t n = l - M;
        long double pn;
        if (n == 0) pn = 1.0L;
        else if (n == 1) pn = ((long double)(a - b) + (long double)(a + b + 2) * x) / 2.0L;
        else {
            long double nn = (long double)n, A = (long double)a, B = (long double)b;
            long double S = 2 * nn + A + B;
            pn = ((S - 1) * (S * (S - 2) * x + A * A - B * B) * pcur -
                  2 * (nn + A - 1) * (nn + B - 1) * S * pprev) /
                 (2 * nn * (nn + A + B) * (S - 2));
        }
        pprev = pcur;
        pcur = pn;
        long double lnorm = 0.5L * (lgammal((long double)n + 1) + lgammal((long double)(n + a + b) + 1) -
                                    lgammal((long double)(n + a) + 1) - lgammal((long double)(n + b) + 1));
        long double val = pref * expl(lnorm) * pn;
        lam[l] = (double)(val * sqrtl((2.0L * l + 1.0L) / (4.0L * (long double)M_PI)));
    }
}

/* ------------------------------------------------------------------------- */
/* Spherical-harmonic transforms                                              */
/* ------------------------------------------------------------------------- */

static inline int64_t alm_index(int64_t lmax, int64_t l, int64_t m)
{
    return m * (2 * lmax + 1 - m) / 2 + l;
}

/* Spin-0 analysis without refinement: alm[idx] (complex interleaved). */
static void ana0(int64_t nside, int64_t lmax, const double *theta, const double *phi0, const double *map, double *alm)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    double w = 4.0 * M_PI / (double)npix;
    double *mapc = calloc(2 * npix, sizeof(double));
    for (int64_t p = 0; p < npix; ++p) mapc[2 * p] = map[p];
    double *F = malloc(sizeof(double) * 2 * nring * L);
    orc_ring_analysis(nside, L, 0, phi0, mapc, F);
    (void)nring;
#pragma omp parallel for schedule(dynamic)
    for (int64_t m = 0; m <= lmax; ++m) {
        double *lam = malloc(sizeof(double) * L);
        double *acc = calloc(2 * L, sizeof(double));
        for (int64_t r = 0; r < nring; ++r) {
            orc_lambda_row(lmax, m, 0, theta[r], lam);
            double gr = w * F[2 * (r * L + m)], gi = w * F[2 * (r * L + m) + 1];
            for (int64_t l = m; l <= lmax; ++l) {
                acc[2 * l] += lam[l] * gr;
                acc[2 * l + 1] += lam[l] * gi;
            }
        }
        for (int64_t l = m; l <= lmax; ++l) {
            alm[2 * alm_index(lmax, l, m)] = acc[2 * l];
            alm[2 * alm_index(lmax, l, m) + 1] = acc[2 * l + 1];
        }
        free(lam); free(acc);
    }
    free(mapc); free(F); 
}

/* Spin-0 synthesis: map_p = sum_l [a_l0 Y_l0 + 2 Re sum_{m>0} a_lm Y_lm]. */
static void syn0(int64_t nside, int64_t lmax, const double *theta, const double *phi0, const double *alm, double *map)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    (void)nring;
    int64_t width = 2 * L - 1;
    double *C = calloc(2 * nring * width, sizeof(double));
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nring; ++r) {
        double *lam = malloc(sizeof(double) * L);
        for (int64_t m = 0; m <= lmax; ++m) {
            orc_lambda_row(lmax, m, 0, theta[r], lam);
            double sr = 0.0, si = 0.0;
            for (int64_t l = m; l <= lmax; ++l) {
                sr += lam[l] * alm[2 * alm_index(lmax, l, m)];
                si += lam[l] * alm[2 * alm_index(lmax, l, m) + 1];
            }
            /* order +m at column m + (L-1); order -m is the conjugate */
            C[2 * (r * width + (L - 1) + m)] = sr;
            C[2 * (r * width + (L - 1) + m) + 1] = si;
            if (m > 0) {
                C[2 * (r * width + (L - 1) - m)] = sr;
                C[2 * (r * width + (L - 1) - m) + 1] = -si;
            }
        }
        free(lam);
    }
    double *mapc = malloc(sizeof(double) * 2 * npix);
    orc_ring_synthesis(nside, L, L - 1, phi0, C, mapc);
    for (int64_t p = 0; p < npix; ++p) map[p] = mapc[2 * p];
    free(mapc); free(C); 
}

/* Spin-2 analysis: (Q, U) maps -> (E, B) alms, each complex interleaved. */
static void ana2(int64_t nside, int64_t lmax, const double *theta, const double *phi0, const double *qu, double *eb)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    double w = 4.0 * M_PI / (double)npix;
    int64_t nelem = L * (L + 1) / 2;
    double *mapc = malloc(sizeof(double) * 2 * npix);
    for (int64_t p = 0; p < npix; ++p) { mapc[2 * p] = qu[p]; mapc[2 * p + 1] = qu[npix + p]; }
    int64_t width = 2 * L - 1;
    double *F = malloc(sizeof(double) * 2 * nring * width);
    orc_ring_analysis(nside, L, L - 1, phi0, mapc, F);  /* FFT of P = Q + iU, m in (-L, L) */
    (void)nring;
#pragma omp parallel for schedule(dynamic)
    for (int64_t m = 0; m <= lmax; ++m) {
        double *lp = malloc(sizeof(double) * L), *lmn = malloc(sizeof(double) * L);
        double *ap = calloc(2 * L, sizeof(double)), *am = calloc(2 * L, sizeof(double));
        for (int64_t r = 0; r < nring; ++r) {
            /* lambda_{+2} = sqrt(..) d^l_{m,-2}, lambda_{-2} = sqrt(..) d^l_{m,+2} */
            orc_lambda_row(lmax, m, -2, theta[r], lp);
            orc_lambda_row(lmax, m, 2, theta[r], lmn);
            /* P~(m) = F[+m]; M~(m) = conj(F[-m]) is the ring sum of Q - iU */
            double pr = w * F[2 * (r * width + (L - 1) + m)], pi = w * F[2 * (r * width + (L - 1) + m) + 1];
            double mr = w * F[2 * (r * width + (L - 1) - m)], mi = -w * F[2 * (r * width + (L - 1) - m) + 1];
            for (int64_t l = m; l <= lmax; ++l) {
                ap[2 * l] += lp[l] * pr; ap[2 * l + 1] += lp[l] * pi;
                am[2 * l] += lmn[l] * mr; am[2 * l + 1] += lmn[l] * mi;
            }
        }
        for (int64_t l = m; l <= lmax; ++l) {
            int64_t i = alm_index(lmax, l, m);
            /* E = -(a2 + a-2)/2, B = i (a2 - a-2)/2 (healpix.py:812-814) */
            eb[2 * i] = -(ap[2 * l] + am[2 * l]) / 2;
            eb[2 * i + 1] = -(ap[2 * l + 1] + am[2 * l + 1]) / 2;
            eb[2 * (nelem + i)] = -(ap[2 * l + 1] - am[2 * l + 1]) / 2;
            eb[2 * (nelem + i) + 1] = (ap[2 * l] - am[2 * l]) / 2;
        }
        free(lp); free(lmn); free(ap); free(am);
    }
    free(mapc); free(F); 
}

/* Spin-2 synthesis: (E, B) -> (Q, U), with a2_lm = -(E + iB) for m >= 0 and
 * a2_{l,-m} = -(-1)^m (E* + i B*) (healpix.py:599-611). */
static void syns(int64_t nside, int64_t lmax, int64_t spin, const double *theta, const double *phi0,
                 const double *eb, double *qu)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    int64_t nelem = L * (L + 1) / 2;
    (void)nring;
    int64_t width = 2 * L - 1;
    double *C = calloc(2 * nring * width, sizeof(double));
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nring; ++r) {
        double *lam = malloc(sizeof(double) * L);
        for (int64_t mm = -lmax; mm <= lmax; ++mm) {
            int64_t m = mm < 0 ? -mm : mm;
            orc_lambda_row(lmax, mm, -spin, theta[r], lam);
            double sr = 0.0, si = 0.0;
            for (int64_t l = m; l <= lmax; ++l) {
                int64_t i = alm_index(lmax, l, m);
                double er = eb[2 * i], ei = eb[2 * i + 1];
                double br = eb[2 * (nelem + i)], bi = eb[2 * (nelem + i) + 1];
                double ar, ai;
                if (mm >= 0) {           /* -(E + iB) */
                    ar = -(er - bi); ai = -(ei + br);
                } else {                 /* -(-1)^m (E* + i B*) */
                    double sg = (m & 1) ? -1.0 : 1.0;
                    ar = -sg * (er + bi); ai = -sg * (-ei + br);
                }
                sr += lam[l] * ar;
                si += lam[l] * ai;
            }
            C[2 * (r * width + (L - 1) + mm)] = sr;
            C[2 * (r * width + (L - 1) + mm) + 1] = si;
        }
        free(lam);
    }
    double *mapc = malloc(sizeof(double) * 2 * npix);
    orc_ring_synthesis(nside, L, L - 1, phi0, C, mapc);
    for (int64_t p = 0; p < npix; ++p) { qu[p] = mapc[2 * p]; qu[npix + p] = mapc[2 * p + 1]; }
    free(mapc); free(C); 
}

/* Spin-s analysis (s >= 1) in the reference's literal form (healpix.py:800-814): with
 * plus(l, m) = sum over rings of w lambda_{l,m,-s} F(m), F the ring FFT of Q + iU for every
 * order -L < m < L, minus(l, m) = (-1)^m conj(plus(l, -m)), E = -(plus + minus)/2 and
 * B = i (plus - minus)/2. */
static void anas(int64_t nside, int64_t lmax, int64_t spin, const double *theta, const double *phi0,
                 const double *qu, double *eb)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    double w = 4.0 * M_PI / (double)npix;
    int64_t nelem = L * (L + 1) / 2;
    double *mapc = malloc(sizeof(double) * 2 * npix);
    for (int64_t p = 0; p < npix; ++p) { mapc[2 * p] = qu[p]; mapc[2 * p + 1] = qu[npix + p]; }
    int64_t width = 2 * L - 1;
    double *F = malloc(sizeof(double) * 2 * nring * width);
    orc_ring_analysis(nside, L, L - 1, phi0, mapc, F);
#pragma omp parallel for schedule(dynamic)
    for (int64_t m = 0; m <= lmax; ++m) {
        double *lp = malloc(sizeof(double) * L), *ln = malloc(sizeof(double) * L);
        double *pp = calloc(2 * L, sizeof(double)), *pn = calloc(2 * L, sizeof(double));
        for (int64_t r = 0; r < nring; ++r) {
            orc_lambda_row(lmax, m, -spin, theta[r], lp);
            orc_lambda_row(lmax, -m, -spin, theta[r], ln);
            double fr = w * F[2 * (r * width + (L - 1) + m)], fi = w * F[2 * (r * width + (L - 1) + m) + 1];
            double gr = w * F[2 * (r * width + (L - 1) - m)], gi = w * F[2 * (r * width + (L - 1) - m) + 1];
            for (int64_t l = m; l <= lmax; ++l) {
                pp[2 * l] += lp[l] * fr; pp[2 * l + 1] += lp[l] * fi;
                pn[2 * l] += ln[l] * gr; pn[2 * l + 1] += ln[l] * gi;
            }
        }
        double sg = (m & 1) ? -1.0 : 1.0;
        for (int64_t l = m; l <= lmax; ++l) {
            int64_t i = alm_index(lmax, l, m);
            double qr = sg * pn[2 * l], qi = -sg * pn[2 * l + 1];   /* minus = (-1)^m conj(plus(-m)) */
            eb[2 * i] = -(pp[2 * l] + qr) / 2;
            eb[2 * i + 1] = -(pp[2 * l + 1] + qi) / 2;
            eb[2 * (nelem + i)] = -(pp[2 * l + 1] - qi) / 2;
            eb[2 * (nelem + i) + 1] = (pp[2 * l] - qr) / 2;
        }
        free(lp); free(ln); free(pp); free(pn);
    }
    free(mapc); free(F);
}

void orc_alm2map(int64_t nside, int64_t lmax, int64_t spin, const double *theta,
                 const double *phi0, const double *alm, double *map)
{
    if (spin == 0) syn0(nside, lmax, theta, phi0, alm, map);
    else syns(nside, lmax, spin, theta, phi0, alm, map);
}

/* One analysis pass: spin 0, the spin-2 form pinned against the golden vectors, or the
 * literal spin-s form (`general` forces it for spin 2 too). */
static void ana_any(int64_t nside, int64_t lmax, int64_t spin, int general, const double *theta,
                    const double *phi0, const double *map, double *alm)
{
    if (spin == 0) ana0(nside, lmax, theta, phi0, map, alm);
    else if (spin == 2 && !general) ana2(nside, lmax, theta, phi0, map, alm);
    else anas(nside, lmax, spin, theta, phi0, map, alm);
}

/* map2alm with n_iter Jacobi refinement (healpix.py:1059-1068). */
static void map2alm_iter(int64_t nside, int64_t lmax, int64_t spin, int64_t n_iter, int general,
                         const double *theta, const double *phi0, const double *map, double *alm)
{
    int64_t npix = 12 * nside * nside, L = lmax + 1, nelem = L * (L + 1) / 2;
    int64_t nmaps = spin == 0 ? 1 : 2;
    ana_any(nside, lmax, spin, general, theta, phi0, map, alm);
    double *res = malloc(sizeof(double) * nmaps * npix);
    double *delta = malloc(sizeof(double) * 2 * nmaps * nelem);
    for (int64_t it = 0; it < n_iter; ++it) {
        orc_alm2map(nside, lmax, spin, theta, phi0, alm, res);
        for (int64_t p = 0; p < nmaps * npix; ++p) res[p] -= map[p];
        ana_any(nside, lmax, spin, general, theta, phi0, res, delta);
        for (int64_t i = 0; i < 2 * nmaps * nelem; ++i) alm[i] -= delta[i];
    }
    free(res); free(delta);
}

void orc_map2alm(int64_t nside, int64_t lmax, int64_t spin, int64_t n_iter,
                 const double *theta, const double *phi0, const double *map, double *alm)
{
    map2alm_iter(nside, lmax, spin, n_iter, 0, theta, phi0, map, alm);
}

/* As orc_map2alm, with the literal spin-s analysis for every spin >= 1 (checks it against
 * the spin-2 form). */
void orc_map2alm_general(int64_t nside, int64_t lmax, int64_t spin, int64_t n_iter,
                         const double *theta, const double *phi0, const double *map, double *alm)
{
    map2alm_iter(nside, lmax, spin, n_iter, 1, theta, phi0, map, alm);
}

/* Analysis restricted to a set of orders (bounded CPU-baseline sample): spin 0,
 * no refinement, alm rows for the orders in `ms` only (acc[im][l] complex). */
void orc_ana0_orders(int64_t nside, int64_t lmax, const double *theta, const double *phi0, const double *map, int64_t nm,
                     const int64_t *ms, double *acc_out)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    double w = 4.0 * M_PI / (double)npix;
    double *mapc = calloc(2 * npix, sizeof(double));
    for (int64_t p = 0; p < npix; ++p) mapc[2 * p] = map[p];
    double *F = malloc(sizeof(double) * 2 * nring * L);
    orc_ring_analysis(nside, L, 0, phi0, mapc, F);
    (void)nring;
#pragma omp parallel for schedule(dynamic)
    for (int64_t im = 0; im < nm; ++im) {
        int64_t m = ms[im];
        double *lam = malloc(sizeof(double) * L);
        double *acc = acc_out + 2 * im * L;
        memset(acc, 0, sizeof(double) * 2 * L);
        for (int64_t r = 0; r < nring; ++r) {
            orc_lambda_row(lmax, m, 0, theta[r], lam);
            double gr = w * F[2 * (r * L + m)], gi = w * F[2 * (r * L + m) + 1];
            for (int64_t l = m; l <= lmax; ++l) {
                acc[2 * l] += lam[l] * gr;
                acc[2 * l + 1] += lam[l] * gi;
            }
        }
        free(lam);
    }
    free(mapc); free(F); 
}

/* ------------------------------------------------------------------------- */
/* Pseudo-C_ell (workspaces.py:86-95)                                         */
/* cls[(i*n2 + j)*L + l] = sum_m (2 - delta_m0) Re(a_i,lm conj(b_j,lm)) / (2l+1) */
/* ------------------------------------------------------------------------- */

void orc_pcl(int64_t lmax, int64_t n1, const double *a, int64_t n2, const double *b,
             double *cls)
{
    int64_t L = lmax + 1, nelem = L * (L + 1) / 2;
    for (int64_t i = 0; i < n1; ++i)
        for (int64_t j = 0; j < n2; ++j)
            for (int64_t l = 0; l <= lmax; ++l) {
                double s = 0.0;
                for (int64_t m = 0; m <= l; ++m) {
                    int64_t k = alm_index(lmax, l, m);
                    double re = a[2 * (i * nelem + k)] * b[2 * (j * nelem + k)] +
                                a[2 * (i * nelem + k) + 1] * b[2 * (j * nelem + k) + 1];
                    s += (m == 0 ? 1.0 : 2.0) * re;
                }
                cls[(i * n2 + j) * L + l] = s / (2.0 * l + 1.0);
            }
}

/* ------------------------------------------------------------------------- */
/* Coupling matrices                                                          */
/* ------------------------------------------------------------------------- */

/* Scalar MCM from the threej closed form, offset by offset
 * (tests/test_workspaces.py:122-144; workspaces.py:440-517).
 * window has 2*lmax+1 entries; M is (lmax+1)^2 row-major, M[l1][l2]. */
void orc_coupling_tt_closed(int64_t lmax, const double *window, double *M)
{
    int64_t n = lmax + 1;
    double *g = malloc(sizeof(double) * (2 * lmax + 1));
    double *mp = malloc(sizeof(double) * (2 * lmax + 1));
    double lg = 0.0;
    g[0] = 1.0;
    for (int64_t p = 1; p <= 2 * lmax; ++p) {
        lg += log((p - 0.5) / (double)p);
        g[p] = exp(lg);
    }
    for (int64_t l = 0; l <= 2 * lmax; ++l) mp[l] = window[l] * (2.0 * l + 1.0) / (4.0 * M_PI);
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < n; ++r)
        for (int64_t c = 0; c < n; ++c) {
            int64_t lo = r < c ? r : c, hi = r < c ? c : r;
            double s = 0.0;
            for (int64_t o = 0; o <= lo; ++o) {
                int64_t pt = hi + o;
                int64_t li = hi - lo + 2 * o;
                if (li > 2 * lmax) li = 2 * lmax;
                s += mp[li] * g[hi - lo + o] * g[o] * g[lo - o] / (g[pt] * (2.0 * pt + 1.0));
            }
            M[r * n + c] = s * (2.0 * c + 1.0);
        }
    free(g); free(mp);
}

/* Gauss-Legendre nodes (ascending) and weights on [-1, 1] by Newton on P_n. */
void orc_gauss_legendre(int64_t n, double *x, double *w)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (n + 1) / 2; ++i) {
        /* i-th root from the top: initial guess (Tricomi) */
        double z = cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int64_t k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / (double)k;
                p0 = p1; p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1.0; }
            pp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / pp;
            z -= dz;
            if (fabs(dz) < 1e-16 * (1.0 + fabs(z)) && it > 2) break;
        }
        {
            double p0 = 1.0, p1 = z;
            for (int64_t k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / (double)k;
                p0 = p1; p1 = p2;
            }
            if (n == 1) { p1 = z; p0 = 1.0; }
            pp = n * (z * p1 - p0) / (z * z - 1.0);
        }
        double wt = 2.0 / ((1.0 - z * z) * pp * pp);
        x[n - 1 - i] = z; w[n - 1 - i] = wt;
        x[i] = -z; w[i] = wt;
    }
    if (n & 1) x[n / 2] = 0.0;
}

/* Wigner d^l_{m,n}(beta) table for l in [0, lmax] on `nb` nodes, row-major
 * [node][l]; Jacobi recurrence with gammaln normalisation (workspaces.py:608-679). */
static void wigner_d_table(int64_t nb, const double *beta, int64_t m, int64_t n,
                           int64_t lmax, double *out)
{
    int64_t minimum = labs(m) > labs(n) ? labs(m) : labs(n);
    memset(out, 0, sizeof(double) * nb * (lmax + 1));
    if (minimum > lmax) return;
    int64_t mu = labs(m - n), nu = labs(m + n);
    double sgn = (((n - m + mu) / 2) & 1) ? -1.0 : 1.0;
    for (int64_t i = 0; i < nb; ++i) {
        double cb = cos(beta[i]);
        double pref = sgn * pow(sin(beta[i] / 2), (double)mu) * pow(cos(beta[i] / 2), (double)nu);
        double prev = 1.0, cur = ((mu - nu) + (mu + nu + 2) * cb) / 2;
        for (int64_t deg = 0; deg <= lmax - minimum; ++deg) {
            double val;
            if (deg == 0) val = 1.0;
            else if (deg == 1) val = cur;
            else {
                double o = (double)deg, t = (double)(mu + nu);
                double nxt = ((2 * o + t - 1) * ((2 * o + t) * (2 * o + t - 2) * cb + mu * mu - nu * nu) * cur -
                              2 * (o + mu - 1) * (o + nu - 1) * (2 * o + t) * prev) /
                             (2 * o * (o + t) * (2 * o + t - 2));
                prev = cur; cur = nxt; val = nxt;
            }
            double norm = exp(0.5 * (lgamma(deg + 1.0) + lgamma(deg + mu + nu + 1.0) -
                                     lgamma(deg + mu + 1.0) - lgamma(deg + nu + 1.0)));
            out[i * (lmax + 1) + minimum + deg] = val * norm * pref;
        }
    }
}

/* Even/odd general coupling matrices by Gauss-Legendre quadrature
 * (workspaces.py:682-732, 878-905):
 *   M[l1,l2] = (2 l2 + 1)/2 sum_i w_i d^l1_{n1 n2}(x_i) xi(x_i) d^l2_{-s1,-s2}(x_i),
 *   xi(x) = sum_L (2L+1)/(4pi) C_L d^L_{s1-n1, s2-n2}(x), split by (-1)^(l1+l2+L).
 * window has lmax_mask+1 entries.  even/odd are (lmax+1)^2 row-major. */
void orc_coupling_quadrature(int64_t lmax, int64_t lmax_mask, const double *window,
                             int64_t s1, int64_t s2, int64_t n1, int64_t n2,
                             double *even, double *odd)
{
    int64_t order = (2 * lmax + lmax_mask) / 2 + 1;
    double *x = malloc(sizeof(double) * order), *w = malloc(sizeof(double) * order);
    double *beta = malloc(sizeof(double) * order);
    orc_gauss_legendre(order, x, w);
    for (int64_t i = 0; i < order; ++i) beta[i] = acos(x[i]);
    int64_t n = lmax + 1, nm = lmax_mask + 1;
    double *first = malloc(sizeof(double) * order * n);
    double *second = malloc(sizeof(double) * order * n);
    double *mask = malloc(sizeof(double) * order * nm);
    wigner_d_table(order, beta, n1, n2, lmax, first);
    wigner_d_table(order, beta, -s1, -s2, lmax, second);
    wigner_d_table(order, beta, s1 - n1, s2 - n2, lmax_mask, mask);
    double *tot = malloc(sizeof(double) * order), *sig = malloc(sizeof(double) * order);
    for (int64_t i = 0; i < order; ++i) {
        double a = 0.0, b = 0.0;
        for (int64_t L = 0; L < nm; ++L) {
            double c = (2.0 * L + 1.0) * window[L] / (4.0 * M_PI) * mask[i * nm + L];
            a += c;
            b += (L & 1) ? -c : c;
        }
        tot[i] = a * w[i];
        sig[i] = b * w[i];
    }
#pragma omp parallel for schedule(dynamic)
    for (int64_t l1 = 0; l1 < n; ++l1)
        for (int64_t l2 = 0; l2 < n; ++l2) {
            double a = 0.0, b = 0.0;
            for (int64_t i = 0; i < order; ++i) {
                double pr = first[i * n + l1] * second[i * n + l2];
                a += pr * tot[i];
                b += pr * sig[i];
            }
            double f = (2.0 * l2 + 1.0) / 2.0;
            double sgn = ((l1 + l2) & 1) ? -1.0 : 1.0;
            a *= f;
            b *= f * sgn;
            even[l1 * n + l2] = (a + b) / 2;
            odd[l1 * n + l2] = (a - b) / 2;
        }
    free(x); free(w); free(beta); free(first); free(second); free(mask); free(tot); free(sig);
}

/* Spin-2 analysis (no refinement) restricted to a set of orders, for the bounded
 * CPU-baseline sample: eb_out[im][2][l] complex (E then B rows). */
void orc_ana2_orders(int64_t nside, int64_t lmax, const double *theta, const double *phi0,
                     const double *qu, int64_t nm, const int64_t *ms, double *eb_out)
{
    int64_t nring = 4 * nside - 1, L = lmax + 1, npix = 12 * nside * nside;
    double w = 4.0 * M_PI / (double)npix;
    double *mapc = malloc(sizeof(double) * 2 * npix);
    for (int64_t p = 0; p < npix; ++p) { mapc[2 * p] = qu[p]; mapc[2 * p + 1] = qu[npix + p]; }
    int64_t width = 2 * L - 1;
    double *F = malloc(sizeof(double) * 2 * nring * width);
    orc_ring_analysis(nside, L, L - 1, phi0, mapc, F);
#pragma omp parallel for schedule(dynamic)
    for (int64_t im = 0; im < nm; ++im) {
        int64_t m = ms[im];
        double *lp = malloc(sizeof(double) * L), *lmn = malloc(sizeof(double) * L);
        double *ap = calloc(2 * L, sizeof(double)), *am = calloc(2 * L, sizeof(double));
        for (int64_t r = 0; r < nring; ++r) {
            orc_lambda_row(lmax, m, -2, theta[r], lp);
            orc_lambda_row(lmax, m, 2, theta[r], lmn);
            double pr = w * F[2 * (r * width + (L - 1) + m)], pi = w * F[2 * (r * width + (L - 1) + m) + 1];
            double mr = w * F[2 * (r * width + (L - 1) - m)], mi = -w * F[2 * (r * width + (L - 1) - m) + 1];
            for (int64_t l = m; l <= lmax; ++l) {
                ap[2 * l] += lp[l] * pr; ap[2 * l + 1] += lp[l] * pi;
                am[2 * l] += lmn[l] * mr; am[2 * l + 1] += lmn[l] * mi;
            }
        }
        double *e = eb_out + 4 * im * L, *b = e + 2 * L;
        for (int64_t l = 0; l <= lmax; ++l) {
            e[2 * l] = -(ap[2 * l] + am[2 * l]) / 2;
            e[2 * l + 1] = -(ap[2 * l + 1] + am[2 * l + 1]) / 2;
            b[2 * l] = -(ap[2 * l + 1] - am[2 * l + 1]) / 2;
            b[2 * l + 1] = (ap[2 * l] - am[2 * l]) / 2;
        }
        free(lp); free(lmn); free(ap); free(am);
    }
    free(mapc); free(F);
}
