// Mask apodisation on the GPU: exact distance from every pixel to the nearest masked pixel,
// then the C1 / C2 tapers or the zeroing step of the "Smooth" type (gmaster/utils.py:61-147,
// where a k-d tree over the masked pixels' unit vectors and healpy's query_disc do this on
// the host).
//
// The search walks HEALPix rings.  Within one ring the chord from a query q to a ring pixel
// grows with |phi - phi_q| (in [0, pi]), so the nearest masked pixel of that ring is the
// first masked pixel met going down from the pixel just below phi_q, or the first met going
// up from the pixel just above it.  k_ring_runs stores both for every pixel (cyclically
// within its ring): prev[p] = the masked pixel at or before p, next[p] = at or after p
// (ring-local indices, -1 for a ring without masked pixels).  k_mask_apodize then visits
// rings outwards from the query's own ring, alternating north and south, two candidates
// per ring, and stops in each direction once the ring's latitude alone puts it beyond the
// best chord found (or the apodisation radius).  The result is the exact minimum over all
// masked pixels, like the k-d tree's.
//
// Chords are evaluated as |v_q - v_c|^2 = dz^2 + ds^2 + 4 s_q s_c sin^2(dphi / 2) with
// z = cos(theta), s = sin(theta): the same Euclidean distance between unit vectors, free of
// the cancellation of 2 - 2 v_q.v_c at small separations.

#include <climits>

#include "gm_common.cuh"

namespace gm {
namespace {

constexpr int kRunThreads = 1024;
constexpr int kApoThreads = 256;
constexpr double kTwoPi = 6.283185307179586;   // 2 pi rounded to double, as numpy's 2*np.pi
constexpr double kInvTwoPi = 0.15915494309189535;

// One CTA per ring (grid-stride over rings).  Thread t scans a contiguous chunk of the ring;
// two block-wide scans give the last masked pixel before each chunk and the first after.
__global__ void __launch_bounds__(kRunThreads) k_ring_runs(int64_t nside,
                                                           const double *__restrict__ mask,
                                                           int32_t *__restrict__ prev,
                                                           int32_t *__restrict__ next)
{
    __shared__ int sp[kRunThreads], sn[kRunThreads];
    const int t = threadIdx.x;
    const int64_t nring = 4 * nside - 1;
    for (int64_t r = blockIdx.x; r < nring; r += gridDim.x) {
        const int n = (int)ring_nphi(nside, r);
        const int64_t off = ring_offset(nside, r);
        const int chunk = (n + kRunThreads - 1) / kRunThreads;
        const int b = min(n, t * chunk), e = min(n, b + chunk);
        int last = -1, first = INT_MAX;
        for (int i = b; i < e; ++i) {
            if (mask[off + i] <= 0.0) {
                if (first == INT_MAX) first = i;
                last = i;
            }
        }
        sp[t] = last;
        sn[t] = first;
        __syncthreads();
        // inclusive prefix max of sp (left to right) and suffix min of sn (right to left)
        for (int d = 1; d < kRunThreads; d <<= 1) {
            const int a = t >= d ? sp[t - d] : -1;
            const int c = t + d < kRunThreads ? sn[t + d] : INT_MAX;
            __syncthreads();
            sp[t] = max(sp[t], a);
            sn[t] = min(sn[t], c);
            __syncthreads();
        }
        const int ring_last = sp[kRunThreads - 1], ring_first = sn[0];
        int carry_p = t > 0 ? sp[t - 1] : -1;
        int carry_n = t + 1 < kRunThreads ? sn[t + 1] : INT_MAX;
        __syncthreads();   // every thread has read sp / sn before the next ring rewrites them
        if (ring_last < 0) {
            for (int i = b; i < e; ++i) {
                prev[off + i] = -1;
                next[off + i] = -1;
            }
            continue;
        }
        if (carry_p < 0) carry_p = ring_last;        // wrap: the ring's last masked pixel
        if (carry_n == INT_MAX) carry_n = ring_first;  // wrap: the ring's first masked pixel
        int run = carry_p;
        for (int i = b; i < e; ++i) {
            if (mask[off + i] <= 0.0) run = i;
            prev[off + i] = run;
        }
        run = carry_n;
        for (int i = e - 1; i >= b; --i) {
            if (mask[off + i] <= 0.0) run = i;
            next[off + i] = run;
        }
    }
}

// Ring table rows (each nring doubles): cos theta, sin theta, phi0, 2 pi / nphi, nphi / (2 pi).
struct Rings {
    const double *z, *s, *phi0, *step, *inv;
};

struct Query {
    double z, s, phi;
    double best;   // smallest chord^2 found so far (starts at the search radius, exclusive)
    bool found;
};

// Visit ring jj for query q: false once the ring's latitude alone is out of reach.
__device__ __forceinline__ bool probe(int64_t nside, int64_t jj, const Rings &rg,
                                      const int32_t *__restrict__ prev,
                                      const int32_t *__restrict__ next, Query &q)
{
    const double zc = rg.z[jj], sc = rg.s[jj];
    const double dz = q.z - zc, ds = q.s - sc;
    const double lb = dz * dz + ds * ds;   // chord^2 to the ring point at the same phi
    if (lb >= q.best) return false;
    const int64_t nn = ring_nphi(nside, jj);
    const int64_t off = ring_offset(nside, jj);
    const double phi0 = rg.phi0[jj], step = rg.step[jj];
    const double tpos = (q.phi - phi0) * rg.inv[jj];
    // phi_q < 2 pi + pi/4 and phi0 >= 0, so floor(tpos) lies in [-1, 9 nn / 8]
    int k = (int)floor(tpos);
    if (k < 0) k += (int)nn;
    if (k >= (int)nn) k -= (int)nn;
    k = min(max(k, 0), (int)nn - 1);
    const int32_t a = prev[off + k];
    if (a < 0) return true;   // no masked pixel on this ring
    const int32_t b = next[off + (k + 1 == nn ? 0 : k + 1)];
    const double w = 4.0 * q.s * sc;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const int32_t c = u == 0 ? a : b;
        double dphi = fma((double)c, step, phi0 - q.phi);
        dphi -= kTwoPi * rint(dphi * kInvTwoPi);   // into [-pi, pi]
        // sin(|x|/2) >= |x|/pi on [0, pi]: skip the sine when even that bound loses
        const double rough = lb + w * (dphi * dphi) * (1.0 / (M_PI * M_PI));
        if (rough >= q.best) continue;
        const double h = sin(0.5 * dphi);
        const double d2 = lb + w * h * h;
        if (d2 < q.best) {
            q.best = d2;
            q.found = true;
        }
    }
    return true;
}

// mode 0: C1 taper, 1: C2 taper (out = mask * f(x) for unmasked pixels closer than the
// radius, x = sqrt(0.5 d^2 / threshold)); mode 2: zeroing step (out = 0 for masked pixels
// and for pixels closer than the radius to a masked one, else the mask value).
__global__ void __launch_bounds__(kApoThreads) k_mask_apodize(
    int64_t nside, Rings rg, const double *__restrict__ mask,
    const int32_t *__restrict__ prev, const int32_t *__restrict__ next, double chord2_max,
    double threshold, int mode, double *__restrict__ out)
{
    const int64_t nring = 4 * nside - 1;
    const int64_t j = blockIdx.y;
    const int64_t n = ring_nphi(nside, j);
    const int64_t i = (int64_t)blockIdx.x * kApoThreads + threadIdx.x;
    if (i >= n) return;
    const int64_t p = ring_offset(nside, j) + i;
    const double m = mask[p];
    if (mode == 2 ? (m <= 0.0) : !(m > 0.0)) {
        out[p] = mode == 2 ? 0.0 : m;
        return;
    }
    Query q;
    q.z = rg.z[j];
    q.s = rg.s[j];
    q.phi = fma((double)i, rg.step[j], rg.phi0[j]);
    q.best = chord2_max;
    q.found = false;
    bool up = true, dn = true;
    for (int64_t d = 0; up || dn; ++d) {
        if (up) up = j + d < nring && probe(nside, j + d, rg, prev, next, q);
        if (dn) dn = j - 1 - d >= 0 && probe(nside, j - 1 - d, rg, prev, next, q);
    }
    if (!q.found) {
        out[p] = m;
        return;
    }
    if (mode == 2) {
        out[p] = 0.0;
        return;
    }
    const double x = sqrt(fmax(0.5 * q.best, 0.0) / threshold);
    const double f = mode == 0 ? x - sin(kTwoPi * x) / kTwoPi : 0.5 * (1.0 - cos(M_PI * x));
    out[p] = m * f;
}

}  // namespace
}  // namespace gm

using namespace gm;

extern "C" int gm_mask_ring_runs(int64_t nside, const double *mask, int32_t *prev, int32_t *next,
                                 void *stream)
{
    if (nside < 1 || nside > 16384) return GM_ERR_BAD_SHAPE;
    if (!mask || !prev || !next) return GM_ERR_BAD_PTR;
    const int64_t nring = 4 * nside - 1;
    const int grid = (int)(nring < 296 ? nring : 296);
    k_ring_runs<<<grid, kRunThreads, 0, as_stream(stream)>>>(nside, mask, prev, next);
    return check_launch("gm_mask_ring_runs");
}

extern "C" int gm_mask_apodize(int64_t nside, const double *ring_table, const double *mask,
                               const int32_t *prev, const int32_t *next, double chord2_max,
                               double threshold, int mode, double *out, void *stream)
{
    if (nside < 1 || nside > 16384) return GM_ERR_BAD_SHAPE;
    if (!ring_table || !mask || !prev || !next || !out) return GM_ERR_BAD_PTR;
    if (mode < 0 || mode > 2) return GM_ERR_UNSUPPORTED;
    if (!(chord2_max > 0.0) || (mode != 2 && !(threshold > 0.0))) return GM_ERR_BAD_SHAPE;
    const int64_t nring = 4 * nside - 1;
    const dim3 grid((unsigned)((4 * nside + kApoThreads - 1) / kApoThreads), (unsigned)nring);
    const Rings rg{ring_table, ring_table + nring, ring_table + 2 * nring, ring_table + 3 * nring,
                   ring_table + 4 * nring};
    k_mask_apodize<<<grid, kApoThreads, 0, as_stream(stream)>>>(nside, rg, mask, prev, next,
                                                                 chord2_max, threshold, mode, out);
    return check_launch("gm_mask_apodize");
}
