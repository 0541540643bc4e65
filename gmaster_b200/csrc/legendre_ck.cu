// Checkpointed Legendre / Wigner-d contraction on the tcgen05 tensor cores (sm_100a).
//
// The rows lambda^{s'}_lm(theta) are generated in single precision by the three-term
// recurrence in its difference form
//     C_l = c1_l (x - 1) + E_l,   D_l = b_l D_{l-1} + C_l v_{l-1},   v_l = v_{l-1} + D_l
// (c1 = alpha, b = beta, E = alpha - beta - 1 - alpha s'c0/|s'|; algebraically the same as
// v_l = alpha (x - c) v_{l-1} - beta v_{l-2}), restarted every kSeg = 128 rows from a
// state computed once per geometry by the FP64 recurrence (the checkpoint table).  The
// difference form keeps each rounding unamplified near the poles and turning points, where
// the plain form multiplies it by 1/sin(phi) (phi the local oscillation phase); over 128 rows
// from an exact start the FP32 rows stay within ~2e-6 of the row scale sqrt((2l+1)/4pi).
// FP64 is kept for the checkpoint states, the seeds and the alm accumulation.
//
// Because every 128-row segment starts from the table, segments are independent:
//   * the analysis generates each 256-row superblock with one warp per 128-row segment and
//     32-lane group, four such warp pairs taking the groups in turn, and its work units
//     (order m, superblock) are independent, so the CTAs that run the superblocks of one
//     order at the same time share that order's right-hand-side images through L2 and each
//     alm element receives exactly one addition per launch, from one unit;
//   * the synthesis runs two sets of 8 generator warps on alternate segments.
// A checkpoint stores the pre-state (v_{l_s - 1}, D_{l_s}) of the segment's first row l_s,
// so that row is the uniform step with coefficients (c1, E, b) = (0, 0, 1).  The state is
// kept in FP32 with a shift n in {0..5}: actual = stored * 2^(-64 n).  Lanes whose rows are
// still far below 2^-16 (the seed region of high orders, where a segment can grow by 2^230)
// carry n > 0, emit v * 2^(-64 n) and renormalise every 8 rows; a warp in which every lane
// has n = 0 takes the plain path.  Segments whose state is below 2^-336 are stored as
// zeros: they cannot reach 2^-40 within 128 rows.
//
// Operands and accumulation as legendre_tc.cu: f16 hi/lo operands, three products
// (hi*hi + hi*lo + lo*hi) into separate hi*hi and cross-product TMEM accumulators, FP64
// alm accumulation in the epilogue.
//
// Replaces gmaster/_native/cuda/march_v2.cu:155-407 (FP32 SIMT march with a two-word
// difference form over all rows) for batched maps.
#include <math.h>

#include "gm_common.cuh"
#include "ltc_common.cuh"
#include "tc_common.cuh"

namespace gm {
namespace lck {

using ltc::alm_idx;
using ltc::Coef;
using ltc::load_coef;
using ltc::pack8;
using ltc::sgn_of;
using ltc::sts128;
using ltc::wait_or_abort;

constexpr int kSeg = 128;                           // rows per checkpoint segment
constexpr int kMaxShift = 5;                        // largest stored shift n (2^-320)
// analysis
constexpr int kSB = 2 * kSeg;                       // superblock rows (one unit; MMA N)
constexpr int kHalf = 64;                           // rows per generation step
constexpr int kKC = 128;                            // lanes per operand image (global layout)
constexpr int kKG = 32;                             // lanes per analysis group (MMA K per group)
constexpr int kSetsA = 4;                           // generator sets (2 warps each, one tile each)
constexpr int kImgBufA = 4;                         // image buffers
constexpr int kMaxGroupsA = 128;                    // lane groups of a unit (two 64-bit words)
constexpr int kGenA = 256;                          // generator threads (8 warps)
constexpr int kMmaWarpA = kGenA / 32;
constexpr int kLoadWarpA = kMmaWarpA + 1;
constexpr int kThrA = kGenA + 64;                   // + the MMA warp and the image loader warp
constexpr uint32_t kAImg = 128u * kKC * 2u;         // one plane of a right-hand-side image (32 KB)
constexpr uint32_t kAImgG = 2u * 128u * kKG * 2u;   // a group's hi and lo image planes (16 KB)
constexpr uint32_t kTileA = 2u * kSB * kKG * 2u;    // tile: 256 rows x 32 lanes, hi + lo (32 KB)
constexpr int kStageLd = kSB + 1;                   // epilogue staging row stride (floats)
// the epilogue stages 128 rows x kStageLd floats in the tiles and coefficient rows
static_assert(128 * kStageLd * 4 <= kSetsA * kTileA + kSB * 16, "epilogue staging does not fit");
// synthesis
constexpr int kLT = 256;                            // lanes per CTA (MMA N)
constexpr int kKL = 64;                             // rows per chunk (MMA K)
constexpr int kGenS = 2 * kLT;                      // generator threads (16 warps, 2 sets)
constexpr int kThrS = kGenS + 32;
constexpr int kMmaWarpS = kGenS / 32;
constexpr uint32_t kSImg = 128u * kKL * 2u;         // one plane of an alm image (16 KB)
constexpr uint32_t kBTileS = kLT * kKL * 2u;        // one plane of a generated tile (32 KB)

struct CkParams {
    int64_t nside, lmax, nlanes;
    int sp;            // s' of the rows: 0, -2 or +2
    int H;             // rows per half (maps x re/im); valid rows 2H <= 128
    int NR;            // rows of the interleaved alm
    int o0, o1;        // output row base of the first / second half (analysis)
    double scale;      // analysis: alm += scale * result; synthesis: output scale
    const double *geom;      // (3, nlanes): cos(theta), log2 sin(theta/2), log2 cos(theta/2)
    const double *coef;      // (nelem, 4): alpha, beta, c0, 0
    const int64_t *segoff;   // (L + 1): first checkpoint segment of each order
    const int64_t *uoff;     // (L + 1): first analysis unit of each order
    const float2 *ck;        // (segments, nlanes): pre-state (v_{l_s - 1}, D_{l_s}), scaled
    const uint8_t *cn;       // (segments, nlanes): shift n
    // optional (NULL: every lane group active): bit g set when a lane of the 64-lane group g
    // has a non-zero stored state, per segment (synthesis) or per analysis unit (the union of
    // its two segments).  A segment that starts from a zero state stays exactly zero.
    const unsigned long long *seg_mask;   // (segments)
    const unsigned long long *unit_mask;  // (analysis units)
};

__device__ __forceinline__ unsigned long long all_groups(int64_t ngroups)
{
    return ngroups >= 64 ? ~0ull : ((1ull << ngroups) - 1ull);
}

// Pops the lowest set bit of r and returns its index, or -1 when r is empty.
__device__ __forceinline__ int pop_group(unsigned long long &r)
{
    if (!r) return -1;
    const int g = __ffsll((long long)r) - 1;
    r &= r - 1ull;
    return g;
}

// A set of up to 128 lane groups (bit g of word g / 64).
struct GroupSet {
    unsigned long long w0, w1;
};

__device__ __forceinline__ int pop_group(GroupSet &r)
{
    const int g = pop_group(r.w0);
    if (g >= 0) return g;
    const int h = pop_group(r.w1);
    return h >= 0 ? 64 + h : -1;
}

// Bit i of the low 32 bits of x to bits 2i and 2i + 1.
__device__ __forceinline__ unsigned long long spread_pairs(unsigned long long x)
{
    x &= 0xffffffffull;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x | (x << 1);
}

// Active 32-lane groups of analysis unit u: both halves of every 64-lane group whose mask
// bit is set (all `ngroups` groups without masks).
__device__ __forceinline__ GroupSet unit_groups(const unsigned long long *__restrict__ unit_mask, int64_t u,
                                                int64_t ngroups)
{
    GroupSet r;
    r.w0 = all_groups(ngroups);
    r.w1 = ngroups > 64 ? all_groups(ngroups - 64) : 0ull;
    if (unit_mask) {
        const unsigned long long mk = __ldg(unit_mask + u);
        r.w0 &= spread_pairs(mk);
        r.w1 &= spread_pairs(mk >> 32);
    }
    return r;
}

__host__ __device__ __forceinline__ int64_t first_row(int64_t m, int sp)
{
    const int64_t a = sp < 0 ? -sp : sp;
    return m > a ? m : a;
}

// Difference-form coefficients of the step to row l of order m (coefficient base mb).
__device__ __forceinline__ float4 diff_coef(const double *__restrict__ coef, int64_t mb, int64_t l,
                                            int64_t L, double sgn_c, bool restart)
{
    if (restart) return make_float4(0.f, 0.f, 1.f, 0.f);   // D = D, v = v + D
    if (l >= L) return make_float4(0.f, -1.f, 0.f, 0.f);   // v = 0 from here on
    const Coef c = load_coef(coef, mb + l);
    return make_float4((float)c.alpha, (float)(c.alpha - c.beta - 1.0 - sgn_c * c.alpha * c.c0),
                       (float)c.beta, 0.f);
}

// A warp-uniform bounded wait: every lane waits, and the warp goes on only if all did.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, volatile int *abort, int *err)
{
    const bool ok = wait_or_abort(bar, parity, abort, err);
    return __all_sync(0xffffffffu, ok);
}

// One step of the FP32 difference form with coefficients q = (c1, E, b):
//   C = c1 (x - 1) + E,  D <- C v + b D,  v <- v + D.
// b D is formed off the dependent chain, so a row costs two dependent operations.
__device__ __forceinline__ void diff_step(const float4 &q, float y, float &v, float &D)
{
    const float C = fmaf(q.x, y, q.y);
    const float bD = q.z * D;
    D = fmaf(C, v, bD);
    v = v + D;
}

// Sixty-four rows of one lane (eight chunks of eight), split into f16 hi/lo and stored as
// 16-byte chunks: chunk cc at base + ((cc ^ sw) << 4), its lo plane lo_delta bytes further.
// SCALED: some lane of the warp still carries a shift n > 0 (decided once per 64 rows; a
// lane's shift only decreases): such lanes emit v * 2^(-64 n) and renormalise every 8 rows.
template <bool SCALED>
__device__ __forceinline__ void gen64(const float4 *__restrict__ cw, float y, float &v, float &D, int &n,
                                      uint32_t base, uint32_t lo_delta, uint32_t sw)
{
#pragma unroll 2
    for (int cc = 0; cc < 8; ++cc) {
        float vals[8];
        if (SCALED) {
            const float sc = n == 0 ? 1.0f : (n == 1 ? 0x1p-64f : 0.0f);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                diff_step(cw[8 * cc + e], y, v, D);
                vals[e] = v * sc;
            }
            // 8 rows grow a value by at most 2^63 (alpha <= sqrt(2m) + 1 at Nside <= 8192),
            // so a renormalisation at 2^48 keeps every shifted value below 2^111
            if (n != 0 && fabsf(v) > 0x1p48f) {
                v *= 0x1p-64f;
                D *= 0x1p-64f;
                --n;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                diff_step(cw[8 * cc + e], y, v, D);
                vals[e] = v;
            }
        }
        uint4 hi, lo;
        pack8(vals, hi, lo);
        const uint32_t off = ((uint32_t)cc ^ sw) << 4;
        sts128(base + off, hi);
        sts128(base + lo_delta + off, lo);
    }
}

__device__ __forceinline__ void gen_rows64(const float4 *__restrict__ cw, float y, float &v, float &D,
                                           int &n, uint32_t base, uint32_t lo_delta, uint32_t sw)
{
    if (__any_sync(0xffffffffu, n != 0)) gen64<true>(cw, y, v, D, n, base, lo_delta, sw);
    else gen64<false>(cw, y, v, D, n, base, lo_delta, sw);
}

// ----------------------------------------------------------------------- checkpoint table

// Stored checkpoint of an FP64 state: (vpre, d) * 2^(600 k) actual.
__device__ __forceinline__ void ck_put(float2 *__restrict__ ck, uint8_t *__restrict__ cn, int64_t idx,
                                       double vpre, double d, int k)
{
    const double mx = fmax(fabs(vpre), fabs(d));
    float2 out = make_float2(0.f, 0.f);
    int n = 0;
    if (mx > 0.0) {
        const int e = ilogb(mx) + 600 * k;   // floor(log2) of the actual largest entry
        const int sh = e < -16 ? (-16 - e + 63) / 64 : 0;
        if (sh <= kMaxShift) {
            const int p = 600 * k + 64 * sh;
            out = make_float2((float)ldexp(vpre, p), (float)ldexp(d, p));
            n = sh;
        }
    }
    ck[idx] = out;
    cn[idx] = (uint8_t)n;
}

// One thread per (order m, lane): the FP64 recurrence with binary-exponent carry (the
// recurrence of legendre_tc.cu), writing the pre-state of every segment's first row.
__global__ void __launch_bounds__(128) k_ck_build(int64_t nside, int64_t lmax, int sp, int var,
                                                  const double *__restrict__ geom,
                                                  const double *__restrict__ seeds,
                                                  const double *__restrict__ coef,
                                                  const int64_t *__restrict__ segoff,
                                                  float2 *__restrict__ ck, uint8_t *__restrict__ cn)
{
    const int64_t nlanes = 2 * nside, L = lmax + 1;
    const int64_t m = blockIdx.y;
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t l0 = first_row(m, sp);
    if (l0 > lmax || j >= nlanes) return;
    const double sgn_c = sgn_of(sp);
    const int64_t mb = alm_idx(lmax, 0, m);
    const double x = geom[j];
    double v, vp = 0.0;
    int k;
    ltc::seed_lane(seeds + ((int64_t)var * L + m) * 4, geom[nlanes + j], geom[2 * nlanes + j], v, k);
    int64_t row = segoff[m] * nlanes + j;
    ck_put(ck, cn, row, 0.0, v, k);   // the seed row: v_{l0 - 1} = 0
    for (int64_t l = l0 + 1; l < L; ++l) {
        const Coef c = load_coef(coef, mb + l);
        const double a = c.alpha * (x - sgn_c * c.c0);
        const double nv = fma(a, v, -c.beta * vp);
        vp = v;
        v = nv;
        if (((l - l0) & (kSeg - 1)) == 0) {
            row += nlanes;
            ck_put(ck, cn, row, vp, v - vp, k);
        }
        if (((l - l0) & 7) == 0) ltc::rescale(v, vp, k);
    }
}

// Non-zero 64-lane groups of every checkpoint segment (nlanes <= 4096): bit g of
// seg_mask[seg] is set when a lane of group g has a non-zero stored state or shift.
__global__ void __launch_bounds__(256) k_ck_seg_mask(int64_t nlanes, int64_t nseg, const float2 *__restrict__ ck,
                                                     const uint8_t *__restrict__ cn,
                                                     unsigned long long *__restrict__ seg_mask)
{
    __shared__ unsigned long long acc;
    for (int64_t seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
        if (threadIdx.x == 0) acc = 0ull;
        __syncthreads();
        unsigned long long bits = 0ull;
        for (int64_t j = threadIdx.x; j < nlanes; j += blockDim.x) {
            const float2 st = __ldg(ck + seg * nlanes + j);
            const uint8_t n = __ldg(cn + seg * nlanes + j);
            if (st.x != 0.f || st.y != 0.f || n != 0) bits |= 1ull << (j >> 6);
        }
        for (int o = 16; o >= 1; o >>= 1) bits |= __shfl_xor_sync(0xffffffffu, bits, o);
        if ((threadIdx.x & 31) == 0 && bits) atomicOr(&acc, bits);
        __syncthreads();
        if (threadIdx.x == 0) seg_mask[seg] = acc;
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------- analysis

struct __align__(8) AnaShared {
    uint64_t a_full[kImgBufA], a_free[kImgBufA], b_full[kSetsA], b_free[kSetsA], d_full, d_free, drain;
    uint32_t tmem;
    int abort;
};

// Order of analysis unit u: the last m with uoff[m] <= u.
__device__ __forceinline__ int64_t unit_order(const int64_t *__restrict__ uoff, int64_t L, int64_t u)
{
    int64_t lo = 0, hi = L;   // uoff[lo] <= u < uoff[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(uoff + mid) <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Analysis unit masks: unit u = (order m, superblock s) takes the union of the masks of
// its segments 2 s and 2 s + 1 (when the order has it).
__global__ void k_ck_unit_mask(int64_t L, const int64_t *__restrict__ segoff, const int64_t *__restrict__ uoff,
                               const unsigned long long *__restrict__ seg_mask,
                               unsigned long long *__restrict__ unit_mask)
{
    const int64_t U = uoff[L];
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = unit_order(uoff, L, u);
        const int64_t s0 = segoff[m] + 2 * (u - uoff[m]);
        unsigned long long mk = seg_mask[s0];
        if (s0 + 1 < segoff[m + 1]) mk |= seg_mask[s0 + 1];
        unit_mask[u] = mk;
    }
}

__device__ __forceinline__ void gen_barrier_a() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Units (m, s): superblock s of order m covers rows l0 + 256 s + [0, 256).  CTA c takes
// units c, c + G, ...  Within a unit the lanes run in groups of 32 (a quarter of a 128-lane
// operand image); a group's image (hi and lo planes, 16 KB) goes into one of four buffers
// that a loader warp refills while the other groups' MMAs run.  Four sets of two warps
// take the active groups in turn (set S the ones at positions S, S + 4, ...), each into
// its own tile: all 256 rows of the superblock for the group's 32 lanes, each warp one
// segment (128 rows) of each lane, f16 hi and lo planes.  A set regenerates its tile once
// the MMAs of its previous group are done, so with four sets a set waits for a quarter of
// the MMA stream (two sets of 64-lane tiles in the same shared memory would wait for half).  Per K
// step the tile is consumed by three MMAs of N = 256 (hi image x hi rows into the hi*hi
// accumulator; hi image x lo rows and lo image x hi rows into the cross accumulator), so
// the image is read from shared memory once per 256 rows and product.
template <int SPIN>
__global__ void __launch_bounds__(kThrA, 1) k_ana_ck(CkParams p, const uint8_t *__restrict__ aimg,
                                                     double *__restrict__ alm_i, int *__restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ AnaShared sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (tc::smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t *smem = smem_raw + (base - tc::smem_u32(smem_raw));
    uint8_t *sA = smem;                                              // kImgBufA image buffers
    uint8_t *sB = smem + kImgBufA * kAImgG;                          // kSetsA tiles
    float4 *sCf = reinterpret_cast<float4 *>(sB + kSetsA * kTileA); // kSB coefficient rows
    const int64_t L = p.lmax + 1, NG = (p.nlanes + kKC - 1) / kKC, NGK = (p.nlanes + kKG - 1) / kKG;
    const int64_t U = p.uoff[L];
    const int64_t G = gridDim.x, c = blockIdx.x;

    if (tid == 0) {
        for (int i = 0; i < kImgBufA; ++i) {
            tc::mbar_init(&sh.a_full[i], 1);
            tc::mbar_init(&sh.a_free[i], 1);
        }
        for (int i = 0; i < kSetsA; ++i) {
            tc::mbar_init(&sh.b_full[i], kGenA / 32 / kSetsA);
            tc::mbar_init(&sh.b_free[i], 1);
        }
        tc::mbar_init(&sh.d_full, 1);
        tc::mbar_init(&sh.d_free, kGenA / 32);
        tc::mbar_init(&sh.drain, 1);
        sh.abort = 0;
        tc::fence_mbar_init();
    }
    if (warp == kMmaWarpA) {
        tc::tmem_alloc(&sh.tmem, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh.tmem;
    volatile int *abort = &sh.abort;

    if (warp == kMmaWarpA) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_f16(128, kSB, 0, 1, 1);
            uint32_t par = 0;              // bit S: parity of the groups consumed from tile S
            uint32_t q = 0;
            int64_t jg = 0;
            bool ok = true;
            for (int64_t u = c; u < U && ok; u += G, ++q) {
                // the previous unit's epilogue has read TMEM (waited for every unit, so the
                // phases stay in step); a unit without active groups only signals d_full
                if (!(ok = wait_or_abort(&sh.d_free, (q & 1) ^ 1, abort, err))) break;
                GroupSet rest = unit_groups(p.unit_mask, u, NGK);
                int k = 0;
                for (int g = pop_group(rest); g >= 0 && ok; g = pop_group(rest), ++jg, ++k) {
                    const uint32_t b = (uint32_t)(jg % kImgBufA);
                    const int S = k % kSetsA;
                    if (!(ok = wait_or_abort(&sh.a_full[b], (uint32_t)(jg / kImgBufA) & 1, abort, err))) break;
                    if (!(ok = wait_or_abort(&sh.b_full[S], (par >> S) & 1u, abort, err))) break;
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_u32(sA + b * kAImgG);
                    const uint32_t b0 = tc::smem_u32(sB + S * kTileA);
#pragma unroll
                    for (int ks = 0; ks < kKG / 16; ++ks) {
                        const uint64_t ah = tc::desc_sw128_mn(a0 + ks * 4096, 1024, 2048);
                        const uint64_t al = tc::desc_sw128_mn(a0 + kAImgG / 2 + ks * 4096, 1024, 2048);
                        const uint64_t bh = tc::desc_sw128_mn(b0 + ks * 8192, 1024, 4096);
                        const uint64_t bl = tc::desc_sw128_mn(b0 + kTileA / 2 + ks * 8192, 1024, 4096);
                        const uint32_t acc = (k > 0 || ks > 0) ? 1u : 0u;
                        tc::mma_f16(tmem, ah, bh, idesc, acc);
                        tc::mma_f16(tmem + kSB, ah, bl, idesc, acc);
                        tc::mma_f16(tmem + kSB, al, bh, idesc, 1u);
                    }
                    tc::mma_commit(&sh.b_free[S]);
                    tc::mma_commit(&sh.a_free[b]);
                    par ^= 1u << S;
                }
                if (!ok) break;
                tc::mma_commit(&sh.d_full);
            }
            // every issued MMA completes before TMEM is released (bounded wait)
            tc::mma_commit(&sh.drain);
            tc::mbar_wait(&sh.drain, 0);
        }
    } else if (warp == kLoadWarpA) {
        // ------------------------------------------------ image loader
        // group g of order m: lanes 32 g + [0, 32) are quarter g % 4 of the 128-lane image
        // g / 4, i.e. 8 KB of its hi plane and 8 KB of its lo plane
        if (lane == 0) {
            int64_t jg = 0;
            uint32_t issued = 0u, last_ph = 0u;   // bit b: buffer b was filled / its last phase
            bool ok = true;
            for (int64_t u = c; u < U && ok; u += G) {
                const int64_t m = unit_order(p.uoff, L, u);
                GroupSet rest = unit_groups(p.unit_mask, u, NGK);
                for (int g = pop_group(rest); g >= 0; g = pop_group(rest), ++jg) {
                    const uint32_t b = (uint32_t)(jg % kImgBufA), ph = (uint32_t)(jg / kImgBufA) & 1;
                    const uint8_t *src = aimg + ((m * NG + (g >> 2)) * 2) * (int64_t)kAImg + (g & 3) * (kAImgG / 2);
                    tc::prefetch_l2(src, kAImgG / 2);
                    tc::prefetch_l2(src + kAImg, kAImgG / 2);
                    if (!(ok = wait_or_abort(&sh.a_free[b], ph ^ 1, abort, err))) break;
                    tc::mbar_arrive_expect_tx(&sh.a_full[b], kAImgG);
                    tc::bulk_g2s(sA + b * kAImgG, src, kAImgG / 2, &sh.a_full[b]);
                    tc::bulk_g2s(sA + b * kAImgG + kAImgG / 2, src + kAImg, kAImgG / 2, &sh.a_full[b]);
                    issued |= 1u << b;
                    last_ph = (last_ph & ~(1u << b)) | (ph << b);
                }
            }
            // copies still in flight land before the CTA exits (bounded waits)
            for (int b = 0; b < kImgBufA; ++b)
                if ((issued >> b) & 1u) tc::mbar_wait(&sh.a_full[b], (last_ph >> b) & 1u);
        }
    } else {
        // ------------------------------------------------ generators + epilogue
        const int S = warp >> 1;                  // set: active groups at positions S, S + 4, ...
        const int sseg = warp & 1;                // segment of the superblock
        const int t = tid & (kKG - 1);            // lane within the group (the MMA K index)
        const double sgn_c = sgn_of(p.sp);
        // tile: MN-major SW128 planes (hi, then lo) of 256 MN rows (the superblock) and 32 K
        // lanes; per 8 lanes 4 blocks of 64 rows; this thread writes blocks 2 sseg, 2 sseg + 1
        const uint32_t rowbase = tc::smem_u32(sB) + (uint32_t)S * kTileA + (t >> 3) * 4096 +
                                 (uint32_t)(2 * sseg) * 1024 + (t & 7) * 128;
        uint32_t js = 0;   // groups generated into this set's tile
        bool dead = false;
        // this thread's coefficient row of a unit, loaded one unit ahead
        auto unit_coef = [&](int64_t uu) {
            const int64_t mm = unit_order(p.uoff, L, uu);
            const int64_t lbb = first_row(mm, p.sp) + (uu - p.uoff[mm]) * kSB;
            return diff_coef(p.coef, alm_idx(p.lmax, 0, mm), lbb + tid, L, sgn_c, (tid & (kSeg - 1)) == 0);
        };
        float4 ncoef = c < U ? unit_coef(c) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int64_t u = c; u < U; u += G) {
            const int64_t m = unit_order(p.uoff, L, u);
            const int64_t s = u - p.uoff[m];
            const int64_t lb = first_row(m, p.sp) + s * kSB;
            const int64_t mb = alm_idx(p.lmax, 0, m);
            // coefficient rows of the unit (the previous unit's rows are no longer read: every
            // generator has passed its epilogue)
            gen_barrier_a();
            if (!dead) sCf[tid] = ncoef;
            gen_barrier_a();
            if (!dead && u + G < U) ncoef = unit_coef(u + G);
            // this thread's segment; the second half of an order's last superblock may lie
            // past the order's last segment (all its rows are >= L): it then starts from zero
            const int64_t seg = p.segoff[m] + 2 * s + sseg;
            const bool has_seg = seg < p.segoff[m + 1];
            const int64_t segrow = seg * p.nlanes;
            // lane state of the set's next group is loaded while this one is generated
            float2 nst = make_float2(0.f, 0.f);
            int nn = 0;
            double nx = 1.0;
            auto fetch = [&](int64_t g) {
                const int64_t j = g * kKG + t;
                nst = make_float2(0.f, 0.f);
                nn = 0;
                nx = 1.0;
                if (has_seg && j < p.nlanes) {   // padding lanes stay exactly zero
                    nst = __ldg(p.ck + segrow + j);
                    nn = __ldg(p.cn + segrow + j);
                    nx = __ldg(p.geom + j);
                }
            };
            // this set's groups: the active groups at positions S, S + 4, ... of the unit
            const GroupSet umask = unit_groups(p.unit_mask, u, NGK);
            GroupSet rest = umask;
            for (int q = 0; q < S; ++q) pop_group(rest);
            int g = pop_group(rest);
            if (!dead && g >= 0) fetch(g);
            for (; g >= 0; ++js) {
                for (int q = 1; q < kSetsA; ++q) pop_group(rest);   // the other sets' groups
                const int gnext = pop_group(rest);
                if (dead) {
                    g = gnext;
                    continue;
                }
                float v = nst.x, D = nst.y;
                const float y = (float)(nx - 1.0);
                int n = nn;
                if (gnext >= 0) fetch(gnext);
                g = gnext;
                if (!warp_wait(&sh.b_free[S], (js & 1) ^ 1, abort, err)) {
                    dead = true;
                    continue;
                }
                // 128 rows of the lane: MN blocks 2 sseg (rows 0-63) and 2 sseg + 1; a thread
                // stores 8 consecutive rows as 16 bytes, the lo plane kTileA / 2 bytes further
                gen_rows64(sCf + kSeg * sseg, y, v, D, n, rowbase, kTileA / 2, (uint32_t)(t & 7));
                gen_rows64(sCf + kSeg * sseg + kHalf, y, v, D, n, rowbase + 1024, kTileA / 2, (uint32_t)(t & 7));
                tc::fence_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh.b_full[S]);
            }
            // epilogue of the unit: each alm element receives exactly one addition per launch,
            // from one thread, so the result does not depend on the order of the units.  Warp
            // w reads TMEM lanes 32 (w % 4), superblock rows 128 (w / 4) + [0, 128).
            const uint32_t q = (uint32_t)((u - c) / G);
            if (!dead && !warp_wait(&sh.d_full, q & 1, abort, err)) dead = true;
            // a unit without active groups adds nothing (its accumulator was never written)
            const bool out = !dead && (umask.w0 | umask.w1) != 0ull;
            if (SPIN == 2 && 2 * p.H >= 64) {
                // spin 2: the north image rows r < H feed alm rows o0 + r and the south rows
                // H + r' feed rows o1 + r' (o0 != o1, so no row receives both): each thread adds
                // its TMEM lane straight into the alm rows, one 256-byte row segment per warp
                // (with fewer than 64 image rows the staged path below spreads the additions
                // over all the worker threads instead)
                if (out) {
                    tc::tc_fence_after();
                    const int r = 32 * (warp & 3) + lane, c0 = 128 * (warp >> 2);
                    const bool north = r < p.H, valid = r < 2 * p.H;
                    const int orow = north ? p.o0 + r : p.o1 + (r - p.H);
                    double *dst = alm_i + (mb + lb) * p.NR + orow;
                    for (int cb = c0; cb < c0 + 128; cb += 16) {
                        uint32_t rh[16], rx[16];
                        const uint32_t ta = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)cb;
                        tc::tmem_ld16(ta, rh);
                        tc::tmem_ld16(ta + kSB, rx);
                        tc::tmem_ld_wait();
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int i = cb + e;
                            if (valid && lb + i < L) {
                                double val = (double)(__uint_as_float(rh[e]) + __uint_as_float(rx[e]));
                                if (!north && ((lb + i + m) & 1)) val = -val;
                                atomicAdd(dst + (int64_t)i * p.NR, val * p.scale);
                            }
                        }
                    }
                    tc::tc_fence_before();
                }
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh.d_free);   // TMEM may be overwritten
                continue;
            }
            // spin 0: the two hemisphere halves of the image rows add into the same alm rows,
            // so the accumulators are staged in shared memory (the tiles and coefficient rows,
            // free now) and each element is then summed by one thread
            float *stage = reinterpret_cast<float *>(sB);   // [128 rows][kStageLd] floats
            if (out) {
                tc::tc_fence_after();
                const int row = 32 * (warp & 3) + lane, c0 = 128 * (warp >> 2);
                for (int cb = c0; cb < c0 + 128; cb += 16) {
                    uint32_t r[16], rx[16];
                    const uint32_t ta = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)cb;
                    tc::tmem_ld16(ta, r);
                    tc::tmem_ld16(ta + kSB, rx);
                    tc::tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        stage[row * kStageLd + cb + e] = __uint_as_float(r[e]) + __uint_as_float(rx[e]);
                }
                tc::tc_fence_before();
            }
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh.d_free);   // TMEM may be overwritten
            gen_barrier_a();                               // every row staged
            if (out) {
                // output (row orow of the interleaved alm, row l = lb + i): the north image row
                // orow - o0 and the south image row H + orow - o1 (with the hemisphere parity
                // (-1)^(l + m)) where they exist; consecutive threads take consecutive orow
                const int nout = p.NR * kSB;
                for (int f = tid; f < nout; f += kGenA) {
                    const int orow = f % p.NR, i = f / p.NR;
                    const int64_t l = lb + i;
                    if (l >= L) continue;
                    const int rn = orow - p.o0, rs = orow - p.o1;
                    double val = 0.0;
                    if (rn >= 0 && rn < p.H) val += (double)stage[rn * kStageLd + i];
                    if (rs >= 0 && rs < p.H) {
                        const double sv = (double)stage[(p.H + rs) * kStageLd + i];
                        val += ((l + m) & 1) ? -sv : sv;
                    }
                    // one reduction per element and launch (no return value: it does not wait)
                    atomicAdd(alm_i + (mb + l) * p.NR + orow, val * p.scale);
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarpA) tc::tmem_dealloc(tmem, 512);
}

// ------------------------------------------------------------------------------ synthesis

struct __align__(8) SynShared {
    uint64_t a_full[2], a_free[2], b_full[2], b_free[2], d_full, drain;
    uint32_t tmem;
    int abort;
};

__device__ __forceinline__ void set_barrier_s(int set)
{
    asm volatile("bar.sync %0, 256;" ::"r"(2 + set) : "memory");
}

// One CTA per (order m, tile of 256 lanes).  Chunk cc of order m covers rows
// l0 + 64 cc + [0, 64) (image index choff[m] + cc); segment k = chunks 2k, 2k + 1.  Only the
// segments in which some lane of the tile has a non-zero state are generated and
// contracted (the others are exactly zero); the i-th of them is generated by set i % 2
// from its checkpoint.  D[row, lane] = sum_l almT[row, l] lambda_l(lane).
constexpr int kMaxSegS = 512;   // segments of an order at lmax <= 65535
template <int SPIN>
__global__ void __launch_bounds__(kThrS, 1) k_syn_ck(CkParams p, const uint8_t *__restrict__ simg,
                                                     const int64_t *__restrict__ choff,
                                                     float *__restrict__ synd, int R2,
                                                     int *__restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ SynShared sh;
    __shared__ short slist[kMaxSegS];   // active segments of the order, ascending
    __shared__ int snact;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (tc::smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t *smem = smem_raw + (base - tc::smem_u32(smem_raw));
    uint8_t *sA = smem;                                              // 2 x (hi, lo) alm images
    uint8_t *sB = smem + 4 * kSImg;                                  // 2 sets x (hi, lo) tiles
    float4 *sCf = reinterpret_cast<float4 *>(sB + 4 * kBTileS);     // 2 sets x kSeg rows
    const int64_t L = p.lmax + 1;
    const int64_t m = blockIdx.y, tile = blockIdx.x;
    const int64_t l0 = first_row(m, p.sp);
    if (l0 > p.lmax) return;
    const int64_t nch = (L - l0 + kKL - 1) / kKL;
    const int nseg = (int)((nch + 1) / 2);

    if (warp == 0) {
        // active segments: some 64-lane group of this tile's 256 lanes has a non-zero state
        const int64_t s0 = p.segoff[m];
        int cnt = 0;
        for (int b0 = 0; b0 < nseg; b0 += 32) {
            const int k = b0 + lane;
            bool act = false;
            if (k < nseg) {
                act = true;
                if (p.seg_mask && p.nlanes <= 4096)
                    act = ((__ldg(p.seg_mask + s0 + k) >> (4 * tile)) & 0xFull) != 0ull;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, act);
            if (act) slist[cnt + __popc(bal & ((1u << lane) - 1u))] = (short)k;
            cnt += __popc(bal);
        }
        if (lane == 0) snact = cnt;
    }
    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sh.a_full[i], 1);
            tc::mbar_init(&sh.a_free[i], 1);
            tc::mbar_init(&sh.b_full[i], kLT / 32);
            tc::mbar_init(&sh.b_free[i], 1);
        }
        tc::mbar_init(&sh.d_full, 1);
        tc::mbar_init(&sh.drain, 1);
        sh.abort = 0;
        tc::fence_mbar_init();
    }
    if (warp == kMmaWarpS) {
        tc::tmem_alloc(&sh.tmem, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh.tmem;
    volatile int *abort = &sh.abort;
    const int nact = snact;
    const uint8_t *img = simg + (choff[m] - choff[0]) * 2 * (int64_t)kSImg;
    // absolute chunk of the c-th active chunk walk: segment slist[i], half h
    auto chunk_of = [&](int i, int h) { return 2 * (int64_t)slist[i] + h; };
    auto chunks_in = [&](int i) { return 2 * (int64_t)slist[i] + 1 < nch ? 2 : 1; };

    if (warp == kMmaWarpS) {
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_f16(128, kLT, 0, 1, 0);
            bool ok = true;
            int issued = -1;            // buffer of an image copy not yet waited for
            uint32_t issued_ph = 0;     // and the phase it completes
            uint32_t cs[2] = {0u, 0u};  // chunks consumed from each set's tile
            int64_t c = 0;              // active chunks so far (image ring position)
            if (nact > 0) {
                tc::mbar_arrive_expect_tx(&sh.a_full[0], 2 * kSImg);
                tc::bulk_g2s(sA, img + chunk_of(0, 0) * 2 * (int64_t)kSImg, 2 * kSImg, &sh.a_full[0]);
                issued = 0;
            }
            for (int i = 0; i < nact && ok; ++i) {
                const int S = i & 1, nh = chunks_in(i);
                for (int h = 0; h < nh && ok; ++h, ++c) {
                    const uint32_t a = (uint32_t)c & 1, pha = (uint32_t)(c >> 1) & 1;
                    if (!(ok = wait_or_abort(&sh.a_full[a], pha, abort, err))) break;
                    issued = -1;
                    if (!(ok = wait_or_abort(&sh.b_full[S], cs[S] & 1, abort, err))) break;
                    tc::tc_fence_after();
                    const uint32_t a0 = tc::smem_u32(sA + a * 2 * kSImg);
                    const uint32_t b0 = tc::smem_u32(sB + S * 2 * kBTileS);
#pragma unroll
                    for (int ks = 0; ks < kKL / 16; ++ks) {
                        const uint64_t ah = tc::desc_sw128_mn(a0 + ks * 4096, 1024, 2048);
                        const uint64_t al = tc::desc_sw128_mn(a0 + kSImg + ks * 4096, 1024, 2048);
                        const uint64_t bh = tc::desc_sw128(b0 + ks * 32);
                        const uint64_t bl = tc::desc_sw128(b0 + kBTileS + ks * 32);
                        const uint32_t acc = (c > 0 || ks > 0) ? 1u : 0u;
                        tc::mma_f16(tmem, ah, bh, idesc, acc);
                        tc::mma_f16(tmem + kLT, ah, bl, idesc, acc);
                        tc::mma_f16(tmem + kLT, al, bh, idesc, 1u);
                    }
                    tc::mma_commit(&sh.b_free[S]);
                    tc::mma_commit(&sh.a_free[a]);
                    ++cs[S];
                    // the next active chunk's image goes into the buffer of chunk c - 1 once
                    // its MMAs are done
                    const bool more = h + 1 < nh || i + 1 < nact;
                    if (more) {
                        const int64_t cn = h + 1 < nh ? chunk_of(i, h + 1) : chunk_of(i + 1, 0);
                        const uint32_t nb = (uint32_t)(c + 1) & 1;
                        if (!(ok = wait_or_abort(&sh.a_free[nb], ((uint32_t)((c + 1) >> 1) & 1) ^ 1, abort, err)))
                            break;
                        tc::mbar_arrive_expect_tx(&sh.a_full[nb], 2 * kSImg);
                        tc::bulk_g2s(sA + nb * 2 * kSImg, img + cn * 2 * (int64_t)kSImg, 2 * kSImg, &sh.a_full[nb]);
                        issued = (int)nb;
                        issued_ph = (uint32_t)((c + 1) >> 1) & 1;
                    }
                }
            }
            if (ok) tc::mma_commit(&sh.d_full);
            tc::mma_commit(&sh.drain);
            tc::mbar_wait(&sh.drain, 0);
            if (issued >= 0) tc::mbar_wait(&sh.a_full[issued], issued_ph);
        }
    } else {
        const int S = warp >> 3;              // set: active segments i with i % 2 == S
        const int t = tid & (kLT - 1);        // lane within the tile (the MMA N row)
        const int64_t jl = tile * kLT + t;
        const bool valid = jl < p.nlanes;
        const double sgn_c = sgn_of(p.sp);
        const int64_t mb = alm_idx(p.lmax, 0, m);
        const float y = valid ? (float)(p.geom[jl] - 1.0) : 0.f;
        float4 *cwin = sCf + kSeg * S;
        const uint32_t b0 = tc::smem_u32(sB + S * 2 * kBTileS);
        const uint32_t rowoff = (uint32_t)((t >> 3) * 1024 + (t & 7) * 128);
        uint32_t js = 0;   // chunks generated by this set
        bool dead = false;
        // state and coefficient row of the set's next segment, loaded one segment ahead
        float2 nst = make_float2(0.f, 0.f);
        int nn = 0;
        float4 ncoef = make_float4(0.f, 0.f, 0.f, 0.f);
        auto fetch = [&](int i) {
            nst = make_float2(0.f, 0.f);
            nn = 0;
            if (i >= nact) return;
            const int64_t k = slist[i];
            if (valid) {
                const int64_t idx = (p.segoff[m] + k) * p.nlanes + jl;
                nst = __ldg(p.ck + idx);
                nn = __ldg(p.cn + idx);
            }
            if (t < kSeg) ncoef = diff_coef(p.coef, mb, l0 + kSeg * k + t, L, sgn_c, t == 0);
        };
        fetch(S);
        for (int i = S; i < nact; i += 2) {
            set_barrier_s(S);   // the set's previous segment is generated: its rows are free
            if (!dead && t < kSeg) cwin[t] = ncoef;
            set_barrier_s(S);
            if (dead) continue;
            float v = nst.x, D = nst.y;
            int n = nn;
            fetch(i + 2);
            const int nh = chunks_in(i);
            for (int half = 0; half < nh; ++half, ++js) {
                if (!warp_wait(&sh.b_free[S], (js & 1) ^ 1, abort, err)) {
                    dead = true;
                    break;
                }
                // tile: K-major SW128, 256 N rows (lanes) of 64 K values (rows l)
                gen_rows64(cwin + kKL * half, y, v, D, n, b0 + rowoff, kBTileS, (uint32_t)(t & 7));
                tc::fence_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh.b_full[S]);
            }
        }
        // epilogue: D[row, lane] -> synd[m][lane][row]; warp w reads TMEM lanes 32 (w % 4)
        // (rows) and the column quarter w / 4 (lanes).  Without active segments the
        // output is zero (the accumulator was never written).
        if (!dead && warp_wait(&sh.d_full, 0, abort, err)) {
            tc::tc_fence_after();
            const int wq = warp & 3, row = wq * 32 + lane;
            const int cbeg = (warp >> 2) * (kLT / 4);
            for (int cb = cbeg; cb < cbeg + kLT / 4; cb += 16) {
                uint32_t r[16], rx[16];
                if (nact > 0) {
                    const uint32_t trow = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)cb;
                    tc::tmem_ld16(trow, r);
                    tc::tmem_ld16(trow + kLT, rx);
                    tc::tmem_ld_wait();
                } else {
#pragma unroll
                    for (int e = 0; e < 16; ++e) r[e] = rx[e] = 0u;
                }
                if (row < R2) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int64_t j2 = tile * kLT + cb + e;
                        if (j2 < p.nlanes)
                            synd[(m * p.nlanes + j2) * R2 + row] =
                                (__uint_as_float(r[e]) + __uint_as_float(rx[e])) * (float)p.scale;
                    }
                }
            }
            tc::tc_fence_before();
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarpS) tc::tmem_dealloc(tmem, 512);
}

}  // namespace lck
}  // namespace gm

using namespace gm;
using namespace gm::lck;

static bool ck_spin_ok(int spin, int sp)
{
    return (spin == 0 && sp == 0) || (spin == 2 && (sp == 2 || sp == -2));
}

static int64_t ck_nseg(int64_t lmax, int spin, int64_t m)
{
    const int64_t l0 = first_row(m, spin);
    return l0 <= lmax ? (lmax + 1 - l0 + kSeg - 1) / kSeg : 0;
}

extern "C" int gm_ck_offsets(int64_t lmax, int spin, int64_t *segoff_host, int64_t *uoff_host)
{
    if (lmax < 2 || lmax > 65535 || (spin != 0 && spin != 2)) return GM_ERR_BAD_SHAPE;
    if (!segoff_host || !uoff_host) return GM_ERR_BAD_PTR;
    int64_t s = 0, u = 0;
    for (int64_t m = 0; m <= lmax; ++m) {
        segoff_host[m] = s;
        uoff_host[m] = u;
        const int64_t n = ck_nseg(lmax, spin, m);
        s += n;
        u += (n + 1) / 2;
    }
    segoff_host[lmax + 1] = s;
    uoff_host[lmax + 1] = u;
    return GM_OK;
}

extern "C" int64_t gm_ck_table_entries(int64_t nside, int64_t lmax, int spin)
{
    if (nside < 1 || lmax < 2 || (spin != 0 && spin != 2)) return -1;
    int64_t s = 0;
    for (int64_t m = 0; m <= lmax; ++m) s += ck_nseg(lmax, spin, m);
    return s * 2 * nside;
}

extern "C" int gm_ck_build(int64_t nside, int64_t lmax, int spin, int sp, const double *geom,
                           const double *seeds, const double *coef, const int64_t *segoff,
                           void *ck_state, uint8_t *ck_shift, void *stream)
{
    if (nside < 1 || lmax < 2 || lmax > 65535 || !ck_spin_ok(spin, sp)) return GM_ERR_BAD_SHAPE;
    if (!geom || !seeds || !coef || !segoff || !ck_state || !ck_shift) return GM_ERR_BAD_PTR;
    const int var = sp == 0 ? 0 : (sp < 0 ? 1 : 2);
    dim3 grid((unsigned)((2 * nside + 127) / 128), (unsigned)(lmax + 1));
    k_ck_build<<<grid, 128, 0, as_stream(stream)>>>(nside, lmax, sp, var, geom, seeds, coef, segoff,
                                                    (float2 *)ck_state, ck_shift);
    return check_launch("gm_ck_build");
}

static CkParams ck_params(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp, const double *geom,
                          const double *coef, const int64_t *segoff, const int64_t *uoff,
                          const void *ck_state, const uint8_t *ck_shift, double scale)
{
    CkParams p;
    p.nside = nside;
    p.lmax = lmax;
    p.nlanes = 2 * nside;
    p.sp = sp;
    p.H = spin == 0 ? (int)(2 * ncomp) : (int)ncomp;
    p.NR = spin == 0 ? p.H : 2 * p.H;
    if (spin == 0) { p.o0 = 0; p.o1 = 0; }
    else if (sp < 0) { p.o0 = 0; p.o1 = p.H; }
    else { p.o0 = p.H; p.o1 = 0; }
    p.scale = scale;
    p.geom = geom;
    p.coef = coef;
    p.segoff = segoff;
    p.uoff = uoff;
    p.ck = (const float2 *)ck_state;
    p.cn = ck_shift;
    p.seg_mask = nullptr;
    p.unit_mask = nullptr;
    return p;
}

static bool ck_shape_ok(int spin, int64_t ncomp)
{
    if (spin == 0) return ncomp >= 1 && ncomp <= 32;
    if (spin == 2) return ncomp >= 2 && ncomp <= 64 && ncomp % 2 == 0;
    return false;
}

static int ck_analysis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp, const double *geom,
                       const double *coef, const int64_t *segoff, const int64_t *uoff, const void *ck_state,
                       const uint8_t *ck_shift, const uint64_t *unit_mask, const void *img, double *alm_i,
                       double scale, int64_t nctas, int32_t *err, void *stream)
{
    // the lane groups of a unit are walked as the bits of two 64-bit words: 128 x kKG lanes
    if (nside < 1 || 2 * nside > kMaxGroupsA * kKG || lmax < 2 || lmax > 65535 || !ck_shape_ok(spin, ncomp) ||
        !ck_spin_ok(spin, sp) || nctas < 1 || nctas > 4096)
        return GM_ERR_BAD_SHAPE;
    if (!geom || !coef || !segoff || !uoff || !ck_state || !ck_shift || !img || !alm_i || !err)
        return GM_ERR_BAD_PTR;
    const size_t smem = kImgBufA * kAImgG + kSetsA * kTileA + kSB * sizeof(float4) + 1024;
    auto kern = spin == 0 ? k_ana_ck<0> : k_ana_ck<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_error("gm_ck_analysis attr", e);
        return GM_ERR_LAUNCH;
    }
    CkParams p = ck_params(nside, lmax, spin, sp, ncomp, geom, coef, segoff, uoff, ck_state, ck_shift, scale);
    p.unit_mask = (const unsigned long long *)unit_mask;
    kern<<<(unsigned)nctas, kThrA, smem, as_stream(stream)>>>(p, (const uint8_t *)img, alm_i, (int *)err);
    return check_launch("gm_ck_analysis");
}

extern "C" int gm_ck_analysis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                              const double *geom, const double *coef, const int64_t *segoff,
                              const int64_t *uoff, const void *ck_state, const uint8_t *ck_shift,
                              const void *img, double *alm_i, double scale, int64_t nctas, int32_t *err,
                              void *stream)
{
    return ck_analysis(nside, lmax, spin, sp, ncomp, geom, coef, segoff, uoff, ck_state, ck_shift, nullptr, img,
                       alm_i, scale, nctas, err, stream);
}

extern "C" int gm_ck_analysis_masked(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                                     const double *geom, const double *coef, const int64_t *segoff,
                                     const int64_t *uoff, const void *ck_state, const uint8_t *ck_shift,
                                     const uint64_t *unit_mask, const void *img, double *alm_i, double scale,
                                     int64_t nctas, int32_t *err, void *stream)
{
    if (!unit_mask) return GM_ERR_BAD_PTR;
    return ck_analysis(nside, lmax, spin, sp, ncomp, geom, coef, segoff, uoff, ck_state, ck_shift, unit_mask,
                       img, alm_i, scale, nctas, err, stream);
}

extern "C" int64_t gm_ck_segments(int64_t lmax, int spin)
{
    if (lmax < 2 || lmax > 65535 || (spin != 0 && spin != 2)) return -1;
    int64_t s = 0;
    for (int64_t m = 0; m <= lmax; ++m) s += ck_nseg(lmax, spin, m);
    return s;
}

extern "C" int gm_ck_masks(int64_t nside, int64_t lmax, int spin, const void *ck_state, const uint8_t *ck_shift,
                           const int64_t *segoff, const int64_t *uoff, uint64_t *seg_mask, uint64_t *unit_mask,
                           void *stream)
{
    if (nside < 1 || 2 * nside > 4096 || lmax < 2 || lmax > 65535 || (spin != 0 && spin != 2))
        return GM_ERR_BAD_SHAPE;
    if (!ck_state || !ck_shift || !segoff || !uoff || !seg_mask || !unit_mask) return GM_ERR_BAD_PTR;
    const int64_t nseg = gm_ck_segments(lmax, spin);
    cudaStream_t s = as_stream(stream);
    const unsigned blocks = (unsigned)(nseg < 148 * 16 ? nseg : 148 * 16);
    k_ck_seg_mask<<<blocks, 256, 0, s>>>(2 * nside, nseg, (const float2 *)ck_state, ck_shift,
                                         (unsigned long long *)seg_mask);
    int st = check_launch("gm_ck_masks segments");
    if (st != GM_OK) return st;
    k_ck_unit_mask<<<148 * 4, 256, 0, s>>>(lmax + 1, segoff, uoff, (const unsigned long long *)seg_mask,
                                          (unsigned long long *)unit_mask);
    return check_launch("gm_ck_masks units");
}

extern "C" int gm_ck_syn_chunk_offsets(int64_t lmax, int spin, int64_t *choff_host)
{
    if (lmax < 0 || (spin != 0 && spin != 2)) return GM_ERR_BAD_SHAPE;
    if (!choff_host) return GM_ERR_BAD_PTR;
    int64_t acc = 0;
    for (int64_t m = 0; m <= lmax; ++m) {
        choff_host[m] = acc;
        const int64_t l0 = first_row(m, spin);
        if (l0 <= lmax) acc += (lmax + 1 - l0 + kKL - 1) / kKL;
    }
    choff_host[lmax + 1] = acc;
    return GM_OK;
}

static int ck_synthesis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp, const double *geom,
                        const double *coef, const int64_t *segoff, const void *ck_state, const uint8_t *ck_shift,
                        const uint64_t *seg_mask, const void *simg, const int64_t *choff, float *synd,
                        double out_scale, int32_t *err, void *stream)
{
    if (nside < 1 || lmax < 2 || lmax > 65535 || !ck_shape_ok(spin, ncomp) || !ck_spin_ok(spin, sp) ||
        !(out_scale > 0.0))
        return GM_ERR_BAD_SHAPE;
    if (!geom || !coef || !segoff || !ck_state || !ck_shift || !simg || !choff || !synd || !err)
        return GM_ERR_BAD_PTR;
    const size_t smem = 4 * kSImg + 4 * kBTileS + 2 * kSeg * sizeof(float4) + 1024;
    auto kern = spin == 0 ? k_syn_ck<0> : k_syn_ck<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_error("gm_ck_synthesis attr", e);
        return GM_ERR_LAUNCH;
    }
    CkParams p = ck_params(nside, lmax, spin, sp, ncomp, geom, coef, segoff, nullptr, ck_state, ck_shift,
                           out_scale);
    p.seg_mask = (const unsigned long long *)seg_mask;
    const int R2 = 2 * p.H;
    dim3 grid((unsigned)((p.nlanes + kLT - 1) / kLT), (unsigned)(lmax + 1));
    kern<<<grid, kThrS, smem, as_stream(stream)>>>(p, (const uint8_t *)simg, choff, synd, R2, (int *)err);
    return check_launch("gm_ck_synthesis");
}

extern "C" int gm_ck_synthesis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                               const double *geom, const double *coef, const int64_t *segoff,
                               const void *ck_state, const uint8_t *ck_shift, const void *simg,
                               const int64_t *choff, float *synd, double out_scale, int32_t *err,
                               void *stream)
{
    return ck_synthesis(nside, lmax, spin, sp, ncomp, geom, coef, segoff, ck_state, ck_shift, nullptr, simg, choff,
                        synd, out_scale, err, stream);
}

extern "C" int gm_ck_synthesis_masked(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                                      const double *geom, const double *coef, const int64_t *segoff,
                                      const void *ck_state, const uint8_t *ck_shift, const uint64_t *seg_mask,
                                      const void *simg, const int64_t *choff, float *synd, double out_scale,
                                      int32_t *err, void *stream)
{
    if (!seg_mask) return GM_ERR_BAD_PTR;
    return ck_synthesis(nside, lmax, spin, sp, ncomp, geom, coef, segoff, ck_state, ck_shift, seg_mask, simg,
                        choff, synd, out_scale, err, stream);
}
