// Batched Legendre / Wigner-d contraction on the 5th-generation tensor cores (sm_100a).
//
// The rows lambda^{s'}_lm(theta) = sqrt((2l+1)/4pi) d^l_{m,s'}(theta) are generated on the
// fly by the FP64 three-term recurrence in l (one lane = one northern ring per thread),
// rounded to FP32 and split into f16 hi + lo, and written straight into the shared-memory
// operand of tcgen05.mma.  The other operand is a batch of right-hand sides (up to 128
// real rows: maps x re/im x hemisphere), delivered by the bulk-copy (TMA) engine as a
// pre-split, pre-swizzled, power-of-two-scaled image.  Each product runs as three f16 MMAs
// (hi*hi + hi*lo + lo*hi) accumulating in FP32 in tensor memory, hi*hi and the two cross
// products in separate accumulators (the tensor-core accumulation truncates, so its bias
// grows with the chain of MMAs into one accumulator); the epilogue adds the two, applies
// the hemisphere parity and accumulates in FP64.
//
// Analysis (map -> alm): D[row, l] = sum_lanes rhs[row, lane] lambda_l(lane).  One
// persistent CTA per order m at a time walks l in superblocks of 256 (two 128-row tiles,
// each with a hi x hi and a cross-product accumulator of 128 columns: the 512 TMEM
// columns) and, inside a superblock, the lanes in groups of 128 (K); the recurrence state
// of every lane is carried across superblocks in a caller-provided scratch buffer.
//
// Synthesis (alm -> ring coefficients): D[row, lane] = sum_l almT[row, l] lambda_l(lane).
// One CTA per (order m, tile of 256 lanes) walks l in chunks of 64 (K).
//
// Replaces gmaster/_native/cuda/march_v2.cu:155-407 (FP32 SIMT march) for batched maps.
#include <math.h>

#include <mutex>

#include "gm_common.cuh"
#include "tc_common.cuh"
#include "ltc_common.cuh"

namespace gm {
namespace ltc {

constexpr int kGen = 128;              // generator threads (4 warps)
constexpr int kThreads = kGen + 32;    // + one warp for the producer / MMA issuer
constexpr int kSB = 256;               // analysis superblock (l per D accumulator)
constexpr int kTmemCols = 512;         // TMEM columns: the hi*hi and the cross accumulators
constexpr int kNB = 128;               // analysis l-tile (MMA N of the hi x hi product)
constexpr int kKC = 128;               // analysis lanes per group (MMA K per group)
constexpr int kLT = 256;               // synthesis lanes per CTA (MMA N)
constexpr int kGenS = kLT;             // synthesis generator threads (8 warps, one lane each)
constexpr int kThreadsS = kGenS + 32;  // + the producer / MMA warp
constexpr int kMmaWarpS = kGenS / 32;  // warp index of the synthesis producer / MMA warp
constexpr int kKL = 64;                // synthesis l-chunk (MMA K per chunk)
constexpr uint32_t kAImg = 128u * kKC * 2u;        // one plane of an analysis A image (32 KB)
constexpr uint32_t kBTileA = kNB * kKC * 2u;       // one plane of an analysis B tile (32 KB)
constexpr uint32_t kSImg = 128u * kKL * 2u;        // one plane of a synthesis A image (16 KB)
constexpr uint32_t kBTileS = kLT * kKL * 2u;       // one plane of a synthesis B tile (32 KB)
struct Params {
    int64_t nside, lmax, nlanes;
    int sp;          // s' of the rows: 0, -2 or +2
    int H;           // rows per half (maps x re/im); valid rows 2H <= 128
    int NR;          // rows of the interleaved alm (spin 0: H, spin 2: 2H)
    int o0, o1;      // output row base of the first / second half (analysis)
    double scale;    // analysis: alm += scale * result
    const double *geom;   // (3, nlanes)
    const double *seeds;  // (3, L, 4)
    const double *coef;   // (nelem, 4) for this spin: alpha, beta, c0, 0
    int var;              // seed variant 0 / 1 / 2
    int64_t mbeg, mend;   // orders handled, [mbeg, mend); images and outputs are indexed by m - mbeg
};

__device__ __forceinline__ void gen_barrier() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
__device__ __forceinline__ void gen_barrier_s() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// ------------------------------------------------------------------------------- analysis

struct __align__(8) AnaShared {
    uint64_t a_full[2], a_free[2], b_full[2], b_free[2], d_full, d_free;
    uint32_t tmem;
    int abort;
};

// The m handled in slot i of CTA c (snake order over gridDim.x CTAs).
__device__ __forceinline__ int64_t snake_m(int64_t i, int64_t c, int64_t G)
{
    const int64_t round = i, pos = (round & 1) ? (G - 1 - c) : c;
    return round * G + pos;
}

template <int SPIN>
__global__ void __launch_bounds__(kThreads, 1) k_ana_tc(Params p, const uint8_t *__restrict__ aimg,
                                                        double *__restrict__ alm_i,
                                                        double *__restrict__ scratch,
                                                        int *__restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ AnaShared sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (tc::smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t *smem = smem_raw + (base - tc::smem_u32(smem_raw));
    uint8_t *sA = smem;                      // right-hand-side image, hi and lo planes (64 KB)
    uint8_t *sB = smem + 2 * kAImg;          // 2 stages of generated tiles, hi and lo (2 x 64 KB)
    double2 *sAB = reinterpret_cast<double2 *>(smem + 2 * kAImg + 4 * kBTileA);   // (alpha, beta) x kSB
    double *sC0 = reinterpret_cast<double *>(sAB + kSB);                          // c0 x kSB (spin 2)
    const int64_t L = p.lmax + 1, NG = (p.nlanes + kKC - 1) / kKC;
    const int64_t G = gridDim.x, c = blockIdx.x;
    const int l0min = abs(p.sp);

    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sh.a_full[i], 1);
            tc::mbar_init(&sh.a_free[i], 1);
            tc::mbar_init(&sh.b_full[i], 4);
            tc::mbar_init(&sh.b_free[i], 1);
        }
        tc::mbar_init(&sh.d_full, 1);
        tc::mbar_init(&sh.d_free, 4);
        sh.abort = 0;
        tc::fence_mbar_init();
    }
    if (warp == 4) {
        tc::tmem_alloc(&sh.tmem, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh.tmem;
    volatile int *abort = &sh.abort;

    if (warp == 4) {
        // ------------------------------------------------ producer + MMA issuer
        if (lane == 0) {
            // The first MMA of a K step multiplies the hi image by the hi and lo generated
            // planes at once (N = 2 kNB: they sit side by side in the tile), writing the
            // hi x hi half and the hi x lo half of the tile's accumulator; the second adds
            // lo x hi into the cross half.  Reading the image once for both products keeps
            // the tensor core's shared-memory traffic, which stalls the generators' own
            // shared-memory accesses, down.
            const uint32_t idesc_cat = tc::idesc_f16(128, 2 * kNB, 0, 1, 1);
            const uint32_t idesc_hi = tc::idesc_f16(128, kNB, 0, 1, 1);
            uint32_t j = 0, u = 0, q = 0;   // job, B-tile and superblock counters
            // job list: (slot i -> m, superblock s, group g)
            auto job_m = [&](int64_t i) { return p.mbeg + snake_m(i, c, G); };
            int64_t i = 0, s = 0, g = 0;
            bool have = job_m(i) < p.mend;
            if (have) {
                tc::mbar_arrive_expect_tx(&sh.a_full[0], 2 * kAImg);
                tc::bulk_g2s(sA, aimg + (((job_m(i) - p.mbeg) * NG + g) * 2) * (int64_t)kAImg, 2 * kAImg,
                             &sh.a_full[0]);
            }
            while (have && !*abort) {
                const int64_t m = job_m(i);
                const int64_t l0 = m > l0min ? m : l0min;
                const int64_t nsb = (L - l0 + kSB - 1) / kSB;
                // next job
                int64_t ni = i, ns = s, ng = g + 1;
                if (ng == NG) { ng = 0; ++ns; }
                if (ns == nsb) { ns = 0; ++ni; }
                const bool next = job_m(ni) < p.mend;
                if (!wait_or_abort(&sh.a_full[0], j & 1, abort, err)) break;
                if (g == 0 && !wait_or_abort(&sh.d_free, (q & 1) ^ 1, abort, err)) break;
                tc::tc_fence_after();
                const uint32_t a0 = tc::smem_u32(sA);
                for (int t = 0; t < kSB / kNB; ++t, ++u) {
                    const uint32_t st = u & 1;
                    if (!wait_or_abort(&sh.b_full[st], (u >> 1) & 1, abort, err)) break;
                    tc::tc_fence_after();
                    const uint32_t b0 = tc::smem_u32(sB + st * 2 * kBTileA);
                    // tile t owns the columns [2 kNB t, 2 kNB (t + 1)): hi x hi first, then the
                    // cross products.  The tensor-core accumulation rounds toward zero, so its
                    // relative bias grows with the number of MMAs chained into one accumulator;
                    // the cross half is 2^-11 smaller and its bias is negligible.
                    const uint32_t dh = tmem + t * 2 * kNB, dx = dh + kNB;
                    const uint32_t acc = g > 0 ? 1u : 0u;
#pragma unroll
                    for (int ks = 0; ks < kKC / 16; ++ks) {
                        const uint64_t ah = tc::desc_sw128_mn(a0 + ks * 4096, 1024, 2048);
                        const uint64_t al = tc::desc_sw128_mn(a0 + kAImg + ks * 4096, 1024, 2048);
                        const uint64_t bt = tc::desc_sw128_mn(b0 + ks * 8192, 1024, 4096);
                        tc::mma_f16(dh, ah, bt, idesc_cat, (acc || ks > 0) ? 1u : 0u);
                        tc::mma_f16(dx, al, bt, idesc_hi, 1u);
                    }
                    tc::mma_commit(&sh.b_free[st]);
                }
                if (*abort) break;
                tc::mma_commit(&sh.a_free[0]);
                if (g == NG - 1) {
                    tc::mma_commit(&sh.d_full);
                    ++q;
                }
                if (next) {
                    // one image buffer: refill it once this job's MMAs have read it (the
                    // generators run ahead into the free tile stages meanwhile)
                    if (!wait_or_abort(&sh.a_free[0], j & 1, abort, err)) break;
                    tc::mbar_arrive_expect_tx(&sh.a_full[0], 2 * kAImg);
                    tc::bulk_g2s(sA, aimg + (((job_m(ni) - p.mbeg) * NG + ng) * 2) * (int64_t)kAImg, 2 * kAImg,
                                 &sh.a_full[0]);
                }
                ++j;
                i = ni;
                s = ns;
                g = ng;
                have = next;
            }
        }
    } else {
        // ------------------------------------------------ generators + epilogue
        const double sgn_c = sgn_of(p.sp);
        uint32_t u = 0, q = 0;
        double *my_scratch = scratch + (int64_t)c * p.nlanes * 3;
        // After a timed-out wait (abort) a generator stops working but keeps taking part in
        // every named barrier of the loops, which are bounded by the work list, so no
        // thread can wait on a barrier that its peers have left.
        bool dead = false;
        for (int64_t i = 0;; ++i) {
            const int64_t m = p.mbeg + snake_m(i, c, G);
            if (m >= p.mend) break;
            const int64_t l0 = m > l0min ? m : l0min;
            const int64_t nsb = (L - l0 + kSB - 1) / kSB;
            const int64_t mb = alm_idx(p.lmax, 0, m);   // coefficient / alm base of order m
            for (int64_t s = 0; s < nsb; ++s) {
                const int64_t lb = l0 + s * kSB;
                // coefficients of this superblock into shared memory (every generator has
                // finished the previous superblock: its epilogue waited for all its tiles)
                // Every row is one uniform step v_l = alpha (x - c) v_{l-1} - beta v_{l-2}: the
                // seed row l0 uses (alpha, beta) = (0, -1) with the state entering as
                // (v, vp) = (0, seed), and rows past lmax use (0, 0), which emit exact zeros.
                for (int e = tid; e < kSB; e += kGen) {
                    const int64_t l = lb + e;
                    Coef cf = Coef{0.0, 0.0, 0.0};
                    if (l == l0) cf.beta = -1.0;
                    else if (l < L) cf = load_coef(p.coef, mb + l);
                    sAB[e] = make_double2(cf.alpha, cf.beta);
                    if (SPIN) sC0[e] = sgn_c * cf.c0 * cf.alpha;   // alpha (x - c) = fma(alpha, x, -alpha c)
                }
                gen_barrier();
                // lane state of group g + 1 is loaded while group g is generated
                // (x, then seed inputs or the carried recurrence state)
                double nx = 0.0, na = 0.0, nb = 0.0, nc = 0.0;
                auto prefetch = [&](int64_t gg) {
                    const int64_t jn = gg * kKC + tid;
                    nx = na = nb = nc = 0.0;
                    if (gg < NG && jn < p.nlanes) {
                        nx = p.geom[jn];
                        if (s == 0) {
                            na = p.geom[p.nlanes + jn];
                            nb = p.geom[2 * p.nlanes + jn];
                        } else {
                            na = my_scratch[jn * 3];
                            nb = my_scratch[jn * 3 + 1];
                            nc = my_scratch[jn * 3 + 2];
                        }
                    }
                };
                dead = dead || *abort;
                if (!dead) prefetch(0);
                for (int64_t g = 0; g < NG && !dead; ++g) {
                    const int64_t jl = g * kKC + tid;
                    const bool valid = jl < p.nlanes;
                    double x = 0.0, v = 0.0, vp = 0.0;   // padding lanes stay exactly zero
                    int k = 0;
                    if (valid) {
                        x = nx;
                        if (s == 0) {
                            seed_lane(p.seeds + ((int64_t)p.var * L + m) * 4, na, nb, vp, k);
                        } else {
                            v = na;
                            vp = nb;
                            k = (int)nc;
                        }
                    }
                    prefetch(g + 1);
                    bool emit = (k == 0);
                    for (int t = 0; t < kSB / kNB; ++t, ++u) {
                        const uint32_t st = u & 1;
                        if (!wait_or_abort(&sh.b_free[st], ((u >> 1) & 1) ^ 1, abort, err)) {
                            dead = true;
                            break;
                        }
                        // tile layout: MN-major, 128-byte swizzle, 256 MN rows = kNB hi rows
                        // then kNB lo rows (sw128_mn_offset(256, r, lane)); a thread writes
                        // 8 consecutive rows of its lane as one 16-byte store per plane
                        const uint32_t b0 = tc::smem_u32(sB + st * 2 * kBTileA);
                        const uint32_t rowbase = b0 + (tid >> 3) * 4096 + (tid & 7) * 128;
                        const double2 *cab = sAB + t * kNB;
                        const double *cc0 = sC0 + t * kNB;
#pragma unroll 8
                        for (int cc = 0; cc < kNB / 8; ++cc) {
                            float vals[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const double2 ab = cab[cc * 8 + e];
                                const double a = SPIN ? fma(ab.x, x, -cc0[cc * 8 + e]) : ab.x * x;
                                const double nv = fma(a, v, -ab.y * vp);
                                vp = v;
                                v = nv;
                                vals[e] = emit ? (float)v : 0.0f;
                            }
                            rescale(v, vp, k);
                            emit = (k == 0);
                            uint4 hi, lo;
                            pack8(vals, hi, lo);
                            const uint32_t off = (cc >> 3) * 1024 + (((cc & 7) ^ (tid & 7)) << 4);
                            sts128(rowbase + off, hi);
                            sts128(rowbase + 2048 + off, lo);
                        }
                        tc::fence_async_smem();
                        __syncwarp();
                        if (lane == 0) tc::mbar_arrive(&sh.b_full[st]);
                    }
                    if (valid && s + 1 < nsb && !dead) {
                        my_scratch[jl * 3] = v;
                        my_scratch[jl * 3 + 1] = vp;
                        my_scratch[jl * 3 + 2] = (double)k;
                    }
                }
                // epilogue of superblock s
                if (dead || !wait_or_abort(&sh.d_full, q & 1, abort, err)) {
                    dead = true;
                    continue;
                }
                tc::tc_fence_after();
                const int row = warp * 32 + lane;
                const bool rvalid = row < 2 * p.H;
                const int orow = row < p.H ? p.o0 + row : p.o1 + (row - p.H);
                const bool parity_row = row >= p.H;
                for (int cb = 0; cb < kSB; cb += 16) {
                    uint32_t r[16], rx[16];
                    // column cb of the superblock: tile cb / kNB, hi x hi half then cross half
                    const uint32_t col = (uint32_t)((cb / kNB) * 2 * kNB + cb % kNB);
                    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16) + col;
                    tc::tmem_ld16(trow, r);
                    tc::tmem_ld16(trow + kNB, rx);
                    tc::tmem_ld_wait();
                    if (rvalid) {
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int64_t l = lb + cb + e;
                            if (l < L) {
                                double val = ((double)__uint_as_float(r[e]) + (double)__uint_as_float(rx[e])) *
                                             p.scale;
                                if (parity_row && ((l + m) & 1)) val = -val;
                                atomicAdd(alm_i + (mb + l) * p.NR + orow, val);
                            }
                        }
                    }
                }
                tc::tc_fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh.d_free);
                ++q;
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 4) tc::tmem_dealloc(tmem, kTmemCols);
}

// ------------------------------------------------------------------------------- synthesis

struct __align__(8) SynShared {
    uint64_t a_full[2], a_free[2], b_full[2], b_free[2], d_full;
    uint32_t tmem;
    int abort;
};

// almT images: chunk cc of order m covers l in [64 (c0(m) + cc), +64), c0(m) = floor(l0(m)/64);
// image index = choff[m] + cc.
template <int SPIN>
__global__ void __launch_bounds__(kThreadsS, 1) k_syn_tc(Params p, const uint8_t *__restrict__ simg,
                                                        const int64_t *__restrict__ choff,
                                                        float *__restrict__ synd, int R2,
                                                        int *__restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ SynShared sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (tc::smem_u32(smem_raw) + 1023u) & ~1023u;
    uint8_t *smem = smem_raw + (base - tc::smem_u32(smem_raw));
    uint8_t *sA = smem;                    // 2 x 32 KB
    uint8_t *sB = smem + 4 * kSImg;        // 2 x 64 KB
    double2 *sAB = reinterpret_cast<double2 *>(smem + 4 * kSImg + 4 * kBTileS);   // 2 x kKL (alpha, beta)
    double *sC0 = reinterpret_cast<double *>(sAB + 2 * kKL);                      // 2 x kKL c0
    const int64_t L = p.lmax + 1;
    const int64_t m = p.mbeg + blockIdx.y, tile = blockIdx.x;
    const int l0min = abs(p.sp);
    const int64_t l0 = m > l0min ? m : l0min;
    if (l0 > p.lmax) return;
    const int64_t c0 = l0 / kKL, nch = (L + kKL - 1) / kKL - c0;

    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&sh.a_full[i], 1);
            tc::mbar_init(&sh.a_free[i], 1);
            tc::mbar_init(&sh.b_full[i], kGenS / 32);
            tc::mbar_init(&sh.b_free[i], 1);
        }
        tc::mbar_init(&sh.d_full, 1);
        sh.abort = 0;
        tc::fence_mbar_init();
    }
    if (warp == kMmaWarpS) {
        tc::tmem_alloc(&sh.tmem, kTmemCols);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh.tmem;
    volatile int *abort = &sh.abort;
    const uint8_t *img = simg + (choff[m] - choff[p.mbeg]) * 2 * (int64_t)kSImg;

    if (warp == kMmaWarpS) {
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_f16(128, kLT, 0, 1, 0);
            tc::mbar_arrive_expect_tx(&sh.a_full[0], 2 * kSImg);
            tc::bulk_g2s(sA, img, 2 * kSImg, &sh.a_full[0]);
            for (int64_t cc = 0; cc < nch && !*abort; ++cc) {
                const uint32_t st = (uint32_t)cc & 1, ph = (uint32_t)(cc >> 1) & 1;
                if (!wait_or_abort(&sh.a_full[st], ph, abort, err)) break;
                if (!wait_or_abort(&sh.b_full[st], ph, abort, err)) break;
                tc::tc_fence_after();
                const uint32_t a0 = tc::smem_u32(sA + st * 2 * kSImg);
                const uint32_t b0 = tc::smem_u32(sB + st * 2 * kBTileS);
#pragma unroll
                for (int ks = 0; ks < kKL / 16; ++ks) {
                    const uint64_t ah = tc::desc_sw128_mn(a0 + ks * 4096, 1024, 2048);
                    const uint64_t al = tc::desc_sw128_mn(a0 + kSImg + ks * 4096, 1024, 2048);
                    const uint64_t bh = tc::desc_sw128(b0 + ks * 32);
                    const uint64_t bl = tc::desc_sw128(b0 + kBTileS + ks * 32);
                    // hi*hi into D_hh (columns [0, kLT)), the cross products into D_x
                    // (columns [kLT, 2 kLT)), as in the analysis
                    tc::mma_f16(tmem, ah, bh, idesc, (cc > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_f16(tmem + kLT, ah, bl, idesc, (cc > 0 || ks > 0) ? 1u : 0u);
                    tc::mma_f16(tmem + kLT, al, bh, idesc, 1u);
                }
                tc::mma_commit(&sh.b_free[st]);
                tc::mma_commit(&sh.a_free[st]);
                // with this chunk's MMAs queued, load the next chunk's image into the buffer
                // of the previous chunk once its MMAs are done
                if (cc + 1 < nch) {
                    const uint32_t nb = (uint32_t)(cc + 1) & 1;
                    if (!wait_or_abort(&sh.a_free[nb], ((uint32_t)((cc + 1) >> 1) & 1) ^ 1, abort, err)) break;
                    tc::mbar_arrive_expect_tx(&sh.a_full[nb], 2 * kSImg);
                    tc::bulk_g2s(sA + nb * 2 * kSImg, img + (cc + 1) * 2 * (int64_t)kSImg, 2 * kSImg,
                                 &sh.a_full[nb]);
                }
            }
            if (!*abort) tc::mma_commit(&sh.d_full);
        }
    } else {
        const double sgn_c = sgn_of(p.sp);
        const int64_t mb = alm_idx(p.lmax, 0, m);
        // one lane (northern ring) per generator thread
        const int64_t jl = tile * kLT + tid;
        const bool valid = jl < p.nlanes;
        const double x = valid ? p.geom[jl] : 0.0;
        double v = 0.0, vp = 0.0;
        int k = 0;
        if (valid)
            seed_lane(p.seeds + ((int64_t)p.var * L + m) * 4, p.geom[p.nlanes + jl],
                      p.geom[2 * p.nlanes + jl], v, k);
        bool emit = (k == 0);
        // Coefficients of chunk cc sit in shared stage cc & 1.  Threads tid < kKL load the
        // chunk two ahead into registers while the current one is generated, and publish
        // the next one right after the barrier that frees its stage.
        auto fetch = [&](int64_t ch) -> Coef {
            const int64_t l = (c0 + ch) * kKL + tid;
            return (tid < kKL && ch < nch && l > l0 && l < L) ? load_coef(p.coef, mb + l)
                                                              : Coef{0.0, 0.0, 0.0};
        };
        auto publish = [&](int64_t ch, const Coef &cf) {
            if (tid < kKL) {
                const int64_t so = (ch & 1) * kKL;
                sAB[so + tid] = make_double2(cf.alpha, cf.beta);
                if (SPIN) sC0[so + tid] = sgn_c * cf.c0 * cf.alpha;
            }
        };
        Coef pre = fetch(0);
        publish(0, pre);
        pre = fetch(1);
        bool dead = false;
        for (int64_t cc = 0; cc < nch; ++cc) {
            const uint32_t st = (uint32_t)cc & 1;
            double2 *cab = sAB + st * kKL;
            double *cc0 = sC0 + st * kKL;
            gen_barrier_s();   // stage st is complete; stage st ^ 1 (chunk cc - 1) is free
            // after a timed-out wait a generator keeps meeting the barrier every chunk (the
            // loop is bounded) but does no more work
            if (dead || !wait_or_abort(&sh.b_free[st], ((uint32_t)(cc >> 1) & 1) ^ 1, abort, err)) {
                dead = true;
                continue;
            }
            publish(cc + 1, pre);
            pre = fetch(cc + 2);
            const uint32_t b0 = tc::smem_u32(sB + st * 2 * kBTileS);
#pragma unroll 2
            for (int sub = 0; sub < kKL / 8; ++sub) {
                float vals[8];
                const int64_t lsub = (c0 + cc) * kKL + sub * 8;
                if (lsub > l0) {   // rows past lmax have zero coefficients and emit zeros
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const double2 ab = cab[sub * 8 + e];
                        const double a = SPIN ? fma(ab.x, x, -cc0[sub * 8 + e]) : ab.x * x;
                        const double nv = fma(a, v, -ab.y * vp);
                        vp = v;
                        v = nv;
                        vals[e] = emit ? (float)v : 0.0f;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int64_t l = lsub + e;
                        const double2 ab = cab[sub * 8 + e];
                        const double a = SPIN ? fma(ab.x, x, -cc0[sub * 8 + e]) : ab.x * x;
                        if (l > l0 && l < L) {
                            const double nv = fma(a, v, -ab.y * vp);
                            vp = v;
                            v = nv;
                        }
                        vals[e] = (l >= l0 && l < L && emit) ? (float)v : 0.0f;
                    }
                }
                rescale(v, vp, k);
                emit = (k == 0);
                uint4 hi, lo;
                pack8(vals, hi, lo);
                const uint32_t row = tid;
                const uint32_t off = (row >> 3) * 1024 + (row & 7) * 128 + (((uint32_t)sub ^ (row & 7)) << 4);
                sts128(b0 + off, hi);
                sts128(b0 + kBTileS + off, lo);
            }
            tc::fence_async_smem();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh.b_full[st]);
        }
        // epilogue: D[row, lane] -> synd[m][lane][row]; a warp reads the TMEM lanes
        // 32 (warp % 4) + [0, 32) (rows), the two warpgroups split the columns (lanes)
        if (!dead && wait_or_abort(&sh.d_full, 0, abort, err)) {
            tc::tc_fence_after();
            const int wq = warp & 3, row = wq * 32 + lane;
            const int cbeg = (warp >> 2) * (kLT / 2);
            for (int cb = cbeg; cb < cbeg + kLT / 2; cb += 16) {
                uint32_t r[16], rx[16];
                const uint32_t trow = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)cb;
                tc::tmem_ld16(trow, r);
                tc::tmem_ld16(trow + kLT, rx);
                tc::tmem_ld_wait();
                if (row < R2) {
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const int64_t jl = tile * kLT + cb + e;
                        if (jl < p.nlanes)
                            synd[((m - p.mbeg) * p.nlanes + jl) * R2 + row] =
                                (__uint_as_float(r[e]) + __uint_as_float(rx[e])) * (float)p.scale;
                    }
                }
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarpS) tc::tmem_dealloc(tmem, kTmemCols);
}

// ------------------------------------------------------------------------------- tables

// coef[(mstart[m] + l) * 4 + {0,1,2,3}] = (alpha, beta, c0, 0) of target degree l for s'^2 = s2.
__global__ void k_coef_table(int64_t lmax, int spin, double *__restrict__ tab)
{
    const int64_t m = blockIdx.y;
    const int64_t L = lmax + 1;
    const int64_t l0 = spin == 0 ? m : (m > 2 ? m : 2);
    const double dm = (double)m, ds = (double)spin;
    for (int64_t l = m + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < L;
         l += (int64_t)gridDim.x * blockDim.x) {
        double a = 0.0, b = 0.0, c0 = 0.0;
        if (l > l0) {
            const double dl = (double)l;
            const double den = sqrt((dl * dl - dm * dm) * (dl * dl - ds * ds));
            a = sqrt((2.0 * dl + 1.0) * (2.0 * dl - 1.0)) * dl / den;
            if (l >= l0 + 2) {
                const double dl1 = dl - 1.0;
                const double num = sqrt((dl1 * dl1 - dm * dm) * (dl1 * dl1 - ds * ds));
                b = sqrt((2.0 * dl + 1.0) / (2.0 * dl - 3.0)) * dl * num / (dl1 * den);
            }
            if (spin != 0) c0 = 2.0 * dm / ((dl - 1.0) * dl);
        }
        const int64_t idx = alm_idx(lmax, l, m);
        tab[4 * idx] = a;
        tab[4 * idx + 1] = b;
        tab[4 * idx + 2] = c0;
        tab[4 * idx + 3] = 0.0;
    }
}

// ------------------------------------------------------------------------------- images

// Initial right-hand side from the ring spectra: ringspec (ncomp, nring, L) complex64 ->
// rhs_map (L, nlanes, ncomp) of float4 (G_N re, im, G_S re, im) and the analysis images.
// One CTA per (block of kPackM orders, lane): the north and south ring spectra of the
// block are read along m (coalesced) into shared memory, rhs_map is written along the
// comps, and each image row (thread = row) is written as f16 hi/lo; rows beyond 2H are
// zeroed.  Image a rows: spin 0 [G_N | G_S] x re/im; spin 2 [P_N | M_S]; image b rows
// (spin 2) [M_N | P_S], P = G_Q + i G_U, M = G_Q - i G_U.
constexpr int kPackM = 32;

__device__ __forceinline__ void put_f16(uint8_t *img, uint32_t plane_bytes, float x)
{
    const __half hi = __float2half_rn(x);
    const __half lo = __float2half_rn(x - __half2float(hi));
    *reinterpret_cast<__half *>(img) = hi;
    *reinterpret_cast<__half *>(img + plane_bytes) = lo;
}

// Row value of image variant v (0: a, 1: b) from the comps' (G_N, G_S) of one order.
__device__ __forceinline__ float image_row(const float4 *__restrict__ g, int spin, int H, int r, int v)
{
    if (r >= 2 * H) return 0.0f;
    const bool south = r >= H;
    const int rr = south ? r - H : r;
    const int item = rr >> 1;
    const bool im = rr & 1;
    if (spin == 0) {
        const float4 q = g[item];
        return south ? (im ? q.w : q.z) : (im ? q.y : q.x);
    }
    const float4 q = g[2 * item], u = g[2 * item + 1];
    const float qr = south ? q.z : q.x, qi = south ? q.w : q.y;
    const float ur = south ? u.z : u.x, ui = south ? u.w : u.y;
    const bool plus = (v == 0) ? !south : south;
    return plus ? (im ? qi + ur : qr - ui) : (im ? qi - ur : qr + ui);
}

__global__ void __launch_bounds__(128) k_pack_tc(int64_t nside, int64_t L, int ncomp, int spin,
                                                 const float2 *__restrict__ spec,
                                                 float4 *__restrict__ rhs_map,
                                                 uint8_t *__restrict__ img_a,
                                                 uint8_t *__restrict__ img_b, float scale,
                                                 int64_t mbeg, int64_t mend)
{
    __shared__ float4 tile[kPackM][64];
    const int64_t nlanes = 2 * nside, nring = 4 * nside - 1, NG = (nlanes + kKC - 1) / kKC;
    const int64_t m0 = mbeg + (int64_t)blockIdx.x * kPackM, j = blockIdx.y;
    const int tid = threadIdx.x;
    const bool two = j != nlanes - 1;
    const int64_t rn = north_ring(j), rs = two ? south_ring(nside, j) : 0;
    // spectra of the block: thread -> (hemisphere, order)
    {
        const int hemi = tid / kPackM, mi = tid % kPackM;   // 4 x 32: hemi 0/1 used, 2/3 idle
        const int64_t m = m0 + mi;
        if (hemi < 2) {
            for (int c = 0; c < ncomp; ++c) {
                float2 v = make_float2(0.f, 0.f);
                if (m < mend && (hemi == 0 || two))
                    v = spec[((int64_t)c * nring + (hemi ? rs : rn)) * L + m];
                float *t = reinterpret_cast<float *>(&tile[mi][c]);
                t[2 * hemi] = v.x;
                t[2 * hemi + 1] = v.y;
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < kPackM * ncomp; e += blockDim.x) {
        const int mi = e / ncomp, c = e % ncomp;
        const int64_t m = m0 + mi;
        if (m < mend && rhs_map) rhs_map[(m * nlanes + j) * ncomp + c] = tile[mi][c];
    }
    const int H = spin == 0 ? 2 * ncomp : ncomp;
    const uint32_t roff = tc::sw128_mn_offset(128, (uint32_t)tid, (uint32_t)(j % kKC));
    const int64_t g = j / kKC;
    for (int mi = 0; mi < kPackM; ++mi) {
        const int64_t m = m0 + mi;
        if (m >= mend) break;
        const int64_t base = ((m - mbeg) * NG + g) * 2 * (int64_t)kAImg + roff;
        put_f16(img_a + base, kAImg, image_row(tile[mi], spin, H, tid, 0) * scale);
        if (spin) put_f16(img_b + base, kAImg, image_row(tile[mi], spin, H, tid, 1) * scale);
    }
}

// Synthesis operand images from the interleaved alm (nelem, NR) float64.
// Rows: spin 0 [a | s a] (src row r mod H); spin 2 variant -2 (lambda+): [2a | s -2a]
// (src row r); variant +2 (lambda-): [-2a | s 2a] (src r < H ? H + r : r - H); s = (-1)^(l+m).
// With `rel` set the chunks start at the order's first row instead: chunk cc covers
// l0 + 64 cc + [0, 64) (the layout of the checkpointed synthesis, legendre_ck.cu).
__global__ void k_prep_syn(int64_t lmax, int spin, int sp, int H, int NR,
                           const double *__restrict__ alm_i, const int64_t *__restrict__ choff,
                           uint8_t *__restrict__ simg, double scale, int64_t mbeg, int rel)
{
    const int64_t m = mbeg + blockIdx.y, L = lmax + 1;
    const int l0min = abs(sp);
    const int64_t l0 = m > l0min ? m : l0min;
    if (l0 > lmax) return;
    const int64_t lfirst = rel ? l0 : (l0 / kKL) * kKL;   // first row of chunk 0
    const int64_t nch = (L - lfirst + kKL - 1) / kKL;
    const int64_t mb = alm_idx(lmax, 0, m);
    // thread -> (chunk cc, l within chunk, 8-row group)
    const int64_t per = (int64_t)kKL * 16;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nch * per;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cc = t / per;
        const int kl = (int)((t % per) / 16), r0 = (int)(t % 16) * 8;
        const int64_t l = lfirst + cc * kKL + kl;
        float v[8];
        const bool lok = l >= l0 && l < L;
        const double sgn = ((l + m) & 1) ? -1.0 : 1.0;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int r = r0 + e;
            float val = 0.0f;
            if (lok && r < 2 * H) {
                const bool second = r >= H;
                int src;
                if (spin == 0) src = second ? r - H : r;
                else if (sp < 0) src = r;
                else src = second ? r - H : H + r;
                double a = alm_i[(mb + l) * NR + src] * scale;
                if (second) a *= sgn;
                val = (float)a;
            }
            v[e] = val;
        }
        uint8_t *img = simg + (choff[m] - choff[mbeg] + cc) * 2 * (int64_t)kSImg;
        uint4 hi, lo;
        pack8(v, hi, lo);
        const uint32_t off = tc::sw128_mn_offset(128, (uint32_t)r0, (uint32_t)kl);
        *reinterpret_cast<uint4 *>(img + off) = hi;
        *reinterpret_cast<uint4 *>(img + kSImg + off) = lo;
    }
}

// Ring-fold residual for the batched path: one CTA per lane, one thread per image row.
//
// The synthesis outputs are already in image-row form: spin 0 synd rows [f_N | f_S] x
// re/im are the rows of the analysis image; spin 2 synd_a rows are [P_N | M_S] and synd_b
// rows [M_N | P_S] (with Q_N = (U1 + V1)/2, U_N = i (V1 - U1)/2 one has P_N = U1 and
// M_N = V1, and likewise P_S = V2, M_S = U2), i.e. the rows of analysis image a and b.
// The fold for residue k of the ring length n sums the row over the orders m' = k + t n
// with the sign (-1)^t of a shifted ring, plus the conjugates of the negative orders
// m' = -k + t n, whose value for a real map is the conjugate of the partner row (the same
// row for spin 0; for spin 2 P(-m') = conj M(m'), i.e. the other variant).  Residues k
// and n - k read each other's orders, so they are summed together and every synthesis
// value is read once.  The image of order m = k + t n is then
//   (-1)^t w n P_k - rhs(m), scaled by `scale`, as f16 hi/lo.
// Reads the synthesis and rhs_map once, writes each image row once (coalesced across the
// row threads); rows beyond 2H and the absent south ring of the equator lane keep the
// zeros the pack wrote.
// Occupancy bound per spin (measured at Nside 2048: spin 0 without spills at 16 CTAs per SM,
// 15.0 -> 11.6 ms; spin 2 at 10, 23.9 -> 21.7 ms, where 16 would spill).
template <int SPIN>
__global__ void __launch_bounds__(128, SPIN == 0 ? 16 : 10) k_fold_tc(int64_t nside, int64_t L, int ncomp,
                                                 const float *__restrict__ synd_a,
                                                 const float *__restrict__ synd_b, int R2,
                                                 const float4 *__restrict__ rhs_map,
                                                 const uint8_t *__restrict__ shifted,
                                                 uint8_t *__restrict__ img_a,
                                                 uint8_t *__restrict__ img_b, float scale)
{
    const int64_t j = blockIdx.x;
    const int r = threadIdx.x;
    const int64_t nlanes = 2 * nside, npix = 12 * nside * nside, NG = (nlanes + kKC - 1) / kKC;
    const int n = (int)ring_nphi(nside, north_ring(j));
    const bool sh = shifted[north_ring(j)] != 0;
    const int H = SPIN == 0 ? 2 * ncomp : ncomp;
    const bool south = r >= H;
    if (r >= 2 * H || (south && j == nlanes - 1)) return;
    const float wn = (float)(4.0 * M_PI / (double)npix * (double)n);
    const int rr = south ? r - H : r;
    const int item = rr >> 1;
    const bool im = rr & 1;
    const float cs = im ? -1.0f : 1.0f;                 // conjugation of this row
    const int64_t stride = nlanes * R2;
    const float *pa = synd_a + j * R2 + r;
    const float *pb = (SPIN ? synd_b : synd_a) + j * R2 + r;
    const uint32_t roff = tc::sw128_mn_offset(128, (uint32_t)r, (uint32_t)(j % kKC));
    const int64_t istride = NG * 2 * (int64_t)kAImg;
    uint8_t *ia = img_a + (j / kKC) * 2 * (int64_t)kAImg + roff;
    uint8_t *ib = SPIN ? img_b + (j / kKC) * 2 * (int64_t)kAImg + roff : nullptr;
    const float4 *rb = rhs_map + j * ncomp;

    // rhs of this row at order m for variant v (0: image a, 1: image b)
    auto rhs = [&](int64_t m, int v) -> float {
        const float4 *b = rb + m * nlanes * ncomp;
        if (SPIN == 0) {
            const float4 q = b[item];
            return south ? (im ? q.w : q.z) : (im ? q.y : q.x);
        }
        const float4 q = b[2 * item], u = b[2 * item + 1];
        const float qr = south ? q.z : q.x, qi = south ? q.w : q.y;
        const float ur = south ? u.z : u.x, ui = south ? u.w : u.y;
        // image a rows [P_N | M_S], image b rows [M_N | P_S]; P = Q + iU, M = Q - iU
        const bool plus = (v == 0) ? !south : south;
        return plus ? (im ? qi + ur : qr - ui) : (im ? qi - ur : qr + ui);
    };
    auto put = [&](uint8_t *img, int64_t m, float val) {
        const float x = val * scale;
        const __half hi = __float2half_rn(x);
        const __half lo = __float2half_rn(x - __half2float(hi));
        *reinterpret_cast<__half *>(img + m * istride) = hi;
        *reinterpret_cast<__half *>(img + m * istride + kAImg) = lo;
    };
    // write the images of residue k from its sums (pa_k: variant a, pb_k: variant b)
    auto emit = [&](int k, float sa, float sb) {
        int t = 0;
        for (int64_t m = k; m < L; m += n, ++t) {
            const float f = (sh && (t & 1)) ? -wn : wn;
            put(ia, m, f * sa - rhs(m, 0));
            if (SPIN) put(ib, m, f * sb - rhs(m, 1));
        }
    };
    const float neg = sh ? -1.0f : 1.0f;   // sign of an order read as a negative alias, relative
                                           // to its sign as a positive alias

    if (n >= L) {
        // rings at least as long as lmax + 1 (the belt): order k is its residue's only
        // positive alias and n - k (when below L) its only negative one, so the residue
        // pairs are independent and the loop keeps several loads in flight.  The same
        // sums as the general loop below, in the same order of operations.
        emit(0, pa[0], pb[0]);
#pragma unroll 4
        for (int k = 1; k <= n / 2 && k < L; ++k) {
            const int k2 = n - k;
            const float ak = pa[(int64_t)k * stride], bk = SPIN ? pb[(int64_t)k * stride] : ak;
            if (k2 == k) {
                put(ia, k, wn * (ak + neg * cs * bk) - rhs(k, 0));
                if (SPIN) put(ib, k, wn * (bk + neg * cs * ak) - rhs(k, 1));
            } else if (k2 < L) {
                const float a2 = pa[(int64_t)k2 * stride], b2 = SPIN ? pb[(int64_t)k2 * stride] : a2;
                put(ia, k, wn * (ak + neg * cs * b2) - rhs(k, 0));
                if (SPIN) put(ib, k, wn * (bk + neg * cs * a2) - rhs(k, 1));
                put(ia, k2, wn * (neg * cs * bk + a2) - rhs(k2, 0));
                if (SPIN) put(ib, k2, wn * (neg * cs * ak + b2) - rhs(k2, 1));
            } else {
                put(ia, k, wn * ak - rhs(k, 0));
                if (SPIN) put(ib, k, wn * bk - rhs(k, 1));
            }
        }
        return;
    }

    // residue 0: orders t n (t >= 0), and t n (t >= 1) as negative aliases
    {
        float s0a = 0.f, s0b = 0.f;
        int t = 0;
        for (int64_t mm = 0; mm < L; mm += n, ++t) {
            const float sg = (sh && (t & 1)) ? -1.f : 1.f;
            const float a = pa[mm * stride], b = SPIN ? pb[mm * stride] : a;
            s0a += sg * a;
            if (SPIN) s0b += sg * b;
            if (mm > 0) {
                s0a += sg * cs * b;                 // conj of the partner row
                if (SPIN) s0b += sg * cs * a;
            }
        }
        emit(0, s0a, s0b);
    }
    // residue pairs (k, n - k), 0 < k < n / 2, and the self-paired residue n / 2
    for (int k = 1; 2 * k <= n && k < L; ++k) {
        const int k2 = n - k;
        float pka = 0.f, pkb = 0.f, p2a = 0.f, p2b = 0.f;
        int t = 0;
        for (int64_t mm = k; mm < L; mm += n, ++t) {
            const float sg = (sh && (t & 1)) ? -1.f : 1.f;
            const float a = pa[mm * stride], b = SPIN ? pb[mm * stride] : a;
            pka += sg * a;
            if (SPIN) pkb += sg * b;
            p2a += neg * sg * cs * b;
            if (SPIN) p2b += neg * sg * cs * a;
        }
        if (k2 != k) {
            t = 0;
            for (int64_t mm = k2; mm < L; mm += n, ++t) {
                const float sg = (sh && (t & 1)) ? -1.f : 1.f;
                const float a = pa[mm * stride], b = SPIN ? pb[mm * stride] : a;
                p2a += sg * a;
                if (SPIN) p2b += sg * b;
                pka += neg * sg * cs * b;
                if (SPIN) pkb += neg * sg * cs * a;
            }
            emit(k, pka, pkb);
            if (k2 < L) emit(k2, p2a, p2b);
        } else {
            // k = n / 2: the set is its own partner; p2 holds the conjugate part
            emit(k, pka + p2a, pkb + p2b);
        }
    }
}

// Interleaved alm (nelem, NR) -> API layout (nalm, nelem) complex128 and back.
// Spin 0: rows (map, re/im).  Spin 2: rows [2a (H) | -2a (H)] with
// E = -(2a + -2a)/2, B = i (2a - -2a)/2 per field; to_api = 1 converts to (E, B),
// to_api = 0 converts (E, B) to (2a, -2a) = (-(E + i B), -(E - i B)).
__global__ void k_alm_layout(int64_t nelem, int spin, int nfield, double *__restrict__ alm_i,
                             double *__restrict__ alm_api, int to_api)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nelem) return;
    if (spin == 0) {
        const int NR = 2 * nfield;
        for (int f = 0; f < nfield; ++f) {
            double *a = alm_api + 2 * ((int64_t)f * nelem + idx);
            double *b = alm_i + idx * NR + 2 * f;
            if (to_api) { a[0] = b[0]; a[1] = b[1]; }
            else { b[0] = a[0]; b[1] = a[1]; }
        }
        return;
    }
    const int H = 2 * nfield, NR = 2 * H;
    for (int f = 0; f < nfield; ++f) {
        double *p2 = alm_i + idx * NR + 2 * f;       // 2a
        double *m2 = alm_i + idx * NR + H + 2 * f;   // -2a
        double *e = alm_api + 2 * ((int64_t)(2 * f) * nelem + idx);
        double *b = alm_api + 2 * ((int64_t)(2 * f + 1) * nelem + idx);
        if (to_api) {
            e[0] = -0.5 * (p2[0] + m2[0]);
            e[1] = -0.5 * (p2[1] + m2[1]);
            // i (x + i y) / 2 with x + i y = 2a - -2a
            b[0] = -0.5 * (p2[1] - m2[1]);
            b[1] = 0.5 * (p2[0] - m2[0]);
        } else {
            // 2a = -(E + i B), -2a = -(E - i B)
            p2[0] = -(e[0] - b[1]);
            p2[1] = -(e[1] + b[0]);
            m2[0] = -(e[0] + b[1]);
            m2[1] = -(e[1] - b[0]);
        }
    }
}

// Tensor-core synthesis output -> per-comp ring coefficients in the lane layout
// syn (L, nlanes, ncomp, 4) float [north re, im, south re, im] used by gm_ring_synthesis.
__global__ void k_synd_to_syn(int64_t nlanes, int64_t nm, int ncomp, int spin,
                              const float *__restrict__ synd_a, const float *__restrict__ synd_b,
                              int R2, float *__restrict__ syn, int64_t mbeg)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nm * nlanes * ncomp) return;
    const int c = (int)(idx % ncomp);
    const int64_t ml = idx / ncomp;   // (m - mbeg) * nlanes + lane
    const int H = R2 / 2;
    const float *a = synd_a + ml * R2;
    float4 o;
    if (spin == 0) {
        o = make_float4(a[2 * c], a[2 * c + 1], a[H + 2 * c], a[H + 2 * c + 1]);
    } else {
        const float *b = synd_b + ml * R2;
        const int f = c >> 1;
        const float2 u1 = make_float2(a[2 * f], a[2 * f + 1]), u2 = make_float2(a[H + 2 * f], a[H + 2 * f + 1]);
        const float2 v1 = make_float2(b[2 * f], b[2 * f + 1]), v2 = make_float2(b[H + 2 * f], b[H + 2 * f + 1]);
        if ((c & 1) == 0)
            o = make_float4(0.5f * (u1.x + v1.x), 0.5f * (u1.y + v1.y), 0.5f * (u2.x + v2.x), 0.5f * (u2.y + v2.y));
        else
            o = make_float4(-0.5f * (v1.y - u1.y), 0.5f * (v1.x - u1.x), -0.5f * (u2.y - v2.y), 0.5f * (u2.x - v2.x));
    }
    reinterpret_cast<float4 *>(syn)[mbeg * nlanes * ncomp + idx] = o;
}

}  // namespace ltc
}  // namespace gm

using namespace gm;
using namespace gm::ltc;

extern "C" int64_t gm_tc_lane_groups(int64_t nside) { return (2 * nside + kKC - 1) / kKC; }

extern "C" int64_t gm_tc_ana_image_bytes(int64_t nside, int64_t lmax)
{
    return (lmax + 1) * gm_tc_lane_groups(nside) * 2 * (int64_t)kAImg;
}

extern "C" int64_t gm_tc_ana_scratch_bytes(int64_t nside, int64_t nctas)
{
    return nctas * 2 * nside * 3 * (int64_t)sizeof(double);
}

// Per-order synthesis chunk offsets for spin (|s'|): choff[m], total in choff[L].
extern "C" int gm_tc_syn_chunk_offsets(int64_t lmax, int spin, int64_t *choff_host)
{
    if (lmax < 0 || !choff_host) return GM_ERR_BAD_SHAPE;
    const int64_t L = lmax + 1;
    int64_t acc = 0;
    for (int64_t m = 0; m < L; ++m) {
        choff_host[m] = acc;
        const int64_t l0 = spin == 0 ? m : (m > 2 ? m : 2);
        if (l0 <= lmax) acc += (L + kKL - 1) / kKL - l0 / kKL;
    }
    choff_host[L] = acc;
    return GM_OK;
}

extern "C" int64_t gm_tc_syn_image_bytes(int64_t nchunks) { return nchunks * 2 * (int64_t)kSImg; }

extern "C" int gm_tc_coef_table(int64_t lmax, int spin, double *tab, void *stream)
{
    if (lmax < 0 || lmax > 65535 || (spin != 0 && spin != 2)) return GM_ERR_BAD_SHAPE;
    if (!tab) return GM_ERR_BAD_PTR;
    k_coef_table<<<dim3(8, (unsigned)(lmax + 1)), 256, 0, as_stream(stream)>>>(lmax, spin, tab);
    return check_launch("gm_tc_coef_table");
}

static int tc_shape_ok(int spin, int64_t ncomp)
{
    if (spin == 0) return ncomp >= 1 && ncomp <= 32;
    if (spin == 2) return ncomp >= 2 && ncomp <= 64 && ncomp % 2 == 0;
    return 0;
}

static bool window_ok(int64_t lmax, int64_t mbeg, int64_t mend)
{
    return mbeg >= 0 && mbeg < mend && mend <= lmax + 1;
}

extern "C" int gm_tc_pack_window(int64_t nside, int64_t lmax, int spin, int64_t ncomp,
                                 const void *ringspec, void *rhs_map, void *img_a, void *img_b,
                                 double img_scale, int64_t mbeg, int64_t mend, void *stream)
{
    if (nside < 1 || lmax < 0 || !tc_shape_ok(spin, ncomp) || !(img_scale > 0.0) ||
        !window_ok(lmax, mbeg, mend))
        return GM_ERR_BAD_SHAPE;
    if (!ringspec || !img_a || (spin && !img_b)) return GM_ERR_BAD_PTR;
    const int64_t NG = gm_tc_lane_groups(nside);
    cudaStream_t s = as_stream(stream);
    // the kernel writes every row of every lane; only the padding lanes of a last, partial
    // group (nside not a multiple of 64) need clearing
    if (NG * kKC != 2 * nside) {
        const size_t bytes = (size_t)(mend - mbeg) * NG * 2 * kAImg;
        if (cudaMemsetAsync(img_a, 0, bytes, s) != cudaSuccess ||
            (spin && cudaMemsetAsync(img_b, 0, bytes, s) != cudaSuccess)) {
            set_error("gm_tc_pack memset", cudaGetLastError());
            return GM_ERR_LAUNCH;
        }
    }
    dim3 grid((unsigned)((mend - mbeg + kPackM - 1) / kPackM), (unsigned)(2 * nside));
    k_pack_tc<<<grid, 128, 0, s>>>(nside, lmax + 1, (int)ncomp, spin, (const float2 *)ringspec,
                                   (float4 *)rhs_map, (uint8_t *)img_a, (uint8_t *)img_b,
                                   (float)img_scale, mbeg, mend);
    return check_launch("gm_tc_pack");
}

extern "C" int gm_tc_pack(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const void *ringspec,
                          void *rhs_map, void *img_a, void *img_b, double img_scale, void *stream)
{
    if (!rhs_map) return GM_ERR_BAD_PTR;
    return gm_tc_pack_window(nside, lmax, spin, ncomp, ringspec, rhs_map, img_a, img_b, img_scale, 0,
                             lmax + 1, stream);
}

static Params make_params(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                          const double *geom, const double *seeds, const double *coef, double scale)
{
    Params p;
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
    p.seeds = seeds;
    p.coef = coef;
    p.var = sp == 0 ? 0 : (sp < 0 ? 1 : 2);
    p.mbeg = 0;
    p.mend = lmax + 1;
    return p;
}

extern "C" int gm_tc_analysis_window(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                                     const double *geom, const double *seeds, const double *coef,
                                     const void *img, double *alm_i, double scale, double *scratch,
                                     int64_t nctas, int64_t mbeg, int64_t mend, int32_t *err,
                                     void *stream)
{
    if (nside < 1 || lmax < 2 || !tc_shape_ok(spin, ncomp) || nctas < 1 || nctas > 4096 ||
        !window_ok(lmax, mbeg, mend))
        return GM_ERR_BAD_SHAPE;
    if ((spin == 0) != (sp == 0) || (spin == 2 && sp != 2 && sp != -2)) return GM_ERR_BAD_SHAPE;
    if (!geom || !seeds || !coef || !img || !alm_i || !scratch || !err) return GM_ERR_BAD_PTR;
    const size_t smem = 2 * kAImg + 4 * kBTileA + kSB * (sizeof(double2) + sizeof(double)) + 1024;
    auto kern = spin == 0 ? k_ana_tc<0> : k_ana_tc<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_error("gm_tc_analysis attr", e);
        return GM_ERR_LAUNCH;
    }
    Params p = make_params(nside, lmax, spin, sp, ncomp, geom, seeds, coef, scale);
    p.mbeg = mbeg;
    p.mend = mend;
    kern<<<(unsigned)nctas, kThreads, smem, as_stream(stream)>>>(p, (const uint8_t *)img, alm_i,
                                                                scratch, (int *)err);
    return check_launch("gm_tc_analysis");
}

extern "C" int gm_tc_analysis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                              const double *geom, const double *seeds, const double *coef,
                              const void *img, double *alm_i, double scale, double *scratch,
                              int64_t nctas, int32_t *err, void *stream)
{
    return gm_tc_analysis_window(nside, lmax, spin, sp, ncomp, geom, seeds, coef, img, alm_i, scale,
                                 scratch, nctas, 0, lmax + 1, err, stream);
}

extern "C" int gm_tc_prep_syn_window(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                                     const int64_t *choff, void *simg, int64_t simg_bytes,
                                     double alm_scale, int64_t mbeg, int64_t mend, void *stream)
{
    if (lmax < 2 || !tc_shape_ok(spin, ncomp) || !(alm_scale > 0.0) || !window_ok(lmax, mbeg, mend))
        return GM_ERR_BAD_SHAPE;
    if (!alm_i || !choff || !simg) return GM_ERR_BAD_PTR;
    const int H = spin == 0 ? (int)(2 * ncomp) : (int)ncomp;
    const int NR = spin == 0 ? H : 2 * H;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(simg, 0, (size_t)simg_bytes, s);
    if (e != cudaSuccess) {
        set_error("gm_tc_prep_syn memset", e);
        return GM_ERR_LAUNCH;
    }
    k_prep_syn<<<dim3(16, (unsigned)(mend - mbeg)), 256, 0, s>>>(lmax, spin, sp, H, NR, alm_i, choff,
                                                                (uint8_t *)simg, alm_scale, mbeg, 0);
    return check_launch("gm_tc_prep_syn");
}

extern "C" int gm_ck_prep_syn(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                              const int64_t *choff, void *simg, int64_t simg_bytes, double alm_scale,
                              void *stream)
{
    if (lmax < 2 || !tc_shape_ok(spin, ncomp) || !(alm_scale > 0.0)) return GM_ERR_BAD_SHAPE;
    if ((spin == 0) != (sp == 0) || (spin == 2 && sp != 2 && sp != -2)) return GM_ERR_BAD_SHAPE;
    if (!alm_i || !choff || !simg) return GM_ERR_BAD_PTR;
    const int H = spin == 0 ? (int)(2 * ncomp) : (int)ncomp;
    const int NR = spin == 0 ? H : 2 * H;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(simg, 0, (size_t)simg_bytes, s);
    if (e != cudaSuccess) {
        set_error("gm_ck_prep_syn memset", e);
        return GM_ERR_LAUNCH;
    }
    k_prep_syn<<<dim3(16, (unsigned)(lmax + 1)), 256, 0, s>>>(lmax, spin, sp, H, NR, alm_i, choff,
                                                              (uint8_t *)simg, alm_scale, 0, 1);
    return check_launch("gm_ck_prep_syn");
}

extern "C" int gm_tc_prep_syn(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                              const int64_t *choff, void *simg, int64_t simg_bytes, double alm_scale,
                              void *stream)
{
    return gm_tc_prep_syn_window(lmax, spin, sp, ncomp, alm_i, choff, simg, simg_bytes, alm_scale, 0,
                                 lmax + 1, stream);
}

extern "C" int gm_tc_synthesis_window(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                                      const double *geom, const double *seeds, const double *coef,
                                      const void *simg, const int64_t *choff, float *synd,
                                      double out_scale, int64_t mbeg, int64_t mend, int32_t *err,
                                      void *stream)
{
    if (nside < 1 || lmax < 2 || !tc_shape_ok(spin, ncomp) || !(out_scale > 0.0) ||
        !window_ok(lmax, mbeg, mend))
        return GM_ERR_BAD_SHAPE;
    if ((spin == 0) != (sp == 0) || (spin == 2 && sp != 2 && sp != -2)) return GM_ERR_BAD_SHAPE;
    if (!geom || !seeds || !coef || !simg || !choff || !synd || !err) return GM_ERR_BAD_PTR;
    const size_t smem = 4 * kSImg + 4 * kBTileS + 2 * kKL * (sizeof(double2) + sizeof(double)) + 1024;
    auto kern = spin == 0 ? k_syn_tc<0> : k_syn_tc<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
        set_error("gm_tc_synthesis attr", e);
        return GM_ERR_LAUNCH;
    }
    Params p = make_params(nside, lmax, spin, sp, ncomp, geom, seeds, coef, out_scale);
    p.mbeg = mbeg;
    p.mend = mend;
    const int R2 = 2 * p.H;
    dim3 grid((unsigned)((p.nlanes + kLT - 1) / kLT), (unsigned)(mend - mbeg));
    kern<<<grid, kThreadsS, smem, as_stream(stream)>>>(p, (const uint8_t *)simg, choff, synd, R2,
                                                     (int *)err);
    return check_launch("gm_tc_synthesis");
}

extern "C" int gm_tc_synthesis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                               const double *geom, const double *seeds, const double *coef,
                               const void *simg, const int64_t *choff, float *synd, double out_scale,
                               int32_t *err, void *stream)
{
    return gm_tc_synthesis_window(nside, lmax, spin, sp, ncomp, geom, seeds, coef, simg, choff, synd,
                                  out_scale, 0, lmax + 1, err, stream);
}

extern "C" int gm_tc_fold(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const float *synd_a,
                          const float *synd_b, const void *rhs_map, const uint8_t *shifted,
                          void *img_a, void *img_b, double img_scale, void *stream)
{
    if (nside < 1 || lmax < 2 || !tc_shape_ok(spin, ncomp) || !(img_scale > 0.0)) return GM_ERR_BAD_SHAPE;
    if (!synd_a || (spin && !synd_b) || !rhs_map || !shifted || !img_a || (spin && !img_b))
        return GM_ERR_BAD_PTR;
    const int H = spin == 0 ? (int)(2 * ncomp) : (int)ncomp;
    auto kern = spin == 0 ? k_fold_tc<0> : k_fold_tc<2>;
    kern<<<(unsigned)(2 * nside), 128, 0, as_stream(stream)>>>(
        nside, lmax + 1, (int)ncomp, synd_a, synd_b, 2 * H, (const float4 *)rhs_map, shifted,
        (uint8_t *)img_a, (uint8_t *)img_b, (float)img_scale);
    return check_launch("gm_tc_fold");
}

extern "C" int gm_tc_alm_layout(int64_t lmax, int spin, int64_t nfield, double *alm_i,
                                double *alm_api, int to_api, void *stream)
{
    if (lmax < 0 || nfield < 1 || nfield > 64 || (spin != 0 && spin != 2)) return GM_ERR_BAD_SHAPE;
    if (!alm_i || !alm_api) return GM_ERR_BAD_PTR;
    const int64_t nelem = (lmax + 1) * (lmax + 2) / 2;
    k_alm_layout<<<(unsigned)((nelem + 255) / 256), 256, 0, as_stream(stream)>>>(
        nelem, spin, (int)nfield, alm_i, alm_api, to_api);
    return check_launch("gm_tc_alm_layout");
}

extern "C" int gm_tc_synd_to_syn_window(int64_t nside, int64_t lmax, int spin, int64_t ncomp,
                                        const float *synd_a, const float *synd_b, float *syn,
                                        int64_t mbeg, int64_t mend, void *stream)
{
    if (nside < 1 || lmax < 2 || !tc_shape_ok(spin, ncomp) || !window_ok(lmax, mbeg, mend))
        return GM_ERR_BAD_SHAPE;
    if (!synd_a || (spin && !synd_b) || !syn) return GM_ERR_BAD_PTR;
    const int H = spin == 0 ? (int)(2 * ncomp) : (int)ncomp;
    const int64_t tot = (mend - mbeg) * 2 * nside * ncomp;
    k_synd_to_syn<<<(unsigned)((tot + 255) / 256), 256, 0, as_stream(stream)>>>(
        2 * nside, mend - mbeg, (int)ncomp, spin, synd_a, synd_b, 2 * H, syn, mbeg);
    return check_launch("gm_tc_synd_to_syn");
}

extern "C" int gm_tc_synd_to_syn(int64_t nside, int64_t lmax, int spin, int64_t ncomp,
                                 const float *synd_a, const float *synd_b, float *syn, void *stream)
{
    return gm_tc_synd_to_syn_window(nside, lmax, spin, ncomp, synd_a, synd_b, syn, 0, lmax + 1, stream);
}

// ------------------------------------------------------------------ allocation-free variant
//
// gm_tc_analysis_noalloc is gm_tc_analysis for callers that cannot call cudaMalloc (see
// include/gm_b200.h).  Its recurrence-state scratch is this file-scope device array
// instead of a caller buffer: up to kNoAllocLaneSlots (CTA, lane) slots of 3 doubles,
// 148 CTAs x 4096 lanes (Nside 2048 on every SM of a B200), 14.5 MB, held by every GPU
// that loads the library until the process exits.  The kernel writes each slot before
// reading it, so no clearing is needed; the array keeps the last call's contents, and
// calls that overlap on the GPU race on it.
namespace gm {
namespace ltc {

constexpr int64_t kNoAllocLaneSlots = 148 * 4096;
static __device__ __align__(256) double g_ana_state[kNoAllocLaneSlots * 3];

// Device address of g_ana_state, looked up once per device with that device current and
// kept for the life of the process.  The cached address belongs to the device's context at
// the time of the lookup: it does not survive cudaDeviceReset (or any teardown of that
// context), after which this entry point must not be called again in the same process.
static double *noalloc_state_ptr(int dev, cudaError_t &err)
{
    static std::mutex mu;
    static double *ptrs[64] = {nullptr};
    err = cudaSuccess;
    if (dev < 0 || dev >= 64) {
        err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptrs[dev]) {
        void *p = nullptr;
        err = cudaGetSymbolAddress(&p, g_ana_state);
        if (err != cudaSuccess) return nullptr;
        ptrs[dev] = static_cast<double *>(p);
    }
    return ptrs[dev];
}

}  // namespace ltc
}  // namespace gm

extern "C" int gm_tc_analysis_noalloc(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                                      const double *geom, const double *seeds, const double *coef,
                                      const void *img, double *alm_i, double scale, int64_t nctas,
                                      int32_t *err, void *stream)
{
    // compared by division so that no product of caller values can wrap around
    if (nside < 1 || nctas < 1 || nctas > gm::ltc::kNoAllocLaneSlots ||
        nside > gm::ltc::kNoAllocLaneSlots / (2 * nctas)) {
        gm::set_error_msg("gm_tc_analysis_noalloc: nctas * 2 * nside exceeds the 606208 lane slots "
                          "of the static scratch (e.g. at most 148 CTAs at Nside 2048)");
        return GM_ERR_BAD_SHAPE;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        gm::set_error("gm_tc_analysis_noalloc cudaGetDevice", e);
        return GM_ERR_LAUNCH;
    }
    double *state = gm::ltc::noalloc_state_ptr(dev, e);
    if (!state) {
        gm::set_error("gm_tc_analysis_noalloc cudaGetSymbolAddress", e);
        return GM_ERR_LAUNCH;
    }
    return gm_tc_analysis(nside, lmax, spin, sp, ncomp, geom, seeds, coef, img, alm_i, scale, state,
                          nctas, err, stream);
}
