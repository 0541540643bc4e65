/*
 * gm_b200.h -- C ABI of the B200-native pseudo-C_ell MASTER hot path.
 *
 * Every entry point takes caller-owned device pointers (plain pointers and sizes,
 * no framework types), launches on the caller's CUDA stream, allocates nothing and
 * returns a gm_status.  Scratch is always a caller-provided buffer whose size is
 * given by the matching *_workspace_bytes / size query.  No entry point
 * synchronises the stream except where stated.
 *
 * Each declaration names the reference (licongxu/GMaster) interface it replaces.
 * The reference binds its kernels as XLA FFI handlers (the .cu files under
 * gmaster/_native/cuda) or lowers the step to XLA library calls (cuFFT, cuBLAS, cuSOLVER,
 * segment_sum); a jax.ffi handler or a ctypes binding calls these entry points directly.
 *
 * Data layouts (all row-major, complex values interleaved re/im):
 *   maps      (ncomp, npix)                  float64 or float32, HEALPix RING order
 *   ringspec  (ncomp, nring, L)              complex, G_r(m) = w e^{-i m phi0_r} DFT_r[m mod nphi_r]
 *   rhs       (L, nlanes, ncomp, 4)          real, per north lane j: [Sum re, Sum im, Diff re, Diff im]
 *                                            with Sum/Diff = G_north(m) +- G_south(m)
 *   syn       (L, nlanes, ncomp, 4)          real, per lane: [north re, north im, south re, south im]
 *   alm       (nalm, nelem)                  complex128, healpy m-major packing
 *   lanes     nlanes = 2 nside (north rings 1..2nside; the last is the equator)
 * ncomp counts real map components: spin 0 -> one per map, spin 2 -> (Q, U) per field.
 */
#ifndef GM_B200_H
#define GM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GM_OK = 0,
    GM_ERR_BAD_SHAPE = 1,   /* sizes inconsistent or out of the supported range */
    GM_ERR_BAD_PTR = 2,     /* a required pointer is null or misaligned */
    GM_ERR_LAUNCH = 3,      /* a kernel launch failed (cudaGetLastError) */
    GM_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    GM_ERR_UNSUPPORTED = 5  /* precision / spin / option not implemented */
} gm_status;

typedef enum { GM_FP64 = 0, GM_MIXED = 1 } gm_precision;

/* Last CUDA error string recorded by a failing call on this thread. */
const char *gm_last_error(void);

/* Library version string. */
const char *gm_version(void);

/* ---------------------------------------------------------------- ring stage */

/* Number of twiddle entries for all ring lengths of `nside`
 * (sum over i in [1, nside] of 2i = nside (nside + 1)).  The table buffer holds that
 * many complex128 entries followed by the same entries as complex64
 * (24 bytes per entry in total). */
int64_t gm_ring_twiddle_count(int64_t nside);

/* Fill the twiddle table: tw[i(i-1) + k] = exp(-2 pi i k / (4 i)), k < 2i (both copies).
 * `shifted` arguments below are one byte per ring: 1 where phi0 = pi / nphi, 0 where
 * phi0 = 0 (the only two HEALPix cases, utils.py:237-243).
 * Replaces the chirp-Z constant tables of gmaster/_sht/rings.py:198-248. */
int gm_ring_twiddles(int64_t nside, void *tw, void *stream);

/* Forward ring transform of real maps (replaces rings.py:251-299
 * `_forward_ring_fft_positive`, the XLA cuFFT belt FFT + Bluestein caps).
 * maps: (ncomp, npix) with `map_dtype_bytes` 8 (float64) or 4 (float32).
 * mask: NULL, or (npix) float64 multiplied into every map as it is read (the masking of
 * gmaster/field.py:219-229 without a masked copy of the maps; the FP64 product is
 * rounded once, as for a pre-masked map).
 * out ringspec: (ncomp, nring, L) complex128 (GM_FP64) or complex64 (GM_MIXED),
 * including the quadrature weight 4 pi / npix and the phase e^{-i m phi0}. */
int gm_ring_analysis(int precision, int64_t nside, int64_t L, int64_t ncomp,
                     const void *maps, int map_dtype_bytes, const double *mask,
                     const void *tw, const uint8_t *shifted, void *ringspec, void *stream);

/* Hemisphere pack of a ring spectrum into the lane-major Legendre right-hand side
 * (replaces march_v2.py:637-663 `_fold_rhs`).  rhs (L, nlanes, ncomp, 4). */
int gm_pack_rhs(int precision, int64_t nside, int64_t L, int64_t ncomp,
                const void *ringspec, void *rhs, void *stream);

/* Ring-fold residual in lane space (replaces march_v2.cu:426-493
 * `ring_fold_residual` + march_v2.py:614-633): for every lane and order m,
 *   rhs_out = pack( w nphi e^{-i m phi0} sum_{m' = m mod nphi, |m'| < L} c(m') e^{i m' phi0} )
 *             - rhs_map
 * where c comes from `syn` (c(-m') = conj c(m')).  This is the analysis-side ring
 * spectrum of the map synthesised from `syn`, minus the input map's, without any FFT. */
int gm_fold_residual(int precision, int64_t nside, int64_t L, int64_t ncomp,
                     const void *syn, const void *rhs_map, const uint8_t *shifted,
                     void *rhs_out, void *stream);

/* Inverse ring transform (replaces rings.py:477-524 `_inverse_ring_fft_herm` and
 * healpix.py:462-471): maps[c][p] = sum_{|m| < L} c_r(m) e^{i m phi_p} with the
 * per-lane coefficients in `syn`.  maps written as float64. */
int gm_ring_synthesis(int precision, int64_t nside, int64_t L, int64_t ncomp,
                      const void *syn, const void *tw, const uint8_t *shifted,
                      double *maps, void *stream);

/* The two ring stages above with a global scratch for the rings that do not fit the
 * shared-memory kernels (single precision only; NULL scratch gives the entries above):
 * belt rings above Nside 7232, whose ping-pong buffers exceed 226 KB, and rings needing
 * Bluestein's method longer than 8192 points (a prime factor above 64, h > 4096).
 * Persistent CTAs, one per scratch slot of gm_ring_big_scratch_bytes(nside, 1) bytes,
 * walk those rings.  hcap_max > 0 lowers the largest half-length kept in shared memory
 * and bs_min > 0 the Bluestein length above which the global path takes a ring (0:
 * defaults; small values route small rings through the global path, for testing).
 * Same reference interfaces (rings.py:251-299, 477-524). */
int64_t gm_ring_big_scratch_bytes(int64_t nside, int64_t nslots);
int gm_ring_analysis_ws(int precision, int64_t nside, int64_t L, int64_t ncomp, const void *maps,
                        int map_dtype_bytes, const double *mask, const void *tw,
                        const uint8_t *shifted, void *ringspec, void *scratch,
                        int64_t scratch_bytes, int64_t hcap_max, int64_t bs_min, void *stream);
int gm_ring_synthesis_ws(int precision, int64_t nside, int64_t L, int64_t ncomp, const void *syn,
                         const void *tw, const uint8_t *shifted, double *maps, void *scratch,
                         int64_t scratch_bytes, int64_t hcap_max, int64_t bs_min, void *stream);

/* ----------------------------------------------------------- Legendre stage */

/* Seed table length (doubles): 17 variants x L orders x 4.  Variant 0 is spin 0; spin
 * s in 1..8 has two consecutive variants (s' = -s, then s' = +s times (-1)^s) starting at
 * 1 for spin 2, 3 for spin 1 and 2s - 1 for s >= 3 (gmaster_b200/sht.py:seed_table). */
int64_t gm_seed_table_len(int64_t L);

/* Spherical-harmonic analysis, latitudinal step (replaces march_v2.cu:155-285
 * `march_analysis` via march_v2.py:666-693 and 817-872):
 *   alm[f][idx(l,m)] += scale * sum_lanes lambda_lm(theta_j) rhs(...)
 * spin 0: ncomp maps -> nalm = ncomp rows; spin s in 1..8: ncomp = 2 nfields ->
 * nalm = 2 nfields rows (E, B per field, healpix.py:800-814); other spins return
 * GM_ERR_UNSUPPORTED.
 * lane_geom: (3, nlanes) float64 [cos theta, log2 sin(theta/2), log2 cos(theta/2)].
 * seeds: gm_seed_table_len(L) doubles (see gmaster_b200/sht.py).
 * alm is accumulated with double-precision atomics: zero it first for a fresh analysis. */
int gm_legendre_analysis(int precision, int spin, int64_t nside, int64_t lmax,
                         int64_t ncomp, const double *lane_geom, const double *seeds,
                         const void *rhs, double *alm, double scale, void *stream);

/* Synthesis, latitudinal step (replaces march_v2.cu:291-407 `march_synthesis` via
 * march_v2.py:752-795 and 886-924): syn(m, lane, comp) from alm. */
int gm_legendre_synthesis(int precision, int spin, int64_t nside, int64_t lmax,
                          int64_t ncomp, const double *lane_geom, const double *seeds,
                          const double *alm, void *syn, void *stream);

/* Tile shapes of the two entries above, for the autotuner (gmaster_b200/autotune.py):
 * gm_legendre_tiles writes up to `capacity` pairs (NC, R) = (components per CTA, lanes
 * per thread) of `spin` into nc_r and returns their number (-1 for another spin).  The
 * _tile entries run tile `tile` of that list (-1: the built-in choice).  The reference
 * picks its march tiles by fixed rules (march_v2.py:290-332); it has no tuner. */
int gm_legendre_tiles(int spin, int32_t *nc_r, int capacity);
int gm_legendre_analysis_tile(int precision, int spin, int64_t nside, int64_t lmax,
                              int64_t ncomp, const double *lane_geom, const double *seeds,
                              const void *rhs, double *alm, double scale, int tile, void *stream);
int gm_legendre_synthesis_tile(int precision, int spin, int64_t nside, int64_t lmax,
                               int64_t ncomp, const double *lane_geom, const double *seeds,
                               const double *alm, void *syn, int tile, void *stream);

/* ------------------------------------------------------------- spectra */

/* Coupled pseudo-C_ell of all component pairs (replaces workspaces.py:86-95
 * `_compute_coupled_cell`): cls[(i n2 + j) (lmax+1) + l].  The sum over orders runs in a
 * fixed order: equal inputs give bit-equal spectra. */
int gm_pseudo_cl(int64_t lmax, int64_t n1, const double *alm1, int64_t n2,
                 const double *alm2, double *cls, void *stream);

/* Coupling blocks by the Wigner-3j three-term recursion in l3 (replaces
 * workspaces.py:352-517 `_coupling_matrix_tt` and 682-924 `_general_coupling_matrix`
 * / `_coupling_matrices_spin2`, and coupling_tt.cu:18-45):
 *   S_x[l1][l2] = sum_l3 (2 l3 + 1) W_l3 / (4 pi) * T_x(l1, l2, l3)
 *   with T_tt = (l1 l2 l3;000)^2, T_te = (000)(2 -2 0) (even J),
 *   T_pp = (2 -2 0)^2 (even J), T_mm = (2 -2 0)^2 (odd J),
 *   blocks[x][l1][l2] = (2 l2 + 1) S_x[l1][l2]; `which` is a bit mask
 *   (1 tt, 2 te, 4 pp, 8 mm); blocks is (4, lmax+1, lmax+1) float64.
 * window has nw entries (entries beyond nw are zero).
 * Persistent kernel with a device work queue: `queue` is one int64 the kernel uses as
 * its counter (zeroed by this call). */
int gm_coupling_blocks(int64_t lmax, const double *window, int64_t nw, int which,
                       double *blocks, int64_t *queue, void *stream);

/* Work units of gm_coupling_blocks for one lmax (a unit is one l1 and 32 consecutive l2). */
int64_t gm_coupling_units(int64_t lmax);

/* Coupling blocks of many workspaces of different lmax in one persistent launch (the
 * uneven-workspace batch; the reference builds each workspace separately,
 * workspaces.py:1760-1912).  Job j is the row jobs[6j .. 6j+5] of a device int64 table:
 * (lmax, offset of its window in `windows`, nw, which, offset of its (4, lmax+1, lmax+1)
 * blocks in `blocks`, index of its first unit); units number consecutively over the jobs
 * (gm_coupling_units(lmax_j) each, nunits in total).  Order the jobs by decreasing lmax so
 * the longest recursions start first.  The caller zeroes `blocks`; `queue` is one int64
 * the kernel uses as its counter (zeroed by this call). */
int gm_coupling_blocks_multi(int64_t njobs, const int64_t *jobs, int64_t nunits,
                             const double *windows, double *blocks, int64_t *queue, void *stream);

/* Scalar coupling sums S_tt(l1, l2) = sum_l3 (2 l3 + 1) W_l3 / (4 pi) (l1 l2 l3; 000)^2 of
 * an explicit list of npairs (l1, l2) pairs (int32 pairs), written symmetrically into the
 * dense (lmax+1)^2 float64 matrix S; unlisted entries are left untouched.  Computes only
 * the entries the Toeplitz approximation reads (replaces workspaces.py:546-590
 * `_coupling_matrix_tt_toeplitz`, with the pair set of :521-538). */
int gm_coupling_pairs_tt(int64_t lmax, const double *window, int64_t nw, const int32_t *pairs,
                         int64_t npairs, double *S, void *stream);

/* Toeplitz approximation of the scalar coupling matrix (replaces workspaces.py:1141-1194
 * `_apply_toeplitz`, NaMaster's Louis et al. 2020 scheme): from S holding the exact entries
 * on the diagonal, in column l_toeplitz, in columns 0..l_exact and on the dl_band
 * sub-diagonals, writes the full symmetric approximation times (2 l' + 1), i.e. the TT
 * coupling block, into out ((lmax+1)^2 float64).  Requires 0 <= l_exact <= l_toeplitz < lmax
 * and 0 <= dl_band < lmax. */
int gm_toeplitz_fill(int64_t lmax, int64_t l_toeplitz, int64_t l_exact, int64_t dl_band,
                     const double *S, double *out, void *stream);

/* Binned coupling matrix B M diag(beam) T for ncls in {1, 2, 4} (replaces
 * workspaces.py:1570-1590 `_banded_operators` and :292-310 `_BlockMCM.banded`).
 * The binning is given in CSR form: band b holds multipoles band_ells[band_ptr[b] ..
 * band_ptr[b+1]); wfl (lmax+1) = weight * f_ell, inv_fl (lmax+1) = 1 / f_ell,
 * beam (lmax+1) = beam1 * beam2.  blocks is the (4, lmax+1, lmax+1) output of
 * gm_coupling_blocks.  scratch holds 2 nbands^2 doubles.  out is (ncls nb)^2 float64 in
 * band-major, channel-minor order with the reference's block slots and signs
 * (workspaces.py:1856-1912). */
int gm_bin_coupling_csr(int64_t lmax, int64_t nbands, int ncls, const double *blocks,
                        const int32_t *band_ptr, const int32_t *band_ells, const double *wfl,
                        const double *inv_fl, const double *beam, double *scratch, double *out,
                        void *stream);

/* Bin spectra: out[c][b] = sum_{l in b} wfl[l] cls[c][l] (bins.py:15-20). */
int gm_bin_cells_csr(int64_t lmax, int64_t nbands, int64_t ncls, const double *cls,
                     const int32_t *band_ptr, const int32_t *band_ells, const double *wfl,
                     double *out, void *stream);

/* In-place LU factorisation with partial pivoting of an n x n float64 matrix and
 * solve of nrhs right-hand sides (replaces the cuSOLVER getrf/getrs behind
 * jnp.linalg.solve, workspaces.py:2146).  piv: n int32.  status: one int32 set to
 * 0 on success or k+1 when the k-th pivot is exactly zero. */
int gm_lu_factor(int64_t n, double *a, int32_t *piv, int32_t *status, void *stream);
/* Blocked form of gm_lu_factor (same factors, pivots and status; the caller zeroes
 * `status`): for each panel [k0, k1): gm_lu_panel (pivoting and factoring the panel's
 * columns, whole-row swaps), gm_lu_trsm (the U rows right of the panel), then
 * gm_lu_update (A[k1:, k1:] -= A[k1:, k0:k1] A[k0:k1, k1:]).  Replaces the reference's
 * jnp.linalg.solve factorisation (workspaces.py:2146) for large binned matrices. */
int gm_lu_panel(int64_t n, double *a, int64_t k0, int64_t k1, int32_t *piv, int32_t *status,
                void *stream);
int gm_lu_trsm(int64_t n, double *a, int64_t k0, int64_t k1, void *stream);
/* Blocked LU trailing update after panel [k0, k1) (k1 - k0 <= 64): a[i][j] -= sum_k
 * a[i][k] a[k][j] over k in [k0, k1), for i, j >= k1, in FP64 (64 x 64 tiles). */
int gm_lu_update(int64_t n, double *a, int64_t k0, int64_t k1, void *stream);
int gm_lu_solve(int64_t n, const double *lu, const int32_t *piv, int64_t nrhs,
                double *b, void *stream);

/* ----------------------------------------------- batched tensor-core Legendre stage */

/* Batched transforms on tcgen05 (replace march_v2.cu:155-407 for many maps per launch).
 * A batch holds up to 128 real right-hand-side rows: spin 0, ncomp <= 32 maps (rows
 * [G_north | G_south] x re/im); spin 2, ncomp = 2F <= 64 (Q, U of F fields; two row
 * variants s' = -2 with rows [P_N | M_S] and s' = +2 with rows [M_N | P_S], P = G_Q + i G_U,
 * M = G_Q - i G_U).  Operand images are f16 hi/lo planes (22 significant bits; the
 * products run as three kind::f16 MMAs, hi*hi + hi*lo + lo*hi, accumulating in FP32) in
 * the 128-byte-swizzled MN-major layout of gm_tc_selftest.  Right-hand-side and alm
 * images carry a caller-chosen power-of-two scale (img_scale, alm_scale) that puts their
 * largest entry near 2^13, inside the f16 range; the analysis `scale` and the synthesis
 * `out_scale` undo it.  The interleaved alm alm_i is (nelem, NR) float64
 * with NR = 2 ncomp (spin 0: map x re/im) or 2 ncomp (spin 2: [a_{+2} | a_{-2}] x re/im). */

/* Lane groups of 128 lanes and analysis image bytes ((lmax+1) x groups x 64 KB). */
int64_t gm_tc_lane_groups(int64_t nside);
int64_t gm_tc_ana_image_bytes(int64_t nside, int64_t lmax);
/* Scratch for the analysis recurrence state: nctas x 2 nside x 3 float64. */
int64_t gm_tc_ana_scratch_bytes(int64_t nside, int64_t nctas);
/* Synthesis chunk offsets (host array of lmax+2 int64; total chunks in choff[lmax+1]) and
 * image bytes for that many chunks (32 KB each). */
int gm_tc_syn_chunk_offsets(int64_t lmax, int spin, int64_t *choff_host);
int64_t gm_tc_syn_image_bytes(int64_t nchunks);
/* Recurrence coefficient table (nelem, 4) float64 for spin 0 or 2: entry idx(l, m) holds
 * (alpha, beta, c0, 0), 32 bytes so that (alpha, beta) is one aligned 16-byte load. */
int gm_tc_coef_table(int64_t lmax, int spin, double *tab, void *stream);
/* Ring spectra (ncomp, nring, L) complex64 -> rhs_map (L, nlanes, ncomp) float4
 * [G_N re, im, G_S re, im] and the analysis images scaled by img_scale (img_b only for
 * spin 2). */
int gm_tc_pack(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const void *ringspec,
               void *rhs_map, void *img_a, void *img_b, double img_scale, void *stream);
/* alm_i += scale * analysis of the rows of `img` for row variant sp (0, -2, +2).
 * scratch: gm_tc_ana_scratch_bytes(nside, nctas); nctas persistent CTAs (one per SM).
 * err (int32) set non-zero if a bounded wait timed out. */
int gm_tc_analysis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                   const double *geom, const double *seeds, const double *coef, const void *img,
                   double *alm_i, double scale, double *scratch, int64_t nctas, int32_t *err,
                   void *stream);
/* gm_tc_analysis without any caller-allocated memory.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc or hand over a scratch buffer: for example a
 * custom call inside a framework that owns every device allocation (an XLA/JAX FFI
 * handler draws only on the framework's own pool), or a service that reserves its device
 * memory once at start-up and must not allocate afterwards (cudaMalloc may synchronise the
 * device and fragments the reserved space).  The recurrence-state scratch is a file-scope
 * device array of 606208 (CTA, lane) slots x 3 float64 (14.5 MB, enough for nctas = 148 at
 * Nside 2048), held by every GPU that loads the library until the process exits; calls with
 * nctas * 2 * nside above 606208 return GM_ERR_BAD_SHAPE.  The first call on a device looks
 * up the array's device address with that device current; make that first call before any
 * stream capture.  That address is kept for the life of the process and does not survive a
 * cudaDeviceReset of the device (or any other teardown of its context): do not call this
 * entry point again after one.  The array keeps the last call's contents (nothing in it needs clearing)
 * and calls that overlap on the GPU race on it.  Inputs and outputs as gm_tc_analysis: the
 * caller zeroes alm_i before the first accumulation and *err before the call. */
int gm_tc_analysis_noalloc(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                           const double *geom, const double *seeds, const double *coef,
                           const void *img, double *alm_i, double scale, int64_t nctas,
                           int32_t *err, void *stream);

/* Synthesis operand images from alm_scale * alm_i for row variant sp (device choff). */
int gm_tc_prep_syn(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                   const int64_t *choff, void *simg, int64_t simg_bytes, double alm_scale,
                   void *stream);
/* synd (L, nlanes, 2H) float32 = out_scale * rows of the synthesis for row variant sp. */
int gm_tc_synthesis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                    const double *geom, const double *seeds, const double *coef, const void *simg,
                    const int64_t *choff, float *synd, double out_scale, int32_t *err,
                    void *stream);
/* Ring-fold residual of the batched synthesis minus rhs_map, written as the next
 * analysis images scaled by img_scale (replaces march_v2.cu:426-493 for the batched
 * path). */
int gm_tc_fold(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const float *synd_a,
               const float *synd_b, const void *rhs_map, const uint8_t *shifted, void *img_a,
               void *img_b, double img_scale, void *stream);
/* Batched synthesis output -> syn layout of gm_ring_synthesis. */
int gm_tc_synd_to_syn(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const float *synd_a,
                      const float *synd_b, float *syn, void *stream);

/* gm_legendre_analysis_tile / gm_legendre_synthesis_tile in mixed precision (spin 0 or 2)
 * with the rows of the checkpoint tables below instead of the FP64 recurrence: the
 * single-precision difference form restarted every 128 rows (same reference interface,
 * march_v2.cu:155-407).  ck_a/cn_a: table of s' = 0 (spin 0) or -2; ck_b/cn_b: s' = +2
 * (ignored for spin 0); segoff: device offsets of gm_ck_offsets.  mask_a / mask_b: NULL, or
 * the per-segment lane-group masks of the two tables (gm_ck_masks' seg_mask; mask_b ignored
 * for spin 0): a CTA whose lanes all start a segment from zero skips its 128 rows (exact). */
int gm_legendre_analysis_ck(int spin, int64_t nside, int64_t lmax, int64_t ncomp,
                            const double *lane_geom, const void *rhs, double *alm, double scale,
                            const int64_t *segoff, const void *ck_a, const uint8_t *cn_a,
                            const void *ck_b, const uint8_t *cn_b, const uint64_t *mask_a,
                            const uint64_t *mask_b, int tile, void *stream);
int gm_legendre_synthesis_ck(int spin, int64_t nside, int64_t lmax, int64_t ncomp,
                             const double *lane_geom, const double *alm, void *syn,
                             const int64_t *segoff, const void *ck_a, const uint8_t *cn_a,
                             const void *ck_b, const uint8_t *cn_b, const uint64_t *mask_a,
                             const uint64_t *mask_b, int tile, void *stream);

/* ---- checkpointed batched Legendre contraction (replaces march_v2.cu:155-407 for batched
 * maps; the reference's window tables march_v2.py:388-450 are its per-geometry constants).
 * The rows are generated in single precision by the difference form of the recurrence,
 * restarted every 128 rows (segment) from a checkpoint table built once per geometry and
 * row variant by the FP64 recurrence.  Order m has ceil((lmax + 1 - l0)/128) segments
 * (l0 = max(m, |s'|)); the table holds, per (segment, lane), the pre-state float2
 * (v_{l_s - 1}, D_{l_s}) scaled by 2^(64 n) and the shift n (uint8).  Analysis units are
 * superblocks of 256 rows (two segments).
 *
 * Host-side offsets: segoff[m] (first segment of order m) and uoff[m] (first analysis unit),
 * lmax + 2 entries each. */
int gm_ck_offsets(int64_t lmax, int spin, int64_t *segoff_host, int64_t *uoff_host);
/* Entries (segments x 2 nside) of one row variant's table, or -1 on bad arguments. */
int64_t gm_ck_table_entries(int64_t nside, int64_t lmax, int spin);
/* Build the checkpoint table of row variant sp (0; -2, +2) from the FP64 recurrence.
 * segoff: device copy of gm_ck_offsets' segoff. */
int gm_ck_build(int64_t nside, int64_t lmax, int spin, int sp, const double *geom,
                const double *seeds, const double *coef, const int64_t *segoff, void *ck_state,
                uint8_t *ck_shift, void *stream);
/* alm_i += scale * analysis of the rows of `img` (gm_tc_pack / gm_tc_fold images) for row
 * variant sp; nctas persistent CTAs.  No scratch: each alm element belongs to one unit.
 * At most 4096 lanes (nside <= 2048; GM_ERR_BAD_SHAPE above).
 * err (int32) set non-zero if a bounded wait timed out. */
int gm_ck_analysis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                   const double *geom, const double *coef, const int64_t *segoff,
                   const int64_t *uoff, const void *ck_state, const uint8_t *ck_shift,
                   const void *img, double *alm_i, double scale, int64_t nctas, int32_t *err,
                   void *stream);
/* Synthesis chunk offsets of the checkpointed layout: chunk cc of order m covers rows
 * l0 + 64 cc + [0, 64); choff_host has lmax + 2 entries. */
int gm_ck_syn_chunk_offsets(int64_t lmax, int spin, int64_t *choff_host);
/* Synthesis operand images (checkpointed layout) from alm_scale * alm_i, row variant sp. */
int gm_ck_prep_syn(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                   const int64_t *choff, void *simg, int64_t simg_bytes, double alm_scale,
                   void *stream);
/* synd (L, nlanes, 2H) float32 = out_scale * rows of the synthesis for row variant sp. */
int gm_ck_synthesis(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                    const double *geom, const double *coef, const int64_t *segoff,
                    const void *ck_state, const uint8_t *ck_shift, const void *simg,
                    const int64_t *choff, float *synd, double out_scale, int32_t *err,
                    void *stream);
/* Lane-group masks of the checkpoint tables (nside <= 2048): bit g of seg_mask[seg] is set
 * when some lane of the 64-lane group g has a non-zero stored state or shift at segment seg
 * (a segment that starts from a zero state stays exactly zero); unit_mask[u] is the union
 * over analysis unit u's two segments.  seg_mask has gm_ck_segments(lmax, spin) entries,
 * unit_mask uoff[lmax + 1]; segoff and uoff are device copies of gm_ck_offsets' tables.
 * Built once per geometry and row variant, beside the tables (the reference's march skips
 * polar lanes whose rows stay below its emission threshold, march_v2.py:290-332, mlim). */
int64_t gm_ck_segments(int64_t lmax, int spin);
int gm_ck_masks(int64_t nside, int64_t lmax, int spin, const void *ck_state, const uint8_t *ck_shift,
                const int64_t *segoff, const int64_t *uoff, uint64_t *seg_mask, uint64_t *unit_mask,
                void *stream);
/* gm_ck_analysis skipping the 64-lane groups of a unit whose rows are all zero, and
 * gm_ck_synthesis skipping the segments in which all 256 lanes of a CTA's tile are zero:
 * bit-identical results (the skipped products are exact zeros). */
int gm_ck_analysis_masked(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                          const double *geom, const double *coef, const int64_t *segoff,
                          const int64_t *uoff, const void *ck_state, const uint8_t *ck_shift,
                          const uint64_t *unit_mask, const void *img, double *alm_i, double scale,
                          int64_t nctas, int32_t *err, void *stream);
int gm_ck_synthesis_masked(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                           const double *geom, const double *coef, const int64_t *segoff,
                           const void *ck_state, const uint8_t *ck_shift, const uint64_t *seg_mask,
                           const void *simg, const int64_t *choff, float *synd, double out_scale,
                           int32_t *err, void *stream);
/* Order windows of the batched transforms, for geometries whose full-size buffers do not
 * fit (Nside 4096 batches, Nside 8192): each entry handles the orders m in [mbeg, mend)
 * only, and its per-order buffers hold just those orders, indexed by m - mbeg (analysis
 * images: (mend - mbeg) x gm_tc_lane_groups(nside) x 64 KB; synthesis images: from
 * choff[mbeg] to choff[mend]; synd: (mend - mbeg, nlanes, rows)).  rhs_map of
 * gm_tc_pack_window may be NULL (transforms without the ring-fold refinement).  The alm
 * accumulator, the ring spectra and the syn buffer keep their full size.  The entries
 * above are these with the window [0, lmax + 1).  Same reference interfaces as above
 * (march_v2.py:637-663, march_v2.cu:155-407); the reference runs its latitudinal
 * transform on order ranges the same way when it splits the orders [0, split) and
 * [split, L) between two GPUs (healpix.py:528-548). */
int gm_tc_pack_window(int64_t nside, int64_t lmax, int spin, int64_t ncomp, const void *ringspec,
                      void *rhs_map, void *img_a, void *img_b, double img_scale, int64_t mbeg,
                      int64_t mend, void *stream);
int gm_tc_analysis_window(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                          const double *geom, const double *seeds, const double *coef,
                          const void *img, double *alm_i, double scale, double *scratch,
                          int64_t nctas, int64_t mbeg, int64_t mend, int32_t *err, void *stream);
int gm_tc_prep_syn_window(int64_t lmax, int spin, int sp, int64_t ncomp, const double *alm_i,
                          const int64_t *choff, void *simg, int64_t simg_bytes, double alm_scale,
                          int64_t mbeg, int64_t mend, void *stream);
int gm_tc_synthesis_window(int64_t nside, int64_t lmax, int spin, int sp, int64_t ncomp,
                           const double *geom, const double *seeds, const double *coef,
                           const void *simg, const int64_t *choff, float *synd, double out_scale,
                           int64_t mbeg, int64_t mend, int32_t *err, void *stream);
int gm_tc_synd_to_syn_window(int64_t nside, int64_t lmax, int spin, int64_t ncomp,
                             const float *synd_a, const float *synd_b, float *syn, int64_t mbeg,
                             int64_t mend, void *stream);
/* alm_i <-> API layout (nalm, nelem) complex128 (spin 2: E, B per field). */
int gm_tc_alm_layout(int64_t lmax, int spin, int64_t nfield, double *alm_i, double *alm_api,
                     int to_api, void *stream);

/* ---------------------------------------------------------- mask apodisation */

/* Replaces the host k-d tree and query_disc of mask_apodization (gmaster/utils.py:61-147).
 * gm_mask_ring_runs: for every pixel p of a RING-ordered (npix,) mask, prev[p] / next[p] =
 * ring-local index of the masked pixel (mask <= 0) at or before / at or after p, cyclically
 * within p's ring; -1 on rings without masked pixels.  prev and next are caller-owned int32
 * (npix,) buffers.  nside in [1, 16384].
 * gm_mask_apodize: ring_table = (5, 4 nside - 1) float64 [cos theta; sin theta; phi0;
 * 2 pi / nphi; nphi / (2 pi)] of the rings.  For every pixel, the chord^2 d^2 to the nearest masked pixel (exact, over all
 * masked pixels) is found when below chord2_max (exclusive).  mode 0 (C1) / 1 (C2): out =
 * mask * f(x), x = sqrt(d^2 / 2 / threshold), for pixels with mask > 0 and d^2 <
 * chord2_max, else out = mask; f = x - sin(2 pi x)/(2 pi) (C1) or (1 - cos(pi x))/2 (C2).
 * mode 2 (zeroing step of "Smooth"): out = 0 for masked pixels and for pixels with d^2 <
 * chord2_max, else mask.  out may not alias mask. */
int gm_mask_ring_runs(int64_t nside, const double *mask, int32_t *prev, int32_t *next,
                      void *stream);
int gm_mask_apodize(int64_t nside, const double *ring_table, const double *mask,
                    const int32_t *prev, const int32_t *next, double chord2_max,
                    double threshold, int mode, double *out, void *stream);

/* ---------------------------------------------------------- Gaussian covariance */

/* Narrow-kernel Gaussian covariance of two pseudo-C_ell power spectra (replaces the jnp
 * assembly and binning of NmtCovarianceWorkspace.gaussian_covariance,
 * gmaster/covariance.py:407-575).  Output block x (< nblocks <= 16) is
 *   cov_x(l1, l2) = sum over terms t in [block_ptr[x], block_ptr[x+1]) of
 *     signs[t] * (A(l1) B(l2) + A(l2) B(l1)) / 2 * xi[k](l1, l2),
 * (k, ra, rb) = terms[3t .. 3t+2], A = spec[ra], B = spec[rb] (rows of L = lmax + 1
 * doubles), xi = (nk, L, L) float64 coupling kernels.  All indices are trusted.
 * gm_cov_binned: out (nblocks, nbands_a, nbands_b) = sum over l1 in band p (CSR ptr_a /
 * ells_a) and l2 in band q of w_a[l1] w_b[l2] cov_x(l1, l2); nbands_a <= 65535.
 * gm_cov_coupled: out (nblocks, L, L) = cov_x; L <= 65535. */
int gm_cov_binned(int64_t lmax, int64_t nblocks, const double *xi, const double *spec,
                  const int32_t *terms, const double *signs, const int32_t *block_ptr,
                  int64_t nbands_a, const int32_t *ptr_a, const int32_t *ells_a,
                  const double *w_a, int64_t nbands_b, const int32_t *ptr_b,
                  const int32_t *ells_b, const double *w_b, double *out, void *stream);
int gm_cov_coupled(int64_t lmax, int64_t nblocks, const double *xi, const double *spec,
                   const int32_t *terms, const double *signs, const int32_t *block_ptr,
                   double *out, void *stream);

/* ---------------------------------------------------------- purified coupling (quadrature) */

/* Gauss-Legendre quadrature for the coupling blocks of purified E/B fields (replaces
 * workspaces.py:593-605 `_gauss_legendre` and :608-679 `_wigner_d_table`, used by
 * :927-1061 `_coupling_matrices_pure_quadrature`).
 * gm_gl_nodes: the n nodes x (ascending) and weights w of the n-point rule on [-1, 1].
 * gm_wigner_table: out (lmax + 1, nnodes) = d^l_mn(arccos x[i]) (zero for l < max(|m|,|n|));
 * norm[k] = sqrt(k! (k+mu+nu)! / ((k+mu)! (k+nu)!)), mu = |m-n|, nu = |m+n|, for
 * k <= lmax - max(|m|,|n|) (at least 2 entries).  |m|, |n| <= 16.
 * gm_wigner_corr: out (nvec, nnodes) = sum_l d^l_mn(arccos x[i]) vec[v][l] for nvec <= 2
 * vectors of lmax + 1 doubles (the rows are not stored). */
int gm_gl_nodes(int64_t n, double *x, double *w, void *stream);
int gm_wigner_table(int64_t nnodes, const double *x, int64_t lmax, int m, int n,
                    const double *norm, double *out, void *stream);
int gm_wigner_corr(int64_t nnodes, const double *x, int64_t lmax, int m, int n,
                   const double *norm, int64_t nvec, const double *vec, double *out,
                   void *stream);

/* ---------------------------------------------------------- tensor-core check */

/* One-CTA tcgen05 check: D[128 x N] (float32, row-major) = A[128 x K] * B[N x K]^T where
 * A and B are bf16 operand images in the K-major 128-byte-swizzled layout the tensor-core
 * kernels use (K in atoms of 64; element (r, k) of an R-row image at byte
 * (k/64) R 128 + (r/8) 1024 + (r%8) 128 + (((k%64)/8) ^ (r%8)) 16 + (k%8) 2).
 * With a_mn / b_mn set, that operand is MN-major instead: element (r, k) of an R-row
 * image (R % 64 == 0) at byte (k/8) (R/64) 1024 + (r/64) 1024 + (k%8) 128
 * + (((r%64)/8) ^ (k%8)) 16 + (r%8) 2.
 * N in [16, 256] step 16, K a multiple of 64.  err (one int32) is set non-zero if a
 * bounded wait timed out.  No counterpart in the reference: a health check of the
 * tensor-core machinery used by gm_legendre_*_tc. */
int gm_tc_selftest(int64_t N, int64_t K, int a_mn, int b_mn, const void *aimg,
                   const void *bimg, float *D, int32_t *err, void *stream);
/* gm_tc_selftest (K-major operands) whose issuer arms the load barrier but issues no copy:
 * every bounded wait runs out after wait_ns (1 us .. 2 s) and *err is set to 1; the kernel
 * skips its MMAs, releases its tensor memory and returns.  Exercises the timeout path of
 * the tensor-core kernels (GM_ERR_TIMEOUT on the host) without a fault or a hang.  No
 * counterpart in the reference (its FFI handlers map launch errors to XLA errors,
 * march_v2.cu:509-518). */
int gm_tc_selftest_timeout(int64_t N, int64_t K, const void *aimg, const void *bimg, float *D,
                           int32_t *err, int64_t wait_ns, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GM_B200_H */
