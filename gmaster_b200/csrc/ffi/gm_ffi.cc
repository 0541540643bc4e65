// XLA FFI handlers (symbols gmb_*) over the C ABI of libgm_b200.so, for jax.ffi.
//
// Each handler binds the typed buffers and attributes of one gm_* entry point, as the
// reference binds its kernels (gmaster/_native/cuda/march_v2.cu:545-594,
// coupling_tt.cu:77-81): XLA owns every buffer, the kernels run on XLA's stream
// (PlatformStream<cudaStream_t>), scratch comes in as extra result buffers sized by the
// gm_*_bytes queries, and a non-zero gm_status becomes an XLA error
// (GM_ERR_BAD_SHAPE / GM_ERR_BAD_PTR: InvalidArgument, anything else: Internal, with the
// library's last error string).  Entries that accumulate into an output (the analyses,
// alm += scale * result) take the accumulator as their last input and write into their
// result buffer in place: the Python side aliases that input to the result
// (jax.ffi.ffi_call(..., input_output_aliases={input: result})), so the two share memory.
//
// Built by gmaster_b200/_build.py only where jax.ffi.include_dir() provides the XLA FFI
// headers (not in every environment), into libgm_b200_ffi.so linked against libgm_b200.so;
// register each handler with jax.ffi.register_ffi_target("gmb_...", capsule, platform="CUDA").
#include <cuda_runtime.h>

#include <cstdint>

#include "gm_b200.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status_error(int st)
{
    if (st == GM_OK) return ffi::Error::Success();
    const char *msg = gm_last_error();
    const char *text = msg && *msg ? msg : "gm_b200 entry point failed";
    if (st == GM_ERR_BAD_SHAPE || st == GM_ERR_BAD_PTR) return ffi::Error::InvalidArgument(text);
    return ffi::Error::Internal(text);
}

template <typename T>
T *ptr(ffi::AnyBuffer b) { return static_cast<T *>(b.untyped_data()); }

template <typename T>
T *rptr(ffi::Result<ffi::AnyBuffer> &b) { return static_cast<T *>(b->untyped_data()); }

// ------------------------------------------------------------------- ring stage

ffi::Error RingAnalysis(cudaStream_t s, ffi::AnyBuffer maps, ffi::AnyBuffer mask, ffi::AnyBuffer tw,
                        ffi::AnyBuffer shifted, ffi::Result<ffi::AnyBuffer> ringspec,
                        ffi::Result<ffi::AnyBuffer> scratch, int32_t precision, int64_t nside, int64_t L,
                        int64_t ncomp, int32_t map_bytes, bool has_mask)
{
    return status_error(gm_ring_analysis_ws(precision, nside, L, ncomp, maps.untyped_data(), map_bytes,
                                            has_mask ? ptr<const double>(mask) : nullptr,
                                            tw.untyped_data(), ptr<const uint8_t>(shifted),
                                            ringspec->untyped_data(), scratch->untyped_data(),
                                            (int64_t)scratch->size_bytes(), 0, 0, s));
}

ffi::Error RingSynthesis(cudaStream_t s, ffi::AnyBuffer syn, ffi::AnyBuffer tw, ffi::AnyBuffer shifted,
                         ffi::Result<ffi::AnyBuffer> maps, ffi::Result<ffi::AnyBuffer> scratch,
                         int32_t precision, int64_t nside, int64_t L, int64_t ncomp)
{
    return status_error(gm_ring_synthesis_ws(precision, nside, L, ncomp, syn.untyped_data(),
                                             tw.untyped_data(), ptr<const uint8_t>(shifted),
                                             rptr<double>(maps), scratch->untyped_data(),
                                             (int64_t)scratch->size_bytes(), 0, 0, s));
}

ffi::Error PackRhs(cudaStream_t s, ffi::AnyBuffer ringspec, ffi::Result<ffi::AnyBuffer> rhs,
                   int32_t precision, int64_t nside, int64_t L, int64_t ncomp)
{
    return status_error(gm_pack_rhs(precision, nside, L, ncomp, ringspec.untyped_data(),
                                    rhs->untyped_data(), s));
}

ffi::Error FoldResidual(cudaStream_t s, ffi::AnyBuffer syn, ffi::AnyBuffer rhs_map, ffi::AnyBuffer shifted,
                        ffi::Result<ffi::AnyBuffer> rhs_out, int32_t precision, int64_t nside, int64_t L,
                        int64_t ncomp)
{
    return status_error(gm_fold_residual(precision, nside, L, ncomp, syn.untyped_data(),
                                         rhs_map.untyped_data(), ptr<const uint8_t>(shifted),
                                         rhs_out->untyped_data(), s));
}

// ------------------------------------------------------------ Legendre stage (SIMT)

ffi::Error LegendreAnalysis(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer seeds, ffi::AnyBuffer rhs,
                            ffi::AnyBuffer alm_in, ffi::Result<ffi::AnyBuffer> alm, int32_t precision, int32_t spin,
                            int64_t nside, int64_t lmax, int64_t ncomp, double scale, int32_t tile)
{
    return status_error(gm_legendre_analysis_tile(precision, spin, nside, lmax, ncomp,
                                                  ptr<const double>(geom), ptr<const double>(seeds),
                                                  rhs.untyped_data(), rptr<double>(alm), scale, tile, s));
}

ffi::Error LegendreSynthesis(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer seeds, ffi::AnyBuffer alm,
                             ffi::Result<ffi::AnyBuffer> syn, int32_t precision, int32_t spin,
                             int64_t nside, int64_t lmax, int64_t ncomp, int32_t tile)
{
    return status_error(gm_legendre_synthesis_tile(precision, spin, nside, lmax, ncomp,
                                                   ptr<const double>(geom), ptr<const double>(seeds),
                                                   ptr<const double>(alm), syn->untyped_data(), tile, s));
}

ffi::Error LegendreAnalysisCk(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer rhs, ffi::AnyBuffer segoff,
                              ffi::AnyBuffer ck_a, ffi::AnyBuffer cn_a, ffi::AnyBuffer ck_b,
                              ffi::AnyBuffer cn_b, ffi::AnyBuffer alm_in, ffi::Result<ffi::AnyBuffer> alm, int32_t spin,
                              int64_t nside, int64_t lmax, int64_t ncomp, double scale, int32_t tile)
{
    return status_error(gm_legendre_analysis_ck(spin, nside, lmax, ncomp, ptr<const double>(geom),
                                                rhs.untyped_data(), rptr<double>(alm), scale,
                                                ptr<const int64_t>(segoff), ck_a.untyped_data(),
                                                ptr<const uint8_t>(cn_a), ck_b.untyped_data(),
                                                ptr<const uint8_t>(cn_b), nullptr, nullptr, tile, s));
}

ffi::Error LegendreSynthesisCk(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer alm, ffi::AnyBuffer segoff,
                               ffi::AnyBuffer ck_a, ffi::AnyBuffer cn_a, ffi::AnyBuffer ck_b,
                               ffi::AnyBuffer cn_b, ffi::Result<ffi::AnyBuffer> syn, int32_t spin,
                               int64_t nside, int64_t lmax, int64_t ncomp, int32_t tile)
{
    return status_error(gm_legendre_synthesis_ck(spin, nside, lmax, ncomp, ptr<const double>(geom),
                                                 ptr<const double>(alm), syn->untyped_data(),
                                                 ptr<const int64_t>(segoff), ck_a.untyped_data(),
                                                 ptr<const uint8_t>(cn_a), ck_b.untyped_data(),
                                                 ptr<const uint8_t>(cn_b), nullptr, nullptr, tile, s));
}

// ------------------------------------------------------- Legendre stage (tensor cores)

ffi::Error TcPack(cudaStream_t s, ffi::AnyBuffer ringspec, ffi::Result<ffi::AnyBuffer> rhs_map,
                  ffi::Result<ffi::AnyBuffer> img_a, ffi::Result<ffi::AnyBuffer> img_b, int64_t nside,
                  int64_t lmax, int32_t spin, int64_t ncomp, double img_scale)
{
    return status_error(gm_tc_pack(nside, lmax, spin, ncomp, ringspec.untyped_data(),
                                   rhs_map->untyped_data(), img_a->untyped_data(),
                                   spin ? img_b->untyped_data() : nullptr, img_scale, s));
}

ffi::Error CkBuild(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer seeds, ffi::AnyBuffer coef,
                   ffi::AnyBuffer segoff, ffi::Result<ffi::AnyBuffer> ck_state,
                   ffi::Result<ffi::AnyBuffer> ck_shift, int64_t nside, int64_t lmax, int32_t spin,
                   int32_t sp)
{
    return status_error(gm_ck_build(nside, lmax, spin, sp, ptr<const double>(geom), ptr<const double>(seeds),
                                    ptr<const double>(coef), ptr<const int64_t>(segoff),
                                    ck_state->untyped_data(), rptr<uint8_t>(ck_shift), s));
}

ffi::Error CoefTable(cudaStream_t s, ffi::Result<ffi::AnyBuffer> tab, int64_t lmax, int32_t spin)
{
    return status_error(gm_tc_coef_table(lmax, spin, rptr<double>(tab), s));
}

ffi::Error CkAnalysis(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer coef, ffi::AnyBuffer segoff,
                      ffi::AnyBuffer uoff, ffi::AnyBuffer ck_state, ffi::AnyBuffer ck_shift, ffi::AnyBuffer img,
                      ffi::AnyBuffer alm_in, ffi::Result<ffi::AnyBuffer> alm_i, ffi::Result<ffi::AnyBuffer> err, int64_t nside,
                      int64_t lmax, int32_t spin, int32_t sp, int64_t ncomp, double scale, int64_t nctas)
{
    return status_error(gm_ck_analysis(nside, lmax, spin, sp, ncomp, ptr<const double>(geom),
                                       ptr<const double>(coef), ptr<const int64_t>(segoff),
                                       ptr<const int64_t>(uoff), ck_state.untyped_data(),
                                       ptr<const uint8_t>(ck_shift), img.untyped_data(), rptr<double>(alm_i),
                                       scale, nctas, rptr<int32_t>(err), s));
}

ffi::Error CkMasks(cudaStream_t s, ffi::AnyBuffer ck_state, ffi::AnyBuffer ck_shift, ffi::AnyBuffer segoff,
                   ffi::AnyBuffer uoff, ffi::Result<ffi::AnyBuffer> seg_mask, ffi::Result<ffi::AnyBuffer> unit_mask,
                   int64_t nside, int64_t lmax, int32_t spin)
{
    return status_error(gm_ck_masks(nside, lmax, spin, ck_state.untyped_data(), ptr<const uint8_t>(ck_shift),
                                    ptr<const int64_t>(segoff), ptr<const int64_t>(uoff), rptr<uint64_t>(seg_mask),
                                    rptr<uint64_t>(unit_mask), s));
}

ffi::Error CkAnalysisMasked(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer coef, ffi::AnyBuffer segoff,
                            ffi::AnyBuffer uoff, ffi::AnyBuffer ck_state, ffi::AnyBuffer ck_shift,
                            ffi::AnyBuffer unit_mask, ffi::AnyBuffer img, ffi::AnyBuffer alm_in,
                            ffi::Result<ffi::AnyBuffer> alm_i, ffi::Result<ffi::AnyBuffer> err, int64_t nside,
                            int64_t lmax, int32_t spin, int32_t sp, int64_t ncomp, double scale, int64_t nctas)
{
    return status_error(gm_ck_analysis_masked(nside, lmax, spin, sp, ncomp, ptr<const double>(geom),
                                              ptr<const double>(coef), ptr<const int64_t>(segoff),
                                              ptr<const int64_t>(uoff), ck_state.untyped_data(),
                                              ptr<const uint8_t>(ck_shift), ptr<const uint64_t>(unit_mask),
                                              img.untyped_data(), rptr<double>(alm_i), scale, nctas,
                                              rptr<int32_t>(err), s));
}

ffi::Error CkPrepSyn(cudaStream_t s, ffi::AnyBuffer alm_i, ffi::AnyBuffer choff, ffi::Result<ffi::AnyBuffer> simg,
                     int64_t lmax, int32_t spin, int32_t sp, int64_t ncomp, double alm_scale)
{
    return status_error(gm_ck_prep_syn(lmax, spin, sp, ncomp, ptr<const double>(alm_i),
                                       ptr<const int64_t>(choff), simg->untyped_data(),
                                       (int64_t)simg->size_bytes(), alm_scale, s));
}

ffi::Error CkSynthesis(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer coef, ffi::AnyBuffer segoff,
                       ffi::AnyBuffer ck_state, ffi::AnyBuffer ck_shift, ffi::AnyBuffer simg, ffi::AnyBuffer choff,
                       ffi::Result<ffi::AnyBuffer> synd, ffi::Result<ffi::AnyBuffer> err, int64_t nside,
                       int64_t lmax, int32_t spin, int32_t sp, int64_t ncomp, double out_scale)
{
    return status_error(gm_ck_synthesis(nside, lmax, spin, sp, ncomp, ptr<const double>(geom),
                                        ptr<const double>(coef), ptr<const int64_t>(segoff),
                                        ck_state.untyped_data(), ptr<const uint8_t>(ck_shift),
                                        simg.untyped_data(), ptr<const int64_t>(choff), rptr<float>(synd),
                                        out_scale, rptr<int32_t>(err), s));
}

ffi::Error CkSynthesisMasked(cudaStream_t s, ffi::AnyBuffer geom, ffi::AnyBuffer coef, ffi::AnyBuffer segoff,
                             ffi::AnyBuffer ck_state, ffi::AnyBuffer ck_shift, ffi::AnyBuffer seg_mask,
                             ffi::AnyBuffer simg, ffi::AnyBuffer choff, ffi::Result<ffi::AnyBuffer> synd,
                             ffi::Result<ffi::AnyBuffer> err, int64_t nside, int64_t lmax, int32_t spin, int32_t sp,
                             int64_t ncomp, double out_scale)
{
    return status_error(gm_ck_synthesis_masked(nside, lmax, spin, sp, ncomp, ptr<const double>(geom),
                                               ptr<const double>(coef), ptr<const int64_t>(segoff),
                                               ck_state.untyped_data(), ptr<const uint8_t>(ck_shift),
                                               ptr<const uint64_t>(seg_mask), simg.untyped_data(),
                                               ptr<const int64_t>(choff), rptr<float>(synd), out_scale,
                                               rptr<int32_t>(err), s));
}

ffi::Error TcFold(cudaStream_t s, ffi::AnyBuffer synd_a, ffi::AnyBuffer synd_b, ffi::AnyBuffer rhs_map,
                  ffi::AnyBuffer shifted, ffi::Result<ffi::AnyBuffer> img_a, ffi::Result<ffi::AnyBuffer> img_b,
                  int64_t nside, int64_t lmax, int32_t spin, int64_t ncomp, double img_scale)
{
    return status_error(gm_tc_fold(nside, lmax, spin, ncomp, ptr<const float>(synd_a),
                                   spin ? ptr<const float>(synd_b) : nullptr, rhs_map.untyped_data(),
                                   ptr<const uint8_t>(shifted), img_a->untyped_data(),
                                   spin ? img_b->untyped_data() : nullptr, img_scale, s));
}

ffi::Error TcAlmLayout(cudaStream_t s, ffi::AnyBuffer alm_i, ffi::Result<ffi::AnyBuffer> alm_api, int64_t lmax,
                       int32_t spin, int64_t nfield)
{
    return status_error(gm_tc_alm_layout(lmax, spin, nfield, ptr<double>(alm_i), rptr<double>(alm_api), 1, s));
}

// ---------------------------------------------------------- spectra and coupling

ffi::Error PseudoCl(cudaStream_t s, ffi::AnyBuffer alm1, ffi::AnyBuffer alm2, ffi::Result<ffi::AnyBuffer> cls,
                    int64_t lmax, int64_t n1, int64_t n2)
{
    return status_error(gm_pseudo_cl(lmax, n1, ptr<const double>(alm1), n2, ptr<const double>(alm2),
                                     rptr<double>(cls), s));
}

ffi::Error CouplingBlocks(cudaStream_t s, ffi::AnyBuffer window, ffi::Result<ffi::AnyBuffer> blocks,
                          ffi::Result<ffi::AnyBuffer> queue, int64_t lmax, int32_t which)
{
    // the work queue counter starts at zero
    if (cudaMemsetAsync(queue->untyped_data(), 0, sizeof(int64_t), s) != cudaSuccess)
        return ffi::Error::Internal("gmb_coupling_blocks: queue reset failed");
    return status_error(gm_coupling_blocks(lmax, ptr<const double>(window), (int64_t)window.element_count(),
                                           which, rptr<double>(blocks), rptr<int64_t>(queue), s));
}

ffi::Error BinCoupling(cudaStream_t s, ffi::AnyBuffer blocks, ffi::AnyBuffer band_ptr, ffi::AnyBuffer band_ells,
                       ffi::AnyBuffer wfl, ffi::AnyBuffer inv_fl, ffi::AnyBuffer beam,
                       ffi::Result<ffi::AnyBuffer> scratch, ffi::Result<ffi::AnyBuffer> out, int64_t lmax,
                       int64_t nbands, int32_t ncls)
{
    return status_error(gm_bin_coupling_csr(lmax, nbands, ncls, ptr<const double>(blocks),
                                            ptr<const int32_t>(band_ptr), ptr<const int32_t>(band_ells),
                                            ptr<const double>(wfl), ptr<const double>(inv_fl),
                                            ptr<const double>(beam), rptr<double>(scratch), rptr<double>(out), s));
}

ffi::Error BinCells(cudaStream_t s, ffi::AnyBuffer cls, ffi::AnyBuffer band_ptr, ffi::AnyBuffer band_ells,
                    ffi::AnyBuffer wfl, ffi::Result<ffi::AnyBuffer> out, int64_t lmax, int64_t nbands, int64_t ncls)
{
    return status_error(gm_bin_cells_csr(lmax, nbands, ncls, ptr<const double>(cls), ptr<const int32_t>(band_ptr),
                                         ptr<const int32_t>(band_ells), ptr<const double>(wfl), rptr<double>(out),
                                         s));
}

ffi::Error LuFactor(cudaStream_t s, ffi::AnyBuffer a, ffi::Result<ffi::AnyBuffer> lu, ffi::Result<ffi::AnyBuffer> piv,
                    ffi::Result<ffi::AnyBuffer> status, int64_t n)
{
    if (cudaMemcpyAsync(lu->untyped_data(), a.untyped_data(), a.size_bytes(), cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess ||
        cudaMemsetAsync(status->untyped_data(), 0, sizeof(int32_t), s) != cudaSuccess)
        return ffi::Error::Internal("gmb_lu_factor: staging the matrix failed");
    return status_error(gm_lu_factor(n, rptr<double>(lu), rptr<int32_t>(piv), rptr<int32_t>(status), s));
}

ffi::Error LuSolve(cudaStream_t s, ffi::AnyBuffer lu, ffi::AnyBuffer piv, ffi::AnyBuffer b,
                   ffi::Result<ffi::AnyBuffer> x, int64_t n, int64_t nrhs)
{
    if (cudaMemcpyAsync(x->untyped_data(), b.untyped_data(), b.size_bytes(), cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess)
        return ffi::Error::Internal("gmb_lu_solve: staging the right-hand sides failed");
    return status_error(gm_lu_solve(n, ptr<const double>(lu), ptr<const int32_t>(piv), nrhs, rptr<double>(x), s));
}

}  // namespace

#define GMB_STREAM ffi::Ffi::Bind().Ctx<ffi::PlatformStream<cudaStream_t>>()

XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ring_analysis, RingAnalysis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int32_t>("precision").Attr<int64_t>("nside").Attr<int64_t>("L")
                                  .Attr<int64_t>("ncomp").Attr<int32_t>("map_bytes").Attr<bool>("has_mask"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ring_synthesis, RingSynthesis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int32_t>("precision")
                                  .Attr<int64_t>("nside").Attr<int64_t>("L").Attr<int64_t>("ncomp"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_pack_rhs, PackRhs,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int32_t>("precision")
                                  .Attr<int64_t>("nside").Attr<int64_t>("L").Attr<int64_t>("ncomp"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_fold_residual, FoldResidual,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Attr<int32_t>("precision").Attr<int64_t>("nside")
                                  .Attr<int64_t>("L").Attr<int64_t>("ncomp"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_legendre_analysis, LegendreAnalysis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int32_t>("precision").Attr<int32_t>("spin")
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int64_t>("ncomp")
                                  .Attr<double>("scale").Attr<int32_t>("tile"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_legendre_synthesis, LegendreSynthesis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Attr<int32_t>("precision").Attr<int32_t>("spin")
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int64_t>("ncomp")
                                  .Attr<int32_t>("tile"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_legendre_analysis_ck, LegendreAnalysisCk,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int32_t>("spin")
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int64_t>("ncomp")
                                  .Attr<double>("scale").Attr<int32_t>("tile"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_legendre_synthesis_ck, LegendreSynthesisCk,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int32_t>("spin")
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int64_t>("ncomp")
                                  .Attr<int32_t>("tile"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_tc_pack, TcPack,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Attr<int64_t>("nside").Attr<int64_t>("lmax")
                                  .Attr<int32_t>("spin").Attr<int64_t>("ncomp").Attr<double>("img_scale"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_build, CkBuild,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int32_t>("sp"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_coef_table, CoefTable,
                              GMB_STREAM.Ret<ffi::AnyBuffer>().Attr<int64_t>("lmax").Attr<int32_t>("spin"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_analysis, CkAnalysis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int32_t>("sp").Attr<int64_t>("ncomp").Attr<double>("scale")
                                  .Attr<int64_t>("nctas"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_masks, CkMasks,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_analysis_masked, CkAnalysisMasked,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int32_t>("sp").Attr<int64_t>("ncomp").Attr<double>("scale")
                                  .Attr<int64_t>("nctas"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_synthesis_masked, CkSynthesisMasked,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int32_t>("sp").Attr<int64_t>("ncomp").Attr<double>("out_scale"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_prep_syn, CkPrepSyn,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("lmax").Attr<int32_t>("spin").Attr<int32_t>("sp")
                                  .Attr<int64_t>("ncomp").Attr<double>("alm_scale"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_ck_synthesis, CkSynthesis,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int32_t>("sp").Attr<int64_t>("ncomp").Attr<double>("out_scale"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_tc_fold, TcFold,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("nside").Attr<int64_t>("lmax").Attr<int32_t>("spin")
                                  .Attr<int64_t>("ncomp").Attr<double>("img_scale"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_tc_alm_layout, TcAlmLayout,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int64_t>("lmax")
                                  .Attr<int32_t>("spin").Attr<int64_t>("nfield"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_pseudo_cl, PseudoCl,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("lmax").Attr<int64_t>("n1").Attr<int64_t>("n2"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_coupling_blocks, CouplingBlocks,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Attr<int64_t>("lmax").Attr<int32_t>("which"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_bin_coupling, BinCoupling,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int64_t>("lmax")
                                  .Attr<int64_t>("nbands").Attr<int32_t>("ncls"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_bin_cells, BinCells,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Attr<int64_t>("lmax")
                                  .Attr<int64_t>("nbands").Attr<int64_t>("ncls"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_lu_factor, LuFactor,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>().Ret<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Attr<int64_t>("n"));
XLA_FFI_DEFINE_HANDLER_SYMBOL(gmb_lu_solve, LuSolve,
                              GMB_STREAM.Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>().Arg<ffi::AnyBuffer>()
                                  .Ret<ffi::AnyBuffer>().Attr<int64_t>("n").Attr<int64_t>("nrhs"));
