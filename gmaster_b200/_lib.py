"""ctypes binding of the in-tree CUDA library ``libgm_b200.so`` (C ABI in include/gm_b200.h).

There is no fallback: if the library is missing or cannot be loaded, every compute
call raises ``RuntimeError`` naming the problem.  Device memory and streams come
from PyTorch; the library only ever sees raw device pointers and the current
stream handle.
"""

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgm_b200.so")

_c_i64 = ctypes.c_int64
_c_int = ctypes.c_int
_c_dbl = ctypes.c_double
_c_vp = ctypes.c_void_p

# name -> (argtypes, restype)
SIGNATURES = {
    "gm_last_error": ([], ctypes.c_char_p),
    "gm_version": ([], ctypes.c_char_p),
    "gm_ring_twiddle_count": ([_c_i64], _c_i64),
    "gm_ring_twiddles": ([_c_i64, _c_vp, _c_vp], _c_int),
    "gm_ring_analysis": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
                         _c_int),
    "gm_pack_rhs": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_fold_residual": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
                         _c_int),
    "gm_ring_synthesis": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
                          _c_int),
    "gm_seed_table_len": ([_c_i64], _c_i64),
    "gm_legendre_analysis": ([_c_int, _c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
                              _c_dbl, _c_vp], _c_int),
    "gm_legendre_synthesis": ([_c_int, _c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
                               _c_vp], _c_int),
    "gm_pseudo_cl": ([_c_i64, _c_i64, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_coupling_blocks": ([_c_i64, _c_vp, _c_i64, _c_int, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_coupling_units": ([_c_i64], _c_i64),
    "gm_coupling_blocks_multi": ([_c_i64, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_coupling_pairs_tt": ([_c_i64, _c_vp, _c_i64, _c_vp, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_toeplitz_fill": ([_c_i64, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_bin_coupling_csr": ([_c_i64, _c_i64, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                             _c_vp, _c_vp, _c_vp], _c_int),
    "gm_bin_cells_csr": ([_c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_lu_factor": ([_c_i64, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_lu_solve": ([_c_i64, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_tc_lane_groups": ([_c_i64], _c_i64),
    "gm_tc_ana_image_bytes": ([_c_i64, _c_i64], _c_i64),
    "gm_tc_ana_scratch_bytes": ([_c_i64, _c_i64], _c_i64),
    "gm_tc_syn_chunk_offsets": ([_c_i64, _c_int, _c_vp], _c_int),
    "gm_tc_syn_image_bytes": ([_c_i64], _c_i64),
    "gm_tc_coef_table": ([_c_i64, _c_int, _c_vp, _c_vp], _c_int),
    "gm_tc_pack": ([_c_i64, _c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_vp], _c_int),
    "gm_tc_analysis": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                        _c_dbl, _c_vp, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_tc_analysis_noalloc": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
                                _c_vp, _c_dbl, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_tc_prep_syn": ([_c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_i64, _c_dbl, _c_vp], _c_int),
    "gm_tc_synthesis": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                         _c_vp, _c_dbl, _c_vp, _c_vp], _c_int),
    "gm_tc_fold": ([_c_i64, _c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl,
                    _c_vp], _c_int),
    "gm_tc_synd_to_syn": ([_c_i64, _c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_legendre_tiles": ([_c_int, _c_vp, _c_int], _c_int),
    "gm_legendre_analysis_tile": ([_c_int, _c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
                                   _c_dbl, _c_int, _c_vp], _c_int),
    "gm_legendre_synthesis_tile": ([_c_int, _c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp,
                                    _c_int, _c_vp], _c_int),
    "gm_lu_panel": ([_c_i64, _c_vp, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_lu_trsm": ([_c_i64, _c_vp, _c_i64, _c_i64, _c_vp], _c_int),
    "gm_lu_update": ([_c_i64, _c_vp, _c_i64, _c_i64, _c_vp], _c_int),
    "gm_ring_big_scratch_bytes": ([_c_i64, _c_i64], _c_i64),
    "gm_ring_analysis_ws": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_int, _c_vp, _c_vp, _c_vp, _c_vp,
                             _c_vp, _c_i64, _c_i64, _c_i64, _c_vp], _c_int),
    "gm_ring_synthesis_ws": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64,
                              _c_i64, _c_i64, _c_vp], _c_int),
    "gm_tc_pack_window": ([_c_i64, _c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_i64,
                           _c_i64, _c_vp], _c_int),
    "gm_tc_analysis_window": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                               _c_dbl, _c_vp, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_tc_prep_syn_window": ([_c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_i64, _c_dbl, _c_i64,
                               _c_i64, _c_vp], _c_int),
    "gm_tc_synthesis_window": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                                _c_vp, _c_dbl, _c_i64, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_tc_synd_to_syn_window": ([_c_i64, _c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_i64, _c_i64,
                                  _c_vp], _c_int),
    "gm_tc_alm_layout": ([_c_i64, _c_int, _c_i64, _c_vp, _c_vp, _c_int, _c_vp], _c_int),
    "gm_tc_selftest": ([_c_i64, _c_i64, _c_int, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_tc_selftest_timeout": ([_c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_vp], _c_int),
    "gm_mask_ring_runs": ([_c_i64, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_cov_binned": ([_c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp,
                       _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_cov_coupled": ([_c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_gl_nodes": ([_c_i64, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_wigner_table": ([_c_i64, _c_vp, _c_i64, _c_int, _c_int, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_wigner_corr": ([_c_i64, _c_vp, _c_i64, _c_int, _c_int, _c_vp, _c_i64, _c_vp, _c_vp, _c_vp],
                       _c_int),
    "gm_mask_apodize": ([_c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_dbl, _c_int, _c_vp, _c_vp],
                        _c_int),
    "gm_legendre_analysis_ck": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_dbl, _c_vp, _c_vp,
                                 _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_int, _c_vp], _c_int),
    "gm_legendre_synthesis_ck": ([_c_int, _c_i64, _c_i64, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                                  _c_vp, _c_vp, _c_vp, _c_vp, _c_int, _c_vp], _c_int),
    "gm_ck_offsets": ([_c_i64, _c_int, _c_vp, _c_vp], _c_int),
    "gm_ck_table_entries": ([_c_i64, _c_i64, _c_int], _c_i64),
    "gm_ck_build": ([_c_i64, _c_i64, _c_int, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
                    _c_int),
    "gm_ck_analysis": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                        _c_vp, _c_vp, _c_dbl, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_ck_syn_chunk_offsets": ([_c_i64, _c_int, _c_vp], _c_int),
    "gm_ck_prep_syn": ([_c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_i64, _c_dbl, _c_vp], _c_int),
    "gm_ck_synthesis": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                         _c_vp, _c_vp, _c_dbl, _c_vp, _c_vp], _c_int),
    "gm_ck_segments": ([_c_i64, _c_int], _c_i64),
    "gm_ck_masks": ([_c_i64, _c_i64, _c_int, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp], _c_int),
    "gm_ck_analysis_masked": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                               _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_i64, _c_vp, _c_vp], _c_int),
    "gm_ck_synthesis_masked": ([_c_i64, _c_i64, _c_int, _c_int, _c_i64, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                                _c_vp, _c_vp, _c_vp, _c_vp, _c_dbl, _c_vp, _c_vp], _c_int),
}

STATUS = {0: "GM_OK", 1: "GM_ERR_BAD_SHAPE", 2: "GM_ERR_BAD_PTR", 3: "GM_ERR_LAUNCH",
          4: "GM_ERR_TIMEOUT", 5: "GM_ERR_UNSUPPORTED"}

FP64 = 0
MIXED = 1

_lib = None

# Kernel launches made by each entry point (for launch accounting); default 1.
LAUNCHES = {"gm_last_error": 0, "gm_version": 0, "gm_ring_twiddle_count": 0,
            "gm_seed_table_len": 0, "gm_bin_coupling_csr": 3, "gm_tc_lane_groups": 0,
            "gm_tc_ana_image_bytes": 0, "gm_tc_ana_scratch_bytes": 0,
            "gm_tc_syn_chunk_offsets": 0, "gm_tc_syn_image_bytes": 0, "gm_legendre_tiles": 0,
            "gm_coupling_units": 0, "gm_ring_big_scratch_bytes": 0, "gm_ck_offsets": 0,
            "gm_ck_table_entries": 0, "gm_ck_syn_chunk_offsets": 0, "gm_ck_segments": 0,
            "gm_ck_masks": 2}
CALLS = {}


def load():
    """Load the CUDA library (raises RuntimeError if it is missing or broken)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"gmaster_b200 CUDA library not found at {LIB_PATH}; build it with "
            "`python -m gmaster_b200._build` (there is no CPU fallback)")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as err:
        raise RuntimeError(f"cannot load {LIB_PATH}: {err}") from err
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class GMError(RuntimeError):
    """A gm_* entry point returned a non-zero status."""

    def __init__(self, name, status, detail):
        self.status = status
        super().__init__(f"{name} failed with {STATUS.get(status, status)}: {detail}")


def call(name, *args):
    """Call a status-returning entry point and raise GMError on failure."""
    fn = getattr(load(), name)
    status = fn(*args)
    CALLS[name] = CALLS.get(name, 0) + LAUNCHES.get(name, 1)
    if status != 0:
        detail = load().gm_last_error()
        raise GMError(name, status, detail.decode() if detail else "")
    return status


def ptr(t):
    """Raw device pointer of a CUDA tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("gmaster_b200 kernels take CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda():
    """Raise unless a CUDA device is available (the product path has no CPU fallback)."""
    load()
    if not torch.cuda.is_available():
        raise RuntimeError("gmaster_b200 needs a CUDA device (no CPU fallback)")
