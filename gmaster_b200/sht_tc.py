"""Batched spherical-harmonic transforms on the tcgen05 tensor cores.

Many maps of one geometry share each generated Legendre row: spin 0 takes up to 32 maps
per launch, spin 2 up to 32 (Q, U) fields.  The ring stage, the hemisphere pack, the
ring-fold residual of the Jacobi refinement and the alm bookkeeping are the kernels of
``legendre_tc.cu``; the contraction runs as bf16 hi/lo three-term MMAs with FP32
accumulation in tensor memory and FP64 accumulation of the alms.
"""

import ctypes
import threading

import numpy as np
import torch

from . import _lib, sht

MAX_MAPS_SPIN0 = 32
MAX_FIELDS_SPIN2 = 32

# The checkpointed kernels (legendre_ck.cu) restart the single-precision recurrence from a
# per-geometry table every 128 rows; the tables of one geometry (all row variants) may take
# at most this share of the device memory, else the carried-state kernels run.
USE_CHECKPOINTS = True
CK_MEMORY_SHARE = 0.2
# lanes (2 Nside) of the largest geometry with checkpoint tables: 64 groups of 64 lanes
CK_MAX_LANES = 4096
# Skip the 64-lane groups whose checkpoint states are all zero (exact: their rows are zero);
# False runs every group, for comparisons.
USE_TILE_SKIP = True

_TC_PLANS = {}
_LOCK = threading.Lock()


class TCPlan:
    """Device constants of the batched path for one (nside, lmax) geometry."""

    def __init__(self, plan):
        self.plan = plan
        lmax, dev = plan.lmax, plan.device
        self.coef = {}
        self.choff = {}
        self.choff_host = {}
        self.nchunks = {}
        lib = _lib.load()
        for spin in (0, 2):
            tab = torch.empty((plan.nelem, 4), dtype=torch.float64, device=dev)
            _lib.call("gm_tc_coef_table", lmax, spin, _lib.ptr(tab), _lib.stream_handle(dev))
            self.coef[spin] = tab
            host = np.zeros(plan.L + 1, dtype=np.int64)
            _lib.call("gm_tc_syn_chunk_offsets", lmax, spin, host.ctypes.data_as(ctypes.c_void_p))
            self.choff[spin] = torch.from_numpy(host).to(dev)
            self.choff_host[spin] = host
            self.nchunks[spin] = int(host[-1])
        # checkpoint tables: segment / unit offsets and relative synthesis chunks per spin;
        # the tables themselves are built on first use (`ck_tables`)
        self.ck_segoff, self.ck_uoff, self.ck_choff, self.ck_nchunks = {}, {}, {}, {}
        self.ck = {}
        self.ck_masks = {}
        self.ck_entries = {}
        for spin in (0, 2):
            seg = np.zeros(plan.L + 1, dtype=np.int64)
            uo = np.zeros(plan.L + 1, dtype=np.int64)
            _lib.call("gm_ck_offsets", lmax, spin, seg.ctypes.data_as(ctypes.c_void_p),
                      uo.ctypes.data_as(ctypes.c_void_p))
            self.ck_segoff[spin] = torch.from_numpy(seg).to(dev)
            self.ck_uoff[spin] = torch.from_numpy(uo).to(dev)
            self.ck_entries[spin] = int(seg[-1]) * plan.nlanes
            ch = np.zeros(plan.L + 1, dtype=np.int64)
            _lib.call("gm_ck_syn_chunk_offsets", lmax, spin, ch.ctypes.data_as(ctypes.c_void_p))
            self.ck_choff[spin] = torch.from_numpy(ch).to(dev)
            self.ck_nchunks[spin] = int(ch[-1])
        self.nctas = torch.cuda.get_device_properties(dev).multi_processor_count
        self.img_bytes = lib.gm_tc_ana_image_bytes(plan.nside, lmax)
        self.img_bytes_per_order = lib.gm_tc_ana_image_bytes(plan.nside, 0)
        self.scratch = torch.empty(lib.gm_tc_ana_scratch_bytes(plan.nside, self.nctas) // 8,
                                   dtype=torch.float64, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)


def get_tc_plan(nside, lmax, device=None):
    plan = sht.get_plan(nside, lmax, device)
    key = (plan.nside, plan.lmax, plan.device.index)
    with _LOCK:
        tp = _TC_PLANS.get(key)
        if tp is None:
            tp = TCPlan(plan)
            _TC_PLANS[key] = tp
    return tp


def _variants(spin):
    return (0,) if spin == 0 else (-2, 2)


def ck_table_bytes(tp, spin):
    """Bytes of the checkpoint tables of both row variants of `spin` (state float2 + shift)."""
    return len(_variants(spin)) * tp.ck_entries[spin] * 9


def ck_tables(tp, spin):
    """{s': (state, shift)} checkpoint tables of the row variants of `spin`, built on the
    first call and kept with the plan; None when checkpoints are switched off, the geometry
    has more than CK_MAX_LANES lanes (the checkpointed analysis walks a unit's lane groups as
    one 64-bit word) or its tables would take more than CK_MEMORY_SHARE of the device
    memory.  Without tables the transforms take the carried-recurrence kernels."""
    if not USE_CHECKPOINTS:
        return None
    p = tp.plan
    if p.nlanes > CK_MAX_LANES:
        return None
    with _LOCK:
        have = tp.ck.get(spin)
        if have is not None:
            return have
        total = torch.cuda.get_device_properties(p.device).total_memory
        built = sum(ck_table_bytes(tp, s) for s in tp.ck)
        if built + ck_table_bytes(tp, spin) > CK_MEMORY_SHARE * total:
            return None
        out = {}
        for sp in _variants(spin):
            state = torch.empty((tp.ck_entries[spin], 2), dtype=torch.float32, device=p.device)
            shift = torch.empty(tp.ck_entries[spin], dtype=torch.uint8, device=p.device)
            _lib.call("gm_ck_build", p.nside, p.lmax, spin, sp, _lib.ptr(p.geom), _lib.ptr(p.seeds),
                      _lib.ptr(tp.coef[spin]), _lib.ptr(tp.ck_segoff[spin]), _lib.ptr(state),
                      _lib.ptr(shift), _lib.stream_handle(p.device))
            out[sp] = (state, shift)
        tp.ck[spin] = out
        masks = {}
        if p.nlanes <= 4096:
            for sp, (state, shift) in out.items():
                seg_mask = torch.empty(int(_lib.load().gm_ck_segments(p.lmax, spin)), dtype=torch.int64,
                                       device=p.device)
                unit_mask = torch.empty(int(tp.ck_uoff[spin][-1].item()), dtype=torch.int64, device=p.device)
                _lib.call("gm_ck_masks", p.nside, p.lmax, spin, _lib.ptr(state), _lib.ptr(shift),
                          _lib.ptr(tp.ck_segoff[spin]), _lib.ptr(tp.ck_uoff[spin]), _lib.ptr(seg_mask),
                          _lib.ptr(unit_mask), _lib.stream_handle(p.device))
                masks[sp] = (seg_mask, unit_mask)
        tp.ck_masks[spin] = masks
        return out


def ck_masks(tp, spin, sp):
    """(seg_mask, unit_mask) of the row variant's checkpoint table, or None (tile skipping
    off, or a geometry above Nside 2048)."""
    if not USE_TILE_SKIP:
        return None
    return getattr(tp, "ck_masks", {}).get(spin, {}).get(sp)


def _rows(spin, ncomp):
    """(H, NR): rows per half and interleaved alm rows."""
    H = 2 * ncomp if spin == 0 else ncomp
    return H, (H if spin == 0 else 2 * H)


# Largest operand entry after scaling: 2^13 leaves headroom for the f16 range (65504)
# in the Jacobi residuals and the spin-2 row combinations.
_TARGET_LOG2 = 13


def pow2_scale(t):
    """Power of two that brings max |t| to about 2^13 (1.0 for an all-zero tensor)."""
    lo, hi = torch.aminmax(t)
    amax = max(abs(float(lo)), abs(float(hi)))
    if not amax > 0.0 or not np.isfinite(amax):
        return 1.0
    return float(2.0 ** (_TARGET_LOG2 - int(np.ceil(np.log2(amax)))))


def _check(tp):
    if int(tp.err.item()):
        tp.err.zero_()
        raise RuntimeError("tensor-core Legendre kernel: a bounded wait timed out")


class _Batch:
    """Buffers of one batched transform."""

    def __init__(self, tp, spin, ncomp, images=True):
        p = tp.plan
        self.tp, self.spin, self.ncomp = tp, spin, ncomp
        self.H, self.NR = _rows(spin, ncomp)
        self.alm_i = None
        self.img_scale = 1.0
        self.img = [torch.empty(tp.img_bytes, dtype=torch.uint8, device=p.device)
                    for _ in _variants(spin)] if images else []

    def zero_alm(self):
        p = self.tp.plan
        self.alm_i = torch.zeros((p.nelem, self.NR), dtype=torch.float64, device=p.device)

    def analysis(self, scale):
        """alm_i += scale * analysis of the images (which carry img_scale)."""
        p, tp = self.tp.plan, self.tp
        ck = ck_tables(tp, self.spin)
        for sp, img in zip(_variants(self.spin), self.img):
            if ck is not None:
                mk = ck_masks(tp, self.spin, sp)
                common = (p.nside, p.lmax, self.spin, sp, self.ncomp, _lib.ptr(p.geom),
                          _lib.ptr(tp.coef[self.spin]), _lib.ptr(tp.ck_segoff[self.spin]),
                          _lib.ptr(tp.ck_uoff[self.spin]), _lib.ptr(ck[sp][0]), _lib.ptr(ck[sp][1]))
                rest = (_lib.ptr(img), _lib.ptr(self.alm_i), float(scale) / self.img_scale, tp.nctas,
                        _lib.ptr(tp.err), _lib.stream_handle(p.device))
                if mk is not None:
                    _lib.call("gm_ck_analysis_masked", *common, _lib.ptr(mk[1]), *rest)
                else:
                    _lib.call("gm_ck_analysis", *common, *rest)
                continue
            _lib.call("gm_tc_analysis", p.nside, p.lmax, self.spin, sp, self.ncomp, _lib.ptr(p.geom),
                      _lib.ptr(p.seeds), _lib.ptr(tp.coef[self.spin]), _lib.ptr(img),
                      _lib.ptr(self.alm_i), float(scale) / self.img_scale, _lib.ptr(tp.scratch),
                      tp.nctas, _lib.ptr(tp.err), _lib.stream_handle(p.device))

    def synthesis(self, synd=None):
        """-> list of synd tensors (L, nlanes, 2H) float32, one per row variant."""
        p, tp = self.tp.plan, self.tp
        ck = ck_tables(tp, self.spin)
        nch = tp.nchunks[self.spin] if ck is None else tp.ck_nchunks[self.spin]
        simg_bytes = _lib.load().gm_tc_syn_image_bytes(nch)
        simg = torch.empty(simg_bytes, dtype=torch.uint8, device=p.device)
        outs = synd if synd is not None else [
            torch.empty((p.L, p.nlanes, 2 * self.H), dtype=torch.float32, device=p.device)
            for _ in _variants(self.spin)]
        alm_scale = pow2_scale(self.alm_i)
        for sp, out in zip(_variants(self.spin), outs):
            if ck is not None:
                _lib.call("gm_ck_prep_syn", p.lmax, self.spin, sp, self.ncomp, _lib.ptr(self.alm_i),
                          _lib.ptr(tp.ck_choff[self.spin]), _lib.ptr(simg), simg_bytes, alm_scale,
                          _lib.stream_handle(p.device))
                mk = ck_masks(tp, self.spin, sp)
                common = (p.nside, p.lmax, self.spin, sp, self.ncomp, _lib.ptr(p.geom),
                          _lib.ptr(tp.coef[self.spin]), _lib.ptr(tp.ck_segoff[self.spin]),
                          _lib.ptr(ck[sp][0]), _lib.ptr(ck[sp][1]))
                rest = (_lib.ptr(simg), _lib.ptr(tp.ck_choff[self.spin]), _lib.ptr(out), 1.0 / alm_scale,
                        _lib.ptr(tp.err), _lib.stream_handle(p.device))
                if mk is not None:
                    _lib.call("gm_ck_synthesis_masked", *common, _lib.ptr(mk[0]), *rest)
                else:
                    _lib.call("gm_ck_synthesis", *common, *rest)
                continue
            _lib.call("gm_tc_prep_syn", p.lmax, self.spin, sp, self.ncomp, _lib.ptr(self.alm_i),
                      _lib.ptr(tp.choff[self.spin]), _lib.ptr(simg), simg_bytes, alm_scale,
                      _lib.stream_handle(p.device))
            _lib.call("gm_tc_synthesis", p.nside, p.lmax, self.spin, sp, self.ncomp, _lib.ptr(p.geom),
                      _lib.ptr(p.seeds), _lib.ptr(tp.coef[self.spin]), _lib.ptr(simg),
                      _lib.ptr(tp.choff[self.spin]), _lib.ptr(out), 1.0 / alm_scale,
                      _lib.ptr(tp.err), _lib.stream_handle(p.device))
        return outs

    def to_api(self):
        p = self.tp.plan
        nfield = self.ncomp if self.spin == 0 else self.ncomp // 2
        out = torch.empty((self.ncomp, p.nelem), dtype=torch.complex128, device=p.device)
        _lib.call("gm_tc_alm_layout", p.lmax, self.spin, nfield, _lib.ptr(self.alm_i), _lib.ptr(out), 1,
                  _lib.stream_handle(p.device))
        return out

    def from_api(self, alm):
        p = self.tp.plan
        nfield = self.ncomp if self.spin == 0 else self.ncomp // 2
        alm = alm.contiguous()
        _lib.call("gm_tc_alm_layout", p.lmax, self.spin, nfield, _lib.ptr(self.alm_i), _lib.ptr(alm), 0,
                  _lib.stream_handle(p.device))


def _check_batch(spin, ncomp):
    if spin == 0 and not 1 <= ncomp <= MAX_MAPS_SPIN0:
        raise ValueError(f"spin-0 batches hold 1..{MAX_MAPS_SPIN0} maps")
    if spin == 2 and not (ncomp % 2 == 0 and 2 <= ncomp <= 2 * MAX_FIELDS_SPIN2):
        raise ValueError(f"spin-2 batches hold 1..{MAX_FIELDS_SPIN2} (Q, U) fields")
    if spin not in (0, 2):
        raise NotImplementedError("only spin 0 and spin 2")


# Per-order buffers of an order window are sized to at most this many bytes.
WINDOW_BYTES = 24 << 30


def _syn_bytes_per_order(tp, spin, ncomp):
    """Largest synthesis image + output bytes of one order (order 0 has the most chunks)."""
    p = tp.plan
    H, _ = _rows(spin, ncomp)
    chunks0 = int(tp.choff_host[spin][1] - tp.choff_host[spin][0])
    return len(_variants(spin)) * (chunks0 * _lib.load().gm_tc_syn_image_bytes(1)
                                   + p.nlanes * 2 * H * 4)


def window_orders(tp, spin, ncomp, budget=None):
    """Orders per window so that the per-order buffers take at most `budget` bytes."""
    budget = WINDOW_BYTES if budget is None else int(budget)
    per = max(len(_variants(spin)) * tp.img_bytes_per_order, _syn_bytes_per_order(tp, spin, ncomp))
    return int(max(1, min(tp.plan.L, budget // per)))


def _full_path_bytes(tp, spin, ncomp, n_iter):
    """Peak device bytes of the single-window map2alm: the ring spectra, right-hand sides
    and images while packing; then (spectra released) the right-hand sides, images, alm
    accumulator and synthesis buffers."""
    p = tp.plan
    H, NR = _rows(spin, ncomp)
    nv = len(_variants(spin))
    spec = ncomp * p.nring * p.L * 8
    base = nv * tp.img_bytes + p.L * p.nlanes * ncomp * 16
    later = base + p.nelem * NR * 8
    if n_iter > 0:
        later += nv * p.L * p.nlanes * 2 * H * 4 + tp.nchunks[spin] * _lib.load().gm_tc_syn_image_bytes(1)
    return max(spec + base, later)


def map2alm_tc(maps, spin, nside, lmax, n_iter, mask=None, window=None, ring_spectra=None):
    """Batched analysis: maps (ncomp, npix) float64/float32 CUDA -> (ncomp, nelem) complex128
    (spin 2: rows E, B per field), with n_iter Jacobi iterations.  `mask` (npix,), if
    given, multiplies every map as the ring stage reads it.

    Device memory: the ring spectra are released before the alm accumulator is made, and
    the iteration buffers before the final alm layout, so the peak is the right-hand
    sides, their operand images, the alm accumulator and the synthesis outputs (about
    106 GB for 64 maps at Nside 2048) besides the caller's maps.  When that does not fit in
    the free device memory (or `window`, a number of orders, is given) the transform runs
    over windows of orders instead (`map2alm_tc_windowed`).  `ring_spectra`, if given, are
    the single-precision ring spectra of the (masked) maps, already computed (a caller
    that streams the maps in can transform each part as it arrives)."""
    ncomp = maps.shape[0]
    _check_batch(spin, ncomp)
    tp = get_tc_plan(nside, lmax, maps.device)
    p = tp.plan
    if window is None:
        free, _ = torch.cuda.mem_get_info(p.device)
        free += torch.cuda.memory_reserved(p.device) - torch.cuda.memory_allocated(p.device)
        if _full_path_bytes(tp, spin, ncomp, n_iter) > 0.95 * free:
            window = window_orders(tp, spin, ncomp)
    if window is not None:
        return map2alm_tc_windowed(maps, spin, nside, lmax, n_iter, mask=mask, window=window)
    if ring_spectra is not None and ring_spectra.shape != (ncomp, p.nring, p.L):
        raise ValueError("ring_spectra must be (ncomp, nring, L)")
    spec = ring_spectra if ring_spectra is not None else sht.ring_analysis(p, maps, _lib.MIXED, mask=mask)
    ring_spectra = None   # the spectra are released after packing unless the caller holds them
    b = _Batch(tp, spin, ncomp)
    # the spin-2 rows G_Q -+ i G_U are at most twice the largest ring value
    b.img_scale = pow2_scale(spec.view(torch.float32)) / (2.0 if spin else 1.0)
    rhs_map = torch.empty((p.L, p.nlanes, ncomp, 4), dtype=torch.float32, device=p.device)
    _lib.call("gm_tc_pack", p.nside, p.lmax, spin, ncomp, _lib.ptr(spec), _lib.ptr(rhs_map),
              _lib.ptr(b.img[0]), _lib.ptr(b.img[1]) if spin else None, b.img_scale,
              _lib.stream_handle(p.device))
    del spec
    b.zero_alm()
    sht._timed(f"tc_analysis_s{spin}", p, spin, ncomp, lambda: b.analysis(1.0))
    synd = None
    for _ in range(int(n_iter)):
        synd = _timed_syn(b, synd)
        _lib.call("gm_tc_fold", p.nside, p.lmax, spin, ncomp, _lib.ptr(synd[0]),
                  _lib.ptr(synd[1]) if spin else None, _lib.ptr(rhs_map), _lib.ptr(p.shifted),
                  _lib.ptr(b.img[0]), _lib.ptr(b.img[1]) if spin else None, b.img_scale,
                  _lib.stream_handle(p.device))
        sht._timed(f"tc_analysis_s{spin}", p, spin, ncomp, lambda: b.analysis(-1.0))
    del synd, rhs_map
    b.img = []
    out = b.to_api()
    _check(tp)
    return out


def _timed_syn(b, synd):
    box = []
    sht._timed(f"tc_synthesis_s{b.spin}", b.tp.plan, b.spin, b.ncomp, lambda: box.append(b.synthesis(synd)))
    return box[0]


def _analysis_windowed(b, spec, scale, window, imgs):
    """alm_i += scale * analysis of the ring spectra, one window of orders at a time."""
    tp, spin, ncomp = b.tp, b.spin, b.ncomp
    p = tp.plan
    img_scale = pow2_scale(spec.view(torch.float32)) / (2.0 if spin else 1.0)
    st = _lib.stream_handle(p.device)
    for m0 in range(0, p.L, window):
        m1 = min(p.L, m0 + window)
        _lib.call("gm_tc_pack_window", p.nside, p.lmax, spin, ncomp, _lib.ptr(spec), None,
                  _lib.ptr(imgs[0]), _lib.ptr(imgs[1]) if spin else None, img_scale, m0, m1, st)
        for sp, img in zip(_variants(spin), imgs):
            _lib.call("gm_tc_analysis_window", p.nside, p.lmax, spin, sp, ncomp, _lib.ptr(p.geom),
                      _lib.ptr(p.seeds), _lib.ptr(tp.coef[spin]), _lib.ptr(img), _lib.ptr(b.alm_i),
                      float(scale) / img_scale, _lib.ptr(tp.scratch), tp.nctas, m0, m1,
                      _lib.ptr(tp.err), st)


def _synthesis_windowed(b, window):
    """Ring coefficients syn (L, nlanes, ncomp, 4) float32 of the alm accumulator, one
    window of orders at a time."""
    tp, spin, ncomp = b.tp, b.spin, b.ncomp
    p = tp.plan
    H, _ = _rows(spin, ncomp)
    host = tp.choff_host[spin]
    st = _lib.stream_handle(p.device)
    syn = torch.empty((p.L, p.nlanes, ncomp, 4), dtype=torch.float32, device=p.device)
    wmax = max(int(host[min(p.L, m0 + window)] - host[m0]) for m0 in range(0, p.L, window))
    simg = torch.empty(max(1, wmax) * _lib.load().gm_tc_syn_image_bytes(1), dtype=torch.uint8,
                       device=p.device)
    synd = [torch.empty((window, p.nlanes, 2 * H), dtype=torch.float32, device=p.device)
            for _ in _variants(spin)]
    alm_scale = pow2_scale(b.alm_i)
    for m0 in range(0, p.L, window):
        m1 = min(p.L, m0 + window)
        nbytes = int(host[m1] - host[m0]) * _lib.load().gm_tc_syn_image_bytes(1)
        for sp, out in zip(_variants(spin), synd):
            _lib.call("gm_tc_prep_syn_window", p.lmax, spin, sp, ncomp, _lib.ptr(b.alm_i),
                      _lib.ptr(tp.choff[spin]), _lib.ptr(simg), nbytes, alm_scale, m0, m1, st)
            _lib.call("gm_tc_synthesis_window", p.nside, p.lmax, spin, sp, ncomp, _lib.ptr(p.geom),
                      _lib.ptr(p.seeds), _lib.ptr(tp.coef[spin]), _lib.ptr(simg),
                      _lib.ptr(tp.choff[spin]), _lib.ptr(out), 1.0 / alm_scale, m0, m1,
                      _lib.ptr(tp.err), st)
        _lib.call("gm_tc_synd_to_syn_window", p.nside, p.lmax, spin, ncomp, _lib.ptr(synd[0]),
                  _lib.ptr(synd[1]) if spin else None, _lib.ptr(syn), m0, m1, st)
    return syn


def map2alm_tc_windowed(maps, spin, nside, lmax, n_iter, mask=None, window=None):
    """map2alm_tc over windows of `window` orders, for geometries whose full-size operand
    buffers do not fit (Nside 4096 batches, Nside 8192).  The per-order buffers (operand
    images, synthesis images and outputs) hold one window; the Jacobi refinement takes its
    residual in map space (synthesis to the rings, S(alm) - mask * map, ring analysis)
    instead of the ring-fold, whose aliasing couples all orders."""
    ncomp = maps.shape[0]
    _check_batch(spin, ncomp)
    tp = get_tc_plan(nside, lmax, maps.device)
    p = tp.plan
    window = window_orders(tp, spin, ncomp) if window is None else int(max(1, min(p.L, window)))
    b = _Batch(tp, spin, ncomp, images=False)
    b.zero_alm()
    imgs = [torch.empty(window * tp.img_bytes_per_order, dtype=torch.uint8, device=p.device)
            for _ in _variants(spin)]
    spec = sht.ring_analysis(p, maps, _lib.MIXED, mask=mask)
    sht._timed(f"tc_analysis_s{spin}", p, spin, ncomp, lambda: _analysis_windowed(b, spec, 1.0, window, imgs))
    del spec
    for _ in range(int(n_iter)):
        box = []
        sht._timed(f"tc_synthesis_s{spin}", p, spin, ncomp,
                   lambda: box.append(_synthesis_windowed(b, window)))
        rec = sht.ring_synthesis(p, box.pop(), _lib.MIXED)
        if mask is None:
            rec.sub_(maps)
        else:
            rec.addcmul_(maps, mask[None, :].to(maps.dtype), value=-1.0)
        spec = sht.ring_analysis(p, rec, _lib.MIXED)
        del rec
        sht._timed(f"tc_analysis_s{spin}", p, spin, ncomp,
                   lambda: _analysis_windowed(b, spec, -1.0, window, imgs))
        del spec
    del imgs
    out = b.to_api()
    _check(tp)
    return out


def alm2map_tc(alm, spin, nside, lmax, window=None):
    """Batched synthesis: (nrows, nelem) complex128 -> (nrows, npix) float64 maps.  With
    `window` (a number of orders), or when the full-size buffers do not fit, the operand
    images and outputs hold one window of orders at a time."""
    ncomp = alm.shape[0]
    _check_batch(spin, ncomp)
    tp = get_tc_plan(nside, lmax, alm.device)
    p = tp.plan
    b = _Batch(tp, spin, ncomp, images=False)
    b.zero_alm()
    b.from_api(alm.to(torch.complex128))
    H, _ = _rows(spin, ncomp)
    if window is None:
        free, _ = torch.cuda.mem_get_info(p.device)
        free += torch.cuda.memory_reserved(p.device) - torch.cuda.memory_allocated(p.device)
        full = (len(_variants(spin)) * p.L * p.nlanes * 2 * H * 4
                + tp.nchunks[spin] * _lib.load().gm_tc_syn_image_bytes(1) + p.L * p.nlanes * ncomp * 16)
        if full > 0.9 * free:
            window = window_orders(tp, spin, ncomp)
    if window is not None:
        syn = _synthesis_windowed(b, int(max(1, min(p.L, window))))
        maps = sht.ring_synthesis(p, syn, _lib.MIXED)
        _check(tp)
        return maps
    synd = b.synthesis()
    syn = torch.empty((p.L, p.nlanes, ncomp, 4), dtype=torch.float32, device=p.device)
    _lib.call("gm_tc_synd_to_syn", p.nside, p.lmax, spin, ncomp, _lib.ptr(synd[0]),
              _lib.ptr(synd[1]) if spin else None, _lib.ptr(syn), _lib.stream_handle(p.device))
    maps = sht.ring_synthesis(p, syn, _lib.MIXED)
    _check(tp)
    return maps
