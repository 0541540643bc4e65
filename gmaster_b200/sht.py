"""HEALPix spherical-harmonic transforms on the GPU (host driver of the CUDA kernels).

A transform is two separable stages, each a hand-written sm_100a kernel:

    maps --[ring FFT, ring.cu]--> ring spectra --[hemisphere pack]--> rhs(m, lane)
         --[Legendre contraction, legendre.cu / legendre_tc.cu]--> alm(l, m)

and ``map2alm`` adds NaMaster's Jacobi refinement ``alm <- alm - A(S(alm) - map)``
(gmaster/_sht/healpix.py:1059-1068).  Inside the loop the residual is formed in
lane space by the ring fold (`gm_fold_residual`), so no ring FFT runs in the loop
(the reference's ring-fold residual, gmaster/_native/cuda/march_v2.cu:409-493).

Precision modes: ``"fp64"`` keeps every stage in double precision (the plain FP64
path); ``"mixed"`` runs the ring stage and the contraction in single precision (or
BF16-split tensor-core products, see legendre_tc.cu) with the recurrence, seeds,
normalisation, alm accumulation and refinement update in double precision.
"""

import math
import threading

import numpy as np
import torch

from . import _lib, autotune

_PLANS = {}
_PLAN_LOCK = threading.Lock()

# Optional kernel timer: when set to a list, every Legendre launch appends
# (kind, start_event, end_event, algorithmic_flops) recorded on the current stream.
TIMER = None


def legendre_flops(plan, spin, ncomp):
    """Algorithmic flops of one Legendre pass: one complex MAC (4 flops) per
    (l, m, northern lane) per map for spin 0 (4 N_north L(L+1)/2 per map), and per
    (l, m in (-L, L), ring) per (Q, U) pair for spin 2 (4 nring L^2)."""
    if spin == 0:
        return 4.0 * plan.nlanes * plan.L * (plan.L + 1) / 2 * ncomp
    return 4.0 * plan.nring * plan.L * plan.L * (ncomp // 2)


def _timed(kind, plan, spin, ncomp, fn):
    if TIMER is None:
        fn()
        return
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    fn()
    end.record()
    TIMER.append((kind, start, end, legendre_flops(plan, spin, ncomp)))


# ----------------------------------------------------------------------------- geometry

def ring_geometry(nside):
    """HEALPix RING geometry, bit-identical to the reference (gmaster/utils.py:223-249).

    Returns ``theta, phi0, nphi, offsets`` for the ``4 nside - 1`` rings, computed
    with the same numpy operations in the same order as the reference.
    """
    nring = 4 * nside - 1
    rings = np.arange(1, 4 * nside)
    north = np.where(rings > 2 * nside, 4 * nside - rings, rings)
    cap = north < nside
    npix = 12 * nside ** 2
    theta = np.empty(nring)
    phi0 = np.empty(nring)
    nphi = np.empty(nring, dtype=np.uint64)
    theta[cap] = 2 * np.arcsin(north[cap] / (np.sqrt(6) * nside))
    phi0[cap] = np.pi / (4 * north[cap])
    nphi[cap] = 4 * north[cap]
    theta[~cap] = np.arccos((2 * nside - north[~cap]) * (8 * nside / npix))
    phi0[~cap] = np.pi / (4 * nside) * (((north[~cap] - nside) & 1) == 0)
    nphi[~cap] = 4 * nside
    south = north != rings
    theta[south] = np.pi - theta[south]
    offsets = np.concatenate([[0], np.cumsum(nphi)[:-1]]).astype(np.uint64)
    return theta, phi0, nphi, offsets


def shifted_flags(nside):
    """1 where a ring's first pixel sits at phi0 = pi / nphi, 0 where phi0 = 0."""
    _, phi0, nphi, _ = ring_geometry(nside)
    flags = (phi0 != 0).astype(np.uint8)
    # every HEALPix ring has phi0 in {0, pi / nphi}; the kernels rely on it
    shifted = np.pi / nphi.astype(np.float64)
    if not np.all((phi0 == 0) | np.isclose(phi0, shifted, rtol=0, atol=1e-15)):
        raise AssertionError("unexpected HEALPix ring phase")
    return flags


def lane_geometry(nside):
    """(3, 2 nside) float64: cos(theta), log2 sin(theta/2), log2 cos(theta/2) of the
    northern rings 1..2 nside (the last lane is the equator)."""
    theta = ring_geometry(nside)[0][: 2 * nside]
    return np.stack([np.cos(theta), np.log2(np.sin(theta / 2)), np.log2(np.cos(theta / 2))])


def _log2_int(n):
    b = n.bit_length()
    if b <= 53:
        return math.log2(n)
    shift = b - 53
    return shift + math.log2(n >> shift)


MAX_SPIN = 8   # spins 1..MAX_SPIN run through the polarised SIMT kernels


def seed_table(L, max_spin=MAX_SPIN):
    """Seeds of the Wigner-d rows: (2 max_spin + 1 variants, L orders, 4) float64.

    Variant 0 is spin 0 (s' = 0); spin s >= 1 has the pair of variants from
    `seed_variant(s)`: first s' = -s (the sY_{+s} rows), then s' = +s multiplied by (-1)^s
    (the sign the E/B combination of the minus-m part carries, healpix.py:800-814, folded
    into the row).  Spin 2 keeps variants 1 and 2, spin 1 takes 3 and 4, spin s >= 3 takes
    2s - 1 and 2s.  Entry
    ``[log2 N, sign, pc, ps]`` gives the first row l0 = max(m, |s'|) as
    ``sign * 2^(log2 N + pc log2 cos(theta/2) + ps log2 sin(theta/2))`` with
    ``N = sqrt((2 l0 + 1)/4pi) sqrt(binomial)`` from the closed forms
    d^m_{m,s'} = (-1)^(m-s') sqrt(C(2m, m+s')) cos^(m+s') sin^(m-s') (m >= |s'|) and
    d^s_{m,+s} = sqrt(C(2s, s+m)) cos^(s+m) sin^(s-m),
    d^s_{m,-s} = (-1)^(m+s) sqrt(C(2s, s-m)) cos^(s-m) sin^(s+m) (m < s); the binomials
    are exact integers, so log2 N is accurate to the last bit.
    """
    out = np.zeros((2 * max_spin + 1, L, 4))
    c = 1  # C(2m, m)
    for m in range(L):
        if m > 0:
            c = c * (2 * m) * (2 * m - 1) // (m * m)
        lc = _log2_int(c)
        sign = -1.0 if (m & 1) else 1.0
        out[0, m] = [0.5 * lc + 0.5 * math.log2((2 * m + 1) / (4 * math.pi)), sign, m, m]
        for sp in range(1, max_spin + 1):
            flip = -1.0 if (sp & 1) else 1.0   # (-1)^s on the +s variant
            if m >= sp:
                # C(2m, m -+ s) = C(2m, m) prod_k (m - k) / (m + 1 + k), k < s
                num = math.prod(m - k for k in range(sp))
                den = math.prod(m + 1 + k for k in range(sp))
                lc2 = lc + math.log2(num) - math.log2(den)
                norm = 0.5 * lc2 + 0.5 * math.log2((2 * m + 1) / (4 * math.pi))
                sg = -sign if (sp & 1) else sign   # (-1)^(m + s)
                vm = seed_variant(sp)
                out[vm, m] = [norm, sg, m - sp, m + sp]
                out[vm + 1, m] = [norm, sg * flip, m + sp, m - sp]
            else:
                vm = seed_variant(sp)
                base = 0.5 * math.log2((2 * sp + 1) / (4 * math.pi))
                sg = -1.0 if ((m + sp) & 1) else 1.0
                out[vm, m] = [base + 0.5 * math.log2(math.comb(2 * sp, sp - m)), sg, sp - m, sp + m]
                out[vm + 1, m] = [base + 0.5 * math.log2(math.comb(2 * sp, sp + m)), flip,
                                  sp + m, sp - m]
    return out


def seed_variant(spin):
    """First of the two seed variants of spin >= 1 (s' = -s, then s' = +s)."""
    return 1 if spin == 2 else (3 if spin == 1 else 2 * spin - 1)


class Plan:
    """Device-resident constants of one (nside, lmax) geometry, cached per device."""

    def __init__(self, nside, lmax, device):
        _lib.require_cuda()
        self.nside, self.lmax, self.L = int(nside), int(lmax), int(lmax) + 1
        self.device = torch.device(device)
        self.npix = 12 * self.nside ** 2
        self.nring = 4 * self.nside - 1
        self.nlanes = 2 * self.nside
        self.nelem = self.L * (self.L + 1) // 2
        lib = _lib.load()
        cnt = lib.gm_ring_twiddle_count(self.nside)
        self.tw = torch.empty(cnt * 24, dtype=torch.uint8, device=self.device)
        _lib.call("gm_ring_twiddles", self.nside, _lib.ptr(self.tw), _lib.stream_handle(self.device))
        self.shifted = torch.from_numpy(shifted_flags(self.nside)).to(self.device)
        self.geom = torch.from_numpy(np.ascontiguousarray(lane_geometry(self.nside))).to(self.device)
        self.seeds = torch.from_numpy(np.ascontiguousarray(seed_table(self.L))).to(self.device)
        # healpy packing helpers (host)
        m = np.arange(self.L)
        self.mstart = m * (2 * self.lmax + 1 - m) // 2


def get_plan(nside, lmax, device=None):
    dev = torch.device(device if device is not None else "cuda")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    key = (int(nside), int(lmax), dev.index)
    with _PLAN_LOCK:
        plan = _PLANS.get(key)
        if plan is None:
            plan = Plan(nside, lmax, dev)
            _PLANS[key] = plan
    return plan


def _prec(precision):
    if precision in ("fp64", _lib.FP64):
        return _lib.FP64
    if precision in ("mixed", _lib.MIXED):
        return _lib.MIXED
    raise ValueError(f"unknown precision {precision!r} (use 'fp64' or 'mixed')")


def _real_dtype(prec):
    return torch.float64 if prec == _lib.FP64 else torch.float32


def _complex_dtype(prec):
    return torch.complex128 if prec == _lib.FP64 else torch.complex64


# ----------------------------------------------------------------------------- stages

def ring_analysis(plan, maps, prec, mask=None, out=None):
    """maps (ncomp, npix) float64/float32 CUDA -> ring spectra (ncomp, nring, L); `mask`
    (npix,) float64, if given, multiplies every map as it is read.  `out`, if given, is a
    contiguous (ncomp, nring, L) tensor of the precision's complex type to write into."""
    maps = maps.contiguous()
    ncomp = maps.shape[0]
    if mask is not None:
        mask = mask.to(torch.float64).contiguous()
        if mask.shape != (plan.npix,):
            raise ValueError("mask must be one HEALPix map of the same resolution")
    if out is not None:
        if (out.shape != (ncomp, plan.nring, plan.L) or out.dtype != _complex_dtype(prec)
                or not out.is_contiguous()):
            raise ValueError("out must be a contiguous (ncomp, nring, L) spectrum tensor")
        spec = out
    else:
        spec = torch.empty((ncomp, plan.nring, plan.L), dtype=_complex_dtype(prec), device=plan.device)
    scratch, sbytes = _ring_scratch(plan, prec)
    _lib.call("gm_ring_analysis_ws", prec, plan.nside, plan.L, ncomp, _lib.ptr(maps),
              maps.element_size(), _lib.ptr(mask) if mask is not None else None,
              _lib.ptr(plan.tw), _lib.ptr(plan.shifted), _lib.ptr(spec), _lib.ptr(scratch), sbytes,
              RING_TUNING["hcap_max"], RING_TUNING["bs_min"], _lib.stream_handle(plan.device))
    return spec


# Global-memory ring path: a scratch of two slots per SM for the rings that do not fit the
# shared-memory kernels (single precision above Nside 4096, double precision above Nside
# 2048).  The knobs lower the thresholds that send a ring there (0: the defaults); they
# exist for tests.
RING_TUNING = {"hcap_max": 0, "bs_min": 0}


def _ring_scratch(plan, prec):
    sc = getattr(plan, "_ring_scratch_buf", None)
    if sc is None:
        nslots = 2 * torch.cuda.get_device_properties(plan.device).multi_processor_count
        nbytes = int(_lib.load().gm_ring_big_scratch_bytes(plan.nside, nslots))
        sc = torch.empty(nbytes, dtype=torch.uint8, device=plan.device)
        plan._ring_scratch_buf = sc
    return sc, sc.numel()


def pack_rhs(plan, spec, prec):
    ncomp = spec.shape[0]
    rhs = torch.empty((plan.L, plan.nlanes, ncomp, 4), dtype=_real_dtype(prec), device=plan.device)
    _lib.call("gm_pack_rhs", prec, plan.nside, plan.L, ncomp, _lib.ptr(spec), _lib.ptr(rhs),
              _lib.stream_handle(plan.device))
    return rhs


def ck_args(plan, spin, prec):
    """Checkpoint-table arguments (segoff, state and shift of the s' = -s and +s variants,
    their lane-group masks or None)
    of the mixed-precision spin-0 / spin-2 Legendre kernels, whose rows then come from the
    single-precision difference form restarted every 128 rows (legendre_ck.cu); None for
    FP64, other spins, checkpoints switched off, or tables larger than their memory share
    (the rows then come from the FP64 recurrence)."""
    from . import sht_tc

    if prec != _lib.MIXED or spin not in (0, 2) or plan.lmax < 2 or not sht_tc.USE_CHECKPOINTS:
        return None
    nvar = 1 if spin == 0 else 2
    need = nvar * 9 * _lib.load().gm_ck_table_entries(plan.nside, plan.lmax, spin)
    if need > sht_tc.CK_MEMORY_SHARE * torch.cuda.get_device_properties(plan.device).total_memory:
        return None
    tp = sht_tc.get_tc_plan(plan.nside, plan.lmax, plan.device)
    tabs = sht_tc.ck_tables(tp, spin)
    if tabs is None:
        return None
    sa, sb = (0, 0) if spin == 0 else (-2, 2)
    a, b = tabs[sa], tabs[sb]
    ma, mb = sht_tc.ck_masks(tp, spin, sa), sht_tc.ck_masks(tp, spin, sb)
    masks = (_lib.ptr(ma[0]), _lib.ptr(mb[0])) if ma is not None and mb is not None else (None, None)
    return (_lib.ptr(tp.ck_segoff[spin]), _lib.ptr(a[0]), _lib.ptr(a[1]), _lib.ptr(b[0]), _lib.ptr(b[1])) + masks


def run_legendre(plan, spin, ncomp, prec, kind, tile, src, dst, scale=1.0, ck=None):
    """One Legendre pass (kind "ana": src = rhs, dst = alm; "syn": src = alm, dst = syn) with
    the given tile shape, through the checkpointed entries when `ck` (ck_args) is given."""
    st = _lib.stream_handle(plan.device)
    if kind == "ana":
        if ck is not None:
            _lib.call("gm_legendre_analysis_ck", spin, plan.nside, plan.lmax, ncomp, _lib.ptr(plan.geom),
                      _lib.ptr(src), _lib.ptr(dst), float(scale), *ck, tile, st)
        else:
            _lib.call("gm_legendre_analysis_tile", prec, spin, plan.nside, plan.lmax, ncomp,
                      _lib.ptr(plan.geom), _lib.ptr(plan.seeds), _lib.ptr(src), _lib.ptr(dst),
                      float(scale), tile, st)
    elif ck is not None:
        _lib.call("gm_legendre_synthesis_ck", spin, plan.nside, plan.lmax, ncomp, _lib.ptr(plan.geom),
                  _lib.ptr(src), _lib.ptr(dst), *ck, tile, st)
    else:
        _lib.call("gm_legendre_synthesis_tile", prec, spin, plan.nside, plan.lmax, ncomp,
                  _lib.ptr(plan.geom), _lib.ptr(plan.seeds), _lib.ptr(src), _lib.ptr(dst), tile, st)


def legendre_analysis(plan, spin, rhs, alm, scale, prec):
    ncomp = rhs.shape[2]
    tile = autotune.tile_for(plan, spin, ncomp, prec, "ana")
    ck = ck_args(plan, spin, prec)
    _timed(f"legendre_analysis_s{spin}", plan, spin, ncomp,
           lambda: run_legendre(plan, spin, ncomp, prec, "ana", tile, rhs, alm, scale, ck))


def legendre_synthesis(plan, spin, alm, ncomp, prec, out=None):
    syn = out if out is not None else torch.empty(
        (plan.L, plan.nlanes, ncomp, 4), dtype=_real_dtype(prec), device=plan.device)
    tile = autotune.tile_for(plan, spin, ncomp, prec, "syn")
    ck = ck_args(plan, spin, prec)
    _timed(f"legendre_synthesis_s{spin}", plan, spin, ncomp,
           lambda: run_legendre(plan, spin, ncomp, prec, "syn", tile, alm, syn, ck=ck))
    return syn


def fold_residual(plan, syn, rhs_map, prec, out=None):
    ncomp = syn.shape[2]
    res = out if out is not None else torch.empty_like(rhs_map)
    _lib.call("gm_fold_residual", prec, plan.nside, plan.L, ncomp, _lib.ptr(syn),
              _lib.ptr(rhs_map), _lib.ptr(plan.shifted), _lib.ptr(res),
              _lib.stream_handle(plan.device))
    return res


def ring_synthesis(plan, syn, prec):
    ncomp = syn.shape[2]
    maps = torch.empty((ncomp, plan.npix), dtype=torch.float64, device=plan.device)
    scratch, sbytes = _ring_scratch(plan, prec)
    _lib.call("gm_ring_synthesis_ws", prec, plan.nside, plan.L, ncomp, _lib.ptr(syn), _lib.ptr(plan.tw),
              _lib.ptr(plan.shifted), _lib.ptr(maps), _lib.ptr(scratch), sbytes,
              RING_TUNING["hcap_max"], RING_TUNING["bs_min"], _lib.stream_handle(plan.device))
    return maps


# ----------------------------------------------------------------------------- transforms

def map2alm_device(maps, spin, nside, lmax, n_iter, precision="mixed"):
    """Analysis of ``maps`` (ncomp, npix) on the GPU with ``n_iter`` Jacobi iterations.

    spin 0: ncomp independent maps -> (ncomp, nelem) complex128 alms.
    spin 2: ncomp = 2 nfields (Q, U pairs) -> (2 nfields, nelem) rows (E, B per field).
    """
    prec = _prec(precision)
    plan = get_plan(nside, lmax, maps.device)
    ncomp = maps.shape[0]
    if spin < 0 or spin > MAX_SPIN:
        raise NotImplementedError(f"transforms are implemented for spins 0..{MAX_SPIN}")
    if spin != 0 and ncomp % 2:
        raise ValueError("spin transforms take (Q, U) pairs")
    spec = ring_analysis(plan, maps, prec)
    rhs_map = pack_rhs(plan, spec, prec)
    del spec
    alm = torch.zeros((ncomp, plan.nelem), dtype=torch.complex128, device=plan.device)
    legendre_analysis(plan, spin, rhs_map, alm, 1.0, prec)
    if n_iter > 0:
        syn = torch.empty_like(rhs_map)
        res = torch.empty_like(rhs_map)
        for _ in range(int(n_iter)):
            legendre_synthesis(plan, spin, alm, ncomp, prec, out=syn)
            fold_residual(plan, syn, rhs_map, prec, out=res)
            legendre_analysis(plan, spin, res, alm, -1.0, prec)
    return alm


def alm2map_device(alm, spin, nside, lmax, precision="mixed"):
    """Synthesis of (nrows, nelem) complex128 alms -> (nrows, npix) float64 maps."""
    prec = _prec(precision)
    plan = get_plan(nside, lmax, alm.device)
    alm = alm.contiguous()
    ncomp = alm.shape[0]
    if spin < 0 or spin > MAX_SPIN:
        raise NotImplementedError(f"transforms are implemented for spins 0..{MAX_SPIN}")
    if spin != 0 and ncomp % 2:
        raise ValueError("spin synthesis takes (E, B) pairs")
    syn = legendre_synthesis(plan, spin, alm, ncomp, prec)
    return ring_synthesis(plan, syn, prec)
