"""Map and harmonic-space utilities (the counterpart of ``gmaster.utils``).

Geometry: `NmtMapInfo` (HEALPix) and `NmtAlmInfo` (healpy-packed alm layout).
Transforms: `map2alm`, `alm2map`, `map2alm_pair` on the GPU (spin 0 and spin 2).
Masks: `mask_apodization` (C1 / C2 / Smooth, on the GPU).
Fixture helpers: `synfast_spherical`, `pix2vec_ring`.

Arrays are returned as CUDA ``torch.Tensor``s; inputs may be numpy arrays or tensors.
"""

import numpy as np
import torch

from . import _lib, sht
from ._config import (get_default_params, get_precision, nmt_params, set_n_iter_default,
                      set_precision, set_sht_calculator, set_tol_pinv_default)

__all__ = [
    "NmtAlmInfo", "NmtMapInfo", "alm2map", "map2alm", "map2alm_pair", "mask_apodization",
    "synfast_spherical", "pix2vec_ring", "nmt_params", "get_default_params",
    "set_n_iter_default", "set_tol_pinv_default", "set_precision", "get_precision",
    "set_sht_calculator", "as_device", "max_pixel_radius", "moore_penrose_pinvh",
]


def as_device(x, dtype=None, device=None):
    """numpy array / tensor -> contiguous CUDA tensor (no copy if already there)."""
    dev = torch.device(device) if device is not None else torch.device("cuda")
    if isinstance(x, torch.Tensor):
        t = x
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if t.device.type != "cuda":
        t = t.to(dev, non_blocking=False)
    return t.contiguous()


class NmtMapInfo:
    """HEALPix pixelisation (gmaster/utils.py:336-461).  CAR maps are not supported."""

    def __init__(self, wcs, axes):
        if wcs is not None:
            raise NotImplementedError("only HEALPix maps are supported")
        nside = 1
        while 12 * nside ** 2 != axes[0]:
            nside *= 2
            if nside > 65536:
                raise ValueError("Something is wrong with your input arrays")
        self.is_healpix = True
        self.nside = nside
        self.npix = 12 * nside ** 2
        self.nx = self.ny = -1
        theta, phi0, nphi, offsets = sht.ring_geometry(nside)
        self.theta, self.phi0, self.nphi, self.offsets = theta, phi0, nphi, offsets
        self.weight = 4 * np.pi / self.npix

    def __eq__(self, other):
        return isinstance(other, NmtMapInfo) and self.nside == other.nside

    def reform_map(self, maps):
        if maps.shape[-1] != self.npix:
            raise ValueError("Incompatible map!")
        return maps

    def get_lmax(self):
        return 3 * self.nside - 1


class NmtAlmInfo:
    """Healpy m-major packing, ``a_lm`` at ``mstart[m] + l`` (gmaster/utils.py:493-524)."""

    def __init__(self, lmax):
        self.lmax = int(lmax)
        self.mmax = self.lmax
        m = np.arange(self.mmax + 1)
        self.mstart = (m * (2 * self.lmax + 1 - m) // 2).astype(np.uint64)
        self.nelem = (self.lmax + 1) * (self.lmax + 2) // 2

    def __eq__(self, other):
        return isinstance(other, NmtAlmInfo) and self.lmax == other.lmax

    def ell_m(self):
        """(ell, m) of every packed coefficient (numpy int64)."""
        L = self.lmax + 1
        order = np.repeat(np.arange(L), L - np.arange(L))
        ell = np.arange(self.nelem) - self.mstart.astype(np.int64)[order]
        return ell, order


def map2alm(map, spin, map_info, alm_info, *, n_iter, precision=None):
    """Spherical-harmonic analysis with Jacobi refinement (gmaster/utils.py:556-605).

    map: (nmaps, npix), nmaps = 1 (spin 0) or 2 (spin 2, Q/U).  Returns (nmaps, nelem)
    complex128 on the GPU; for spin 2 the rows are E and B.
    """
    nmaps = 1 if spin == 0 else 2
    maps = as_device(map, torch.float64)
    if maps.ndim != 2 or tuple(maps.shape) != (nmaps, map_info.npix):
        raise ValueError("Input map has wrong shape")
    if spin < 0 or spin > alm_info.lmax:
        raise ValueError("spin must satisfy 0 <= spin <= lmax")
    return sht.map2alm_device(maps, spin, map_info.nside, alm_info.lmax, int(n_iter),
                              precision or get_precision())


def map2alm_pair(map_a, map_b, map_info, alm_info, *, n_iter, precision=None):
    """Two spin-0 maps in one shared latitudinal pass (gmaster/utils.py:608-642).

    The Legendre rows are generated once and contracted against both maps.
    Returns ``(alm_a, alm_b)``, each (1, nelem).
    """
    a = as_device(map_a, torch.float64)
    b = as_device(map_b, torch.float64)
    if a.shape != (1, map_info.npix) or b.shape != (1, map_info.npix):
        raise ValueError("shared-band pair expects two (1, npix) spin-0 maps")
    alm = sht.map2alm_device(torch.cat([a, b]), 0, map_info.nside, alm_info.lmax, int(n_iter),
                             precision or get_precision())
    return alm[0:1], alm[1:2]


def alm2map(alm, spin, map_info, alm_info, precision=None):
    """Spherical-harmonic synthesis (gmaster/utils.py:645-672): (nmaps, npix) float64."""
    nmaps = 1 if spin == 0 else 2
    a = as_device(alm, torch.complex128)
    if a.ndim != 2 or tuple(a.shape) != (nmaps, alm_info.nelem):
        raise ValueError("Input alm has wrong shape")
    if spin < 0 or spin > alm_info.lmax:
        raise ValueError("spin must satisfy 0 <= spin <= lmax")
    return sht.alm2map_device(a, spin, map_info.nside, alm_info.lmax, precision or get_precision())


# ----------------------------------------------------------------------------- fixtures

def pix2vec_ring(nside, pix=None):
    """Unit vectors of HEALPix RING pixel centres (the healpy pix2vec formulas)."""
    theta, phi0, nphi, offsets = sht.ring_geometry(nside)
    nphi = nphi.astype(np.int64)
    ring = np.repeat(np.arange(4 * nside - 1), nphi)
    within = np.arange(12 * nside ** 2) - offsets.astype(np.int64)[ring]
    phi = phi0[ring] + 2 * np.pi * within / nphi[ring]
    th = theta[ring]
    vec = np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)], axis=1)
    return vec if pix is None else vec[pix]


_APO_TABLES = {}


def _apo_ring_table(nside, device):
    """(5, nring) float64 [cos theta; sin theta; phi0; 2 pi / nphi; nphi / (2 pi)] of the
    rings on `device` (cached)."""
    key = (int(nside), device.index)
    tab = _APO_TABLES.get(key)
    if tab is None:
        theta, phi0, nphi, _ = sht.ring_geometry(nside)
        n = nphi.astype(np.float64)
        host = np.stack([np.cos(theta), np.sin(theta), phi0, 2 * np.pi / n, n / (2 * np.pi)])
        tab = torch.from_numpy(host).to(device)
        _APO_TABLES[key] = tab
    return tab


def max_pixel_radius(nside):
    """Upper bound of the angular distance from a HEALPix pixel centre to its pixel's edge.

    At the latitude of ring k the pixel vertices interleave with ring k's centres, half an
    azimuthal step (pi / nphi_k) from them.  A pixel of ring j has its vertices on the
    latitudes of rings j - 1, j and j + 1 (the poles beyond the first and last ring), each
    within half that latitude's step of the centre's longitude; the bound is the largest
    such distance over all rings.
    """
    theta, _, nphi, _ = sht.ring_geometry(nside)
    half = np.pi / nphi.astype(np.float64)
    north_t = np.concatenate([[0.0], theta[:-1]])
    north_h = np.concatenate([[0.0], half[:-1]])
    south_t = np.concatenate([theta[1:], [np.pi]])
    south_h = np.concatenate([half[1:], [0.0]])

    def dist(t1, t2, dphi):
        # great-circle angle between (t1, 0) and (t2, dphi), haversine form
        h = np.sin(0.5 * (t2 - t1)) ** 2 + np.sin(t1) * np.sin(t2) * np.sin(0.5 * dphi) ** 2
        return 2 * np.arcsin(np.sqrt(np.minimum(h, 1.0)))

    return float(max(dist(theta, north_t, north_h).max(), dist(theta, south_t, south_h).max(),
                     dist(theta, theta, half).max()))


def mask_apodization(mask_in, aposize, apotype="C1"):
    """Apodise a binary HEALPix mask on the GPU (gmaster/utils.py:61-147).

    A pixel counts as masked where the mask is <= 0.  With theta the angular distance from
    a pixel to the nearest masked pixel, theta_* = `aposize` (degrees) and
    x = sqrt((1 - cos theta) / (1 - cos theta_*)), unmasked pixels closer than theta_* are
    multiplied by x - sin(2 pi x) / (2 pi) ("C1") or (1 - cos(pi x)) / 2 ("C2").  The
    distance is exact over all masked pixels (the reference queries a k-d tree of their unit
    vectors; here the CUDA kernel walks the HEALPix rings, gm_mask_apodize).

    "Smooth": pixels within 2.5 theta_* of a masked pixel are zeroed, the result is
    smoothed with a Gaussian beam of standard deviation theta_* (map2alm with n_iter = 3,
    alm2map) and multiplied by the mask.  The reference selects the zeroed pixels with
    healpy's inclusive query_disc (pixels overlapping the discs, "maybe a few more"); here
    a pixel is zeroed when its centre lies within 2.5 theta_* + `max_pixel_radius(nside)`
    of a masked pixel's centre, which contains every overlapping pixel.

    Returns a numpy array for "C1"/"C2" when `mask_in` is not a tensor, else a CUDA tensor;
    "Smooth" always returns a CUDA tensor (the reference returns a device array there).
    """
    if apotype not in ("C1", "C2", "Smooth"):
        raise ValueError(
            f"Apodization type {apotype} unknown. Choose from ['C1', 'C2', 'Smooth']")
    if aposize < 0:
        raise ValueError("Apodization scale must be a positive number")
    as_numpy = not isinstance(mask_in, torch.Tensor) and apotype != "Smooth"
    if isinstance(mask_in, torch.Tensor) and mask_in.ndim != 1:
        raise ValueError("Mask must be a one-dimensional HEALPix map")
    if not isinstance(mask_in, torch.Tensor) and np.ndim(mask_in) != 1:
        raise ValueError("Mask must be a one-dimensional HEALPix map")
    _lib.require_cuda()
    mask = as_device(mask_in, torch.float64)

    def result(t):
        return t.cpu().numpy() if as_numpy else t

    if aposize == 0:
        return result(mask.clone())
    npix = mask.shape[0]
    nside = int(round(np.sqrt(npix / 12)))
    if 12 * nside * nside != npix:
        raise ValueError("Mask size is not a valid HEALPix map size")
    radius = np.radians(aposize)
    scale = 2.5 if apotype == "Smooth" else 1.2
    if int(4 * npix * (1 - np.cos(scale * radius))) < 2:
        raise ValueError("Your apodization scale is too small for this pixel size")
    if not bool((mask <= 0).any()):
        return result(mask.clone())
    dev = mask.device
    prev = torch.empty(npix, dtype=torch.int32, device=dev)
    nxt = torch.empty(npix, dtype=torch.int32, device=dev)
    out = torch.empty_like(mask)
    stream = _lib.stream_handle(dev)
    _lib.call("gm_mask_ring_runs", nside, _lib.ptr(mask), _lib.ptr(prev), _lib.ptr(nxt), stream)
    table = _apo_ring_table(nside, dev)
    if apotype == "Smooth":
        reach = min(2.5 * radius + max_pixel_radius(nside), np.pi)
        chord2 = 4.0 * np.sin(0.5 * reach) ** 2
        if reach >= np.pi:
            chord2 = 5.0   # every pixel is within reach
        _lib.call("gm_mask_apodize", nside, _lib.ptr(table), _lib.ptr(mask), _lib.ptr(prev),
                  _lib.ptr(nxt), float(chord2), 0.0, 2, _lib.ptr(out), stream)
        del prev, nxt
        lmax = 3 * nside - 1
        prec = get_precision()
        alm = sht.map2alm_device(out[None], 0, nside, lmax, 3, prec)
        ell = torch.from_numpy(NmtAlmInfo(lmax).ell_m()[0].astype(np.float64)).to(dev)
        beam = torch.exp(-0.5 * ell * (ell + 1) * radius ** 2)
        smoothed = sht.alm2map_device(alm * beam[None], 0, nside, lmax, prec)[0]
        return smoothed * mask
    threshold = 1 - np.cos(radius)
    _lib.call("gm_mask_apodize", nside, _lib.ptr(table), _lib.ptr(mask), _lib.ptr(prev),
              _lib.ptr(nxt), float(2 * threshold), float(threshold),
              0 if apotype == "C1" else 1, _lib.ptr(out), stream)
    return result(out)


def moore_penrose_pinvh(mat, tol_pinv):
    """Pseudo-inverse of a Hermitian matrix on the GPU (gmaster/utils.py:527-556): the
    eigenvalues below ``tol_pinv`` times the largest have their inverse set to zero; with
    ``tol_pinv`` None or <= 0 the ordinary inverse is returned."""
    t = mat if isinstance(mat, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(mat))
    m = as_device(t, torch.complex128 if t.is_complex() else torch.float64)
    if tol_pinv is None or tol_pinv <= 0:
        return torch.linalg.inv(m)
    vals, vecs = torch.linalg.eigh(m)
    inv = torch.where(vals >= tol_pinv * vals.max(), 1.0 / vals, torch.zeros_like(vals))
    return (vecs * inv[None, :]) @ vecs.conj().T


def gaussian_alm(cls, lmax, rng):
    """Gaussian alms (healpy packing) for spectra cls[(ncomp, >= lmax+1)] of independent or
    correlated fields; `cls` is (n, n, L) covariance or (L,) for one field."""
    cls = np.asarray(cls, dtype=np.float64)
    if cls.ndim == 1:
        cls = cls[None, None, :]
    n = cls.shape[0]
    L = lmax + 1
    info = NmtAlmInfo(lmax)
    ell, order = info.ell_m()
    z = (rng.normal(size=(n, info.nelem)) + 1j * rng.normal(size=(n, info.nelem))) / np.sqrt(2)
    z[:, order == 0] = z[:, order == 0].real * np.sqrt(2)
    cov = np.moveaxis(cls[:, :, :L], 2, 0)                      # (L, n, n)
    w, v = np.linalg.eigh(cov)
    root = v * np.sqrt(np.maximum(w, 0))[:, None, :]            # (L, n, n)
    out = np.empty((n, info.nelem), dtype=np.complex128)
    chunk = 1 << 22
    for s in range(0, info.nelem, chunk):
        r = root[ell[s:s + chunk]]                              # (c, n, n)
        out[:, s:s + chunk] = np.einsum("cij,jc->ic", r, z[:, s:s + chunk])
    return out


def synfast_spherical(nside, cls, spin_arr, seed=-1, beam=None, precision=None):
    """Gaussian realisation of fields with the given power spectra (gmaster/utils.py:823-927).

    spin_arr lists the spin of each field (0 or 2); `cls` holds the upper-triangular
    spectra in NaMaster order for the field components.  Returns a list of maps
    ((1, npix) for spin 0, (2, npix) for spin 2) as CUDA tensors.
    """
    spin_arr = list(spin_arr)
    ncomp = sum(1 if s == 0 else 2 for s in spin_arr)
    lmax = 3 * nside - 1
    L = lmax + 1
    cls = np.asarray(cls, dtype=np.float64)
    cov = np.zeros((ncomp, ncomp, L))
    k = 0
    for i in range(ncomp):
        for j in range(i, ncomp):
            row = cls[k][:L]
            cov[i, j, : len(row)] = row
            cov[j, i, : len(row)] = row
            k += 1
    rng = np.random.default_rng(None if seed < 0 else seed)
    alm = gaussian_alm(cov, lmax, rng)
    if beam is not None:
        info = NmtAlmInfo(lmax)
        ell, _ = info.ell_m()
        alm = alm * np.asarray(beam)[:, ell] if np.ndim(beam) == 2 else alm * np.asarray(beam)[ell]
    out = []
    ainfo = NmtAlmInfo(lmax)
    minfo = NmtMapInfo(None, (12 * nside ** 2,))
    c = 0
    for s in spin_arr:
        nm = 1 if s == 0 else 2
        out.append(alm2map(alm[c:c + nm], s, minfo, ainfo, precision=precision))
        c += nm
    return out
