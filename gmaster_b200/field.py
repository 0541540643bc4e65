"""Curved-sky fields (`NmtField`), the counterpart of gmaster/field.py:20-499.

Supported: HEALPix spin-0 and spin-2 fields with a beam, ``n_iter`` / ``n_iter_mask``,
``lmax`` / ``lmax_mask``, ``masked_on_input``, ``lite`` and E/B purification
(``purify_e`` / ``purify_b``, `pure.purify_alms`).  Contaminant templates and anisotropic
masks are outside this build and raise ``NotImplementedError``.
"""

import weakref

import numpy as np
import torch

from . import sht
from ._config import get_precision, nmt_params
from .utils import NmtAlmInfo, NmtMapInfo, as_device


# Mask alms shared by the fields built on the same mask tensor: a TQU estimator makes a
# spin-0 and a spin-2 field on one mask, and each would otherwise transform the mask.
# Keyed by the identity of the mask tensor (a weak reference confirms it is still the same
# object; the entry is dropped when the tensor is released), then by its in-place version
# counter and the transform parameters, so a mask changed in place is never served stale.
_MASK_ALMS = {}


def _mask_key(field):
    return (field.mask._version, field.ainfo_mask.lmax, field.n_iter_mask, field.precision)


def _cached_mask_alms(field):
    entry = _MASK_ALMS.get(id(field.mask))
    if entry is None or entry[0]() is not field.mask:
        return None
    return entry[1].get(_mask_key(field))


def _store_mask_alms(field, alms):
    key = id(field.mask)
    entry = _MASK_ALMS.get(key)
    if entry is None or entry[0]() is not field.mask:
        ref = weakref.ref(field.mask, lambda _r, k=key: _MASK_ALMS.pop(k, None))
        entry = (ref, {})
        _MASK_ALMS[key] = entry
    entry[1][_mask_key(field)] = alms


class NmtField:
    """A masked field: mask, maps and their spherical-harmonic coefficients.

    For spin-0 fields the field and its mask are analysed in one shared latitudinal
    pass (two maps contracted against the same generated Legendre rows), as the
    reference does (gmaster/field.py:266-289).
    """

    def __init__(self, mask, maps, *, spin=None, templates=None, beam=None, purify_e=False,
                 purify_b=False, n_iter=None, n_iter_mask=None, tol_pinv=None, wcs=None,
                 lmax=None, lmax_mask=None, masked_on_input=False, lite=False, mask_22=None,
                 mask_12=None, precision=None):
        if templates is not None:
            raise NotImplementedError("contaminant deprojection is not part of this build")
        if mask_22 is not None or mask_12 is not None:
            raise NotImplementedError("anisotropic masks are not part of this build")
        self.lite = bool(lite)
        self.precision = precision or get_precision()
        self.n_iter = nmt_params.n_iter_default if n_iter is None else int(n_iter)
        self.n_iter_mask = nmt_params.n_iter_mask_default if n_iter_mask is None else int(n_iter_mask)
        self.pure_e, self.pure_b = bool(purify_e), bool(purify_b)
        self.is_catalog = False
        self.anisotropic_mask = False
        self.alm = self.alm_mask = self.maps = self.temp = None
        self.n_temp = 0
        self._Nw = self._Nf = 0

        mask_t = as_device(mask, torch.float64)
        if mask_t.ndim != 1:
            raise ValueError("Mask must be a one-dimensional HEALPix map")
        self.minfo = NmtMapInfo(wcs, tuple(mask_t.shape))
        self.mask = mask_t
        lmax = self.minfo.get_lmax() if lmax is None else int(lmax)
        lmax_mask = self.minfo.get_lmax() if lmax_mask is None else int(lmax_mask)
        if lmax <= 0 or lmax_mask <= 0:
            raise ValueError("`lmax` and `lmax_mask` must be positive")
        self.ainfo = NmtAlmInfo(lmax)
        self.ainfo_mask = NmtAlmInfo(lmax_mask)
        if beam is None:
            self.beam = torch.ones(lmax + 1, dtype=torch.float64, device=mask_t.device)
        else:
            b = np.asarray(beam.cpu() if isinstance(beam, torch.Tensor) else beam, dtype=np.float64)
            if b.ndim != 1 or len(b) <= lmax:
                raise ValueError(f"Input beam must have at least {lmax + 1} elements "
                                 "given the input map resolution")
            self.beam = torch.from_numpy(np.ascontiguousarray(b[: lmax + 1])).to(mask_t.device)

        if maps is None:
            if spin is None:
                raise ValueError("Please supply field spin")
            self.spin = int(spin)
            self.nmaps = 1 if self.spin == 0 else 2
            return
        maps_t = as_device(maps, torch.float64)
        if maps_t.ndim == 1:
            maps_t = maps_t[None]
        if maps_t.shape[0] not in (1, 2):
            raise ValueError("Must supply 1 or 2 maps per field")
        if maps_t.shape[1] != self.minfo.npix:
            raise ValueError("Maps and mask have different sizes")
        if spin is None:
            spin = 0 if maps_t.shape[0] == 1 else 2
        if (spin == 0) != (maps_t.shape[0] == 1):
            raise ValueError("Spin-zero fields are associated with a single map")
        if spin < 0 or spin > sht.MAX_SPIN:
            raise NotImplementedError(f"fields of spin 0..{sht.MAX_SPIN} are implemented")
        self.spin = int(spin)
        self.nmaps = 1 if self.spin == 0 else 2
        pure_any = self.pure_e or self.pure_b
        if pure_any and self.spin != 2:
            raise ValueError("Purification only implemented for spin-2 fields")
        if pure_any and self.ainfo != self.ainfo_mask:
            raise ValueError("Pure fields require lmax == lmax_mask")
        maps_unmasked = None
        if pure_any:
            # field.py:196-206: the purification needs the maps before masking
            maps_unmasked = maps_t
            if masked_on_input:
                good = self.mask > 0
                den = torch.where(good, self.mask, torch.ones_like(self.mask))
                maps_unmasked = torch.where(good[None, :], maps_t / den[None, :], maps_t)
        if not masked_on_input:
            maps_t = maps_t * self.mask[None, :]
        if pure_any:
            from .pure import purify_alms

            self.alm = purify_alms(self, self.get_mask_alms(), maps_unmasked,
                                   (self.pure_e, self.pure_b))
            if not self.lite:
                self.maps = sht.alm2map_device(self.alm, 2, self.minfo.nside, self.ainfo.lmax,
                                               self.precision)
            return
        nside = self.minfo.nside
        cached = _cached_mask_alms(self)
        if cached is not None and not self.lite:
            self.alm_mask = cached
        if (self.spin == 0 and not self.lite and cached is None and self.ainfo == self.ainfo_mask
                and self.n_iter == self.n_iter_mask):
            both = sht.map2alm_device(torch.cat([maps_t, self.mask[None, :]]), 0, nside,
                                      self.ainfo.lmax, self.n_iter, self.precision)
            self.alm, self.alm_mask = both[0:1], both[1]
            _store_mask_alms(self, self.alm_mask)
        else:
            self.alm = sht.map2alm_device(maps_t, self.spin, nside, self.ainfo.lmax, self.n_iter,
                                          self.precision)
        if not self.lite:
            self.maps = maps_t

    def is_compatible(self, other, strict=True):
        if strict and self.minfo != other.minfo:
            return False
        return self.ainfo_mask == other.ainfo_mask and self.ainfo == other.ainfo

    def get_mask(self):
        return self.mask

    def get_maps(self):
        if self.maps is None:
            raise ValueError("Input maps unavailable for this field")
        return self.maps

    def get_alms(self):
        if self.alm is None:
            raise ValueError("Input alms unavailable for this field")
        return self.alm

    def get_templates(self):
        raise ValueError("Input templates unavailable for this field")

    def get_mask_alms(self):
        """Mask alms (nelem_mask,), computed on first call (gmaster/field.py:348-376)."""
        if self.alm_mask is None:
            alms = _cached_mask_alms(self)
            if alms is None:
                alms = sht.map2alm_device(self.mask[None, :], 0, self.minfo.nside, self.ainfo_mask.lmax,
                                          self.n_iter_mask, self.precision)[0]
                _store_mask_alms(self, alms)
            if not self.lite:
                self.alm_mask = alms
            return alms
        return self.alm_mask

    @property
    def Nw(self):
        return self._Nw

    @property
    def Nf(self):
        return self._Nf
