"""Gaussian covariance of curved-sky pseudo-C_ell bandpowers (gmaster/covariance.py).

`NmtCovarianceWorkspace` holds the coupling kernels Xi of the narrow-kernel approximation
(NaMaster's; gmaster/covariance.py:197-406): the coupling blocks of the power spectra of
the mask products, from the same FP64 3j kernel as the mode-coupling matrices, divided
by 2 l' + 1.  `gaussian_covariance` evaluates the signed sums of (C C + C C) / 2 * Xi
terms of every output block and bins both sides in one CUDA kernel (`gm_cov_binned`),
then decouples with the LU factors of the two workspaces (covariance.py:479-575).
`get_iNKA_cell` gives the improved-NKA input spectra (covariance.py:970-1024).

Map-based spin-0 and spin-2 fields only: the catalog shot-noise terms and the flat-sky
variant of the reference are outside this build.
"""

import itertools

import numpy as np
import torch

from . import _lib, fits, sht
from .bins import NmtBin
from .utils import as_device
from .workspaces import (_BLOCK_MM, _BLOCK_PP, _BLOCK_TE, _BLOCK_TT, NmtWorkspace,
                         compute_coupled_cell, coupling_blocks, coupling_tt_toeplitz, pseudo_cl,
                         toeplitz_fill, toeplitz_sanity)

__all__ = ["NmtCovarianceWorkspace", "gaussian_covariance", "get_iNKA_cell"]

KERNEL_NAMES = ("00", "0s", "pp", "mm")
_FITS_LABELS = {"00": "00", "0s": "02", "pp": "22P", "mm": "22M"}
_WICK_SUFFIX = ("1122", "1221")

# Component family linking an output spin-2 x spin-2 pair (o1, o2) to an input pair
# (i1, i2), indexed by i2 + 2 i1 + 4 (o2 + 2 o1) (covariance.py:149-165).
_SPIN2_FAMILY = ("+", "--", "-+", "Z", "-+", "+", "Z", "-+",
                 "--", "Z", "+", "--", "Z", "--", "-+", "+")


def _family(n1, n2, out1, out2, in1, in2):
    """Which kernel family couples output components (out1, out2) of a field pair with
    n1, n2 components to input components (in1, in2): "0" (spin 0), "+", "-+", "--"
    (spin-2 combinations) or "Z" (no coupling)."""
    if n1 == 1 and n2 == 1:
        return "0"
    if n1 == 1:
        return "0" if out2 == in2 else "Z"
    if n2 == 1:
        return "0" if out1 == in1 else "Z"
    return _SPIN2_FAMILY[in2 + 2 * in1 + 4 * (out2 + 2 * out1)]


def _paired(first, second):
    """(sign, kernel) of the product of two families; (0, None) when they do not couple
    (covariance.py:177-189)."""
    pair = {first, second}
    if first == second == "0":
        return 1.0, "00"
    if pair == {"0", "+"}:
        return 1.0, "0s"
    if first == second == "+":
        return 1.0, "pp"
    if first == second and first in ("-+", "--"):
        return -1.0, "mm"
    if pair == {"-+", "--"}:
        return 1.0, "mm"
    return 0.0, None


def _kernel_spins(s1, s2, t1, t2):
    """Spin pair of the kernels a Wick contraction needs when it pairs fields of spins
    (s1, t1) and (s2, t2): both pairs spin 2 x spin 2 -> (2, 2); one of them -> (0, 2);
    neither -> (0, 0) (the table of covariance.py:266-283)."""
    both = (s1 == 2 and t1 == 2) + (s2 == 2 and t2 == 2)
    return {0: (0, 0), 1: (0, 2), 2: (2, 2)}[both]


def _mask_product_alm(first, second, cache):
    """Alms of the product of two fields' masks, transformed with the first field's mask
    resolution and n_iter_mask (covariance.py:47-90).  `cache` shares one transform among
    the four products when the fields share mask tensors."""
    if not first.is_compatible(second, strict=False):
        raise ValueError("Fields have incompatible pixelizations.")
    key = (tuple(sorted((id(first.get_mask()), id(second.get_mask())))), first.minfo.nside,
           second.minfo.nside if first.minfo != second.minfo else None, first.ainfo_mask.lmax,
           first.n_iter_mask, first.precision)
    if key in cache:
        return cache[key]
    mask_a = first.get_mask()
    if first.minfo == second.minfo:
        mask_b = second.get_mask()
    else:
        mask_b = sht.alm2map_device(second.get_mask_alms()[None], 0, first.minfo.nside,
                                    second.ainfo_mask.lmax, first.precision)[0]
    alm = sht.map2alm_device((mask_a * mask_b)[None], 0, first.minfo.nside,
                             first.ainfo_mask.lmax, first.n_iter_mask, first.precision)[0]
    cache[key] = alm
    return alm


def _kernels(cell, spins, lmax, l_toeplitz, l_exact, dl_band):
    """Coupling kernels Xi (blocks / (2 l' + 1)) of a mask-product spectrum for one spin
    pair (covariance.py:100-146); the kernels the pair does not need are None."""
    nw = min(cell.shape[0], 2 * lmax + 1)
    window = cell[:nw].contiguous()
    cols = (2.0 * torch.arange(lmax + 1, dtype=torch.float64, device=cell.device) + 1.0)[None, :]
    out = {name: None for name in KERNEL_NAMES}
    if spins == (0, 0):
        if l_toeplitz > 0:
            out["00"] = coupling_tt_toeplitz(window, lmax, l_toeplitz, l_exact, dl_band) / cols
        else:
            out["00"] = coupling_blocks(window, lmax, 1)[_BLOCK_TT] / cols
    elif spins == (0, 2):
        out["0s"] = coupling_blocks(window, lmax, 2)[_BLOCK_TE] / cols
    else:
        blocks = coupling_blocks(window, lmax, 12)
        out["pp"] = blocks[_BLOCK_PP] / cols
        out["mm"] = blocks[_BLOCK_MM] / cols
    if l_toeplitz > 0:
        for name in ("0s", "pp", "mm"):
            if out[name] is not None:
                out[name] = toeplitz_fill(out[name].contiguous(), lmax, l_toeplitz, l_exact,
                                          dl_band) / cols
    return {k: (None if v is None else v.contiguous()) for k, v in out.items()}


class NmtCovarianceWorkspace:
    """Coupling kernels for the Gaussian covariance of the spectra of (fla1, fla2) and
    (flb1, flb2) (covariance.py:197-660): same interface as the reference's."""

    def __init__(self, fla1=None, fla2=None, flb1=None, flb2=None, l_toeplitz=-1, l_exact=-1,
                 dl_band=-1, fname=None):
        if fname is not None:
            self.read_from(fname)
        elif fla1 is not None or fla2 is not None:
            self.compute_coupling_coefficients(fla1, fla2, flb1=flb1, flb2=flb2,
                                               l_toeplitz=l_toeplitz, l_exact=l_exact,
                                               dl_band=dl_band)

    @classmethod
    def from_fields(cls, fla1, fla2, flb1=None, flb2=None, **kwargs):
        return cls(fla1, fla2, flb1, flb2, **kwargs)

    @classmethod
    def from_file(cls, fname):
        return cls(fname=fname)

    def _post_init(self):
        self.nmaps = tuple(1 if s == 0 else 2 for s in self.spins)
        self.nclsa = self.nmaps[0] * self.nmaps[1]
        self.nclsb = self.nmaps[2] * self.nmaps[3]

    def compute_coupling_coefficients(self, fla1, fla2, flb1=None, flb2=None, l_toeplitz=-1,
                                      l_exact=-1, dl_band=-1):
        flb1 = fla1 if flb1 is None else flb1
        flb2 = fla2 if flb2 is None else flb2
        fields = (fla1, fla2, flb1, flb2)
        if any(f.spin not in (0, 2) for f in fields):
            raise ValueError("Covariance matrix estimation is only implemented for "
                             "spin-0 and spin-2 fields.")
        if any(getattr(f, "anisotropic_mask", False) for f in fields):
            raise NotImplementedError(
                "Covariance matrix estimation not implemented for anisotropic weights.")
        toeplitz_sanity(l_toeplitz, l_exact, dl_band, fla1.ainfo.lmax)
        if any(not fla1.is_compatible(f, strict=False) for f in fields[1:]):
            raise ValueError("Fields have incompatible pixelizations.")
        self.spins = tuple(int(f.spin) for f in fields)
        self.spin_a1, self.spin_a2, self.spin_b1, self.spin_b2 = self.spins
        self.lmax = fla1.ainfo.lmax
        self.lmax_mask = fla1.ainfo_mask.lmax
        self.l_toeplitz, self.l_exact, self.dl_band = int(l_toeplitz), int(l_exact), int(dl_band)
        self._post_init()
        cache = {}
        s11 = _mask_product_alm(fla1, flb1, cache)
        s22 = _mask_product_alm(fla2, flb2, cache)
        s12 = _mask_product_alm(fla1, flb2, cache)
        s21 = _mask_product_alm(fla2, flb1, cache)
        cell_1122 = pseudo_cl(s11[None], s22[None], self.lmax_mask)[0]
        cell_1221 = pseudo_cl(s12[None], s21[None], self.lmax_mask)[0]
        sa1, sa2, sb1, sb2 = self.spins
        pairs = (_kernel_spins(sa1, sa2, sb1, sb2), _kernel_spins(sa1, sa2, sb2, sb1))
        xi0 = _kernels(cell_1122, pairs[0], self.lmax, self.l_toeplitz, self.l_exact, self.dl_band)
        if pairs[1] == pairs[0] and torch.equal(cell_1221, cell_1122):
            xi1 = dict(xi0)   # one mask for all four fields: the contractions share kernels
        else:
            xi1 = _kernels(cell_1221, pairs[1], self.lmax, self.l_toeplitz, self.l_exact,
                           self.dl_band)
        self.xiSS = [xi0, xi1]

    # ------------------------------------------------------------------ covariance

    def _terms(self):
        """Flattened term table: per output block X = (ia nb + ib) nclsb + (ic nd + id) the
        (kernel, row of A, row of B, sign) of every non-zero term (covariance.py:407-429),
        with rows into the concatenated spectra [c11; c12; c21; c22]."""
        na, nb, nc, nd = self.nmaps
        off = (0, na * nc, na * nc + na * nd, na * nc + na * nd + nb * nc)
        kernels, kindex = [], {}
        rows, signs, bptr = [], [], [0]
        outputs = itertools.product(range(na), range(nb), range(nc), range(nd))
        for ia, ib, ic, id_ in outputs:
            inputs = itertools.product(range(na), range(nb), range(nc), range(nd), range(2))
            for iap, ibp, icp, idp, wick in inputs:
                if wick == 0:   # <a1 b1><a2 b2>
                    fa = _family(na, nc, ia, ic, iap, icp)
                    fb = _family(nb, nd, ib, id_, ibp, idp)
                    ra, rb = off[0] + icp + nc * iap, off[3] + idp + nd * ibp
                else:           # <a1 b2><a2 b1>
                    fa = _family(na, nd, ia, id_, iap, idp)
                    fb = _family(nb, nc, ib, ic, ibp, icp)
                    ra, rb = off[1] + idp + nd * iap, off[2] + icp + nc * ibp
                sign, name = _paired(fa, fb)
                xi = None if name is None else self.xiSS[wick][name]
                if xi is None:
                    continue
                if (wick, name) not in kindex:
                    kindex[wick, name] = len(kernels)
                    kernels.append(xi)
                rows.append((kindex[wick, name], ra, rb))
                signs.append(sign)
            bptr.append(len(rows))
        return kernels, rows, signs, bptr

    def gaussian_covariance(self, cla1b1, cla1b2, cla2b1, cla2b2, wa, wb=None, coupled=False):
        """Covariance of the two power spectra: (nbands_a ncls_a, nbands_b ncls_b) for the
        decoupled bandpowers, or ((lmax+1) ncls_a, (lmax+1) ncls_b) for the coupled
        pseudo-C_ell if `coupled`, bandpower (or l) index slowest (covariance.py:479-575)."""
        wb = wa if wb is None else wb
        na, nb, nc, nd = self.nmaps
        if wa.ncls != na * nb or wb.ncls != nc * nd:
            raise ValueError("Field spins do not match input workspaces")
        dev = wa.mcm_binned.device if wa.mcm_binned is not None else torch.device("cuda")
        cls = [as_device(c, torch.float64, dev) for c in (cla1b1, cla1b2, cla2b1, cla2b2)]
        expected = (na * nc, na * nd, nb * nc, nb * nd)
        if any(c.ndim != 2 or c.shape[0] != n for c, n in zip(cls, expected)):
            raise ValueError("Field spins do not match input power spectrum shapes")
        L = self.lmax + 1
        if any(c.shape[1] < L for c in cls):
            raise ValueError(f"Input C_ls have a weird length. Expected {L}, but got "
                             f"{tuple(c.shape[1] for c in cls)}.")
        if wa.lmax != self.lmax or wb.lmax != self.lmax:
            raise ValueError("Input workspaces have a different lmax than the covariance workspace")
        spec = torch.cat([c[:, :L] for c in cls]).contiguous()
        kernels, rows, signs, bptr = self._terms()
        nblocks = len(bptr) - 1
        st = _lib.stream_handle(dev)
        if kernels:
            xi = torch.stack(kernels).contiguous()
        else:
            xi = torch.zeros((1, L, L), dtype=torch.float64, device=dev)
        terms = torch.tensor(rows if rows else [(0, 0, 0)], dtype=torch.int32).to(dev)
        sg = torch.tensor(signs if signs else [0.0], dtype=torch.float64).to(dev)
        bp = torch.tensor(bptr, dtype=torch.int32).to(dev)
        if coupled:
            out = torch.empty((nblocks, L, L), dtype=torch.float64, device=dev)
            _lib.call("gm_cov_coupled", self.lmax, nblocks, _lib.ptr(xi), _lib.ptr(spec),
                      _lib.ptr(terms), _lib.ptr(sg), _lib.ptr(bp), _lib.ptr(out), st)
            nx, ny = L, L
        else:
            opa = wa.bins.device_operators(dev)
            opb = wb.bins.device_operators(dev)
            nx, ny = wa.nbands, wb.nbands
            out = torch.empty((nblocks, nx, ny), dtype=torch.float64, device=dev)
            _lib.call("gm_cov_binned", self.lmax, nblocks, _lib.ptr(xi), _lib.ptr(spec),
                      _lib.ptr(terms), _lib.ptr(sg), _lib.ptr(bp), nx, _lib.ptr(opa["ptr"]),
                      _lib.ptr(opa["ells"]), _lib.ptr(opa["wfl"]), ny, _lib.ptr(opb["ptr"]),
                      _lib.ptr(opb["ells"]), _lib.ptr(opb["wfl"]), _lib.ptr(out), st)
        cov = out.view(self.nclsa, self.nclsb, nx, ny).permute(2, 0, 3, 1)
        cov = cov.reshape(nx * self.nclsa, ny * self.nclsb)
        if coupled:
            return cov.contiguous()
        wa._lu.check()
        wb._lu.check()
        half = wb._lu.solve(cov.T.contiguous()).T
        return wa._lu.solve(half.contiguous())

    # ------------------------------------------------------------------ files

    def write_to(self, fname):
        """Write the kernels in the reference's FITS layout (covariance.py:578-608): a
        primary HDU CWSP_PRIMARY with the keywords, one image XI<label>_<1122|1221> per
        kernel."""
        if not hasattr(self, "xiSS"):
            raise RuntimeError("Must initialize workspace before writing")
        header = {"LMAX": self.lmax, "LMAX_MASK": self.lmax_mask, "SPIN_A1": self.spin_a1,
                  "SPIN_A2": self.spin_a2, "SPIN_B1": self.spin_b1, "SPIN_B2": self.spin_b2,
                  "L_TOEPLITZ": self.l_toeplitz, "L_EXACT": self.l_exact, "DL_BAND": self.dl_band}
        hdus = [{"kind": "image", "name": "CWSP_PRIMARY", "data": np.ones((1, 1)), "header": header}]
        for wick, suffix in enumerate(_WICK_SUFFIX):
            for name in KERNEL_NAMES:
                xi = self.xiSS[wick][name]
                if xi is not None:
                    hdus.append({"kind": "image", "name": f"XI{_FITS_LABELS[name]}_{suffix}",
                                 "data": xi.cpu().numpy()})
        fits.write(fname, hdus)

    def read_from(self, fname, device=None):
        """Read kernels written by `write_to` (covariance.py:610-658)."""
        dev = torch.device(device) if device is not None else torch.device("cuda")
        hdus = {h["name"]: h for h in fits.read(fname)}
        if "CWSP_PRIMARY" not in hdus:
            raise ValueError(f"{fname} is not a covariance workspace file")
        hdr = hdus["CWSP_PRIMARY"]["header"]
        self.lmax = int(hdr["LMAX"])
        self.lmax_mask = int(hdr.get("LMAX_MASK", self.lmax))
        self.spins = tuple(int(hdr.get(k, 0)) for k in ("SPIN_A1", "SPIN_A2", "SPIN_B1", "SPIN_B2"))
        self.spin_a1, self.spin_a2, self.spin_b1, self.spin_b2 = self.spins
        self.l_toeplitz = int(hdr.get("L_TOEPLITZ", -1))
        self.l_exact = int(hdr.get("L_EXACT", -1))
        self.dl_band = int(hdr.get("DL_BAND", -1))
        n = self.lmax + 1
        self.xiSS = []
        for suffix in _WICK_SUFFIX:
            kern = {}
            for name in KERNEL_NAMES:
                h = hdus.get(f"XI{_FITS_LABELS[name]}_{suffix}")
                if h is None:
                    kern[name] = None
                    continue
                if h["data"].shape != (n, n):
                    raise ValueError(f"XI{_FITS_LABELS[name]}_{suffix} shape does not match "
                                     "expected dimensions")
                kern[name] = torch.from_numpy(np.ascontiguousarray(h["data"])).to(dev)
            self.xiSS.append(kern)
        self._post_init()


def gaussian_covariance(cw, spin_a1, spin_a2, spin_b1, spin_b2, cla1b1, cla1b2, cla2b1, cla2b2,
                        wa, wb=None, coupled=False):
    """Module-level form of `NmtCovarianceWorkspace.gaussian_covariance` that checks the
    spins against the workspace's (covariance.py:916-948)."""
    if (spin_a1, spin_a2, spin_b1, spin_b2) != cw.spins:
        raise ValueError("Requested spins do not match those used to initialize the workspace")
    return cw.gaussian_covariance(cla1b1, cla1b2, cla2b1, cla2b2, wa, wb=wb, coupled=coupled)


def get_iNKA_cell(fla, flb, cl_guess=None, w=None):
    """Input spectra of the improved narrow-kernel approximation (covariance.py:970-1024):
    the coupled pseudo-C_ell (measured, or `cl_guess` coupled by `w`) divided by the mean
    of the product of the two masks."""
    if not fla.is_compatible(flb, strict=False):
        raise ValueError("Fields have incompatible pixelizations")
    if fla.minfo == flb.minfo:
        fsky = (fla.get_mask() * flb.get_mask()).mean()
    else:
        lmax = fla.ainfo_mask.lmax
        cell = pseudo_cl(fla.get_mask_alms()[None], flb.get_mask_alms()[None], lmax)[0]
        ell = torch.arange(lmax + 1, dtype=torch.float64, device=cell.device)
        fsky = ((2 * ell + 1) * cell).sum() / (4 * np.pi)
    if cl_guess is None:
        coupled = compute_coupled_cell(fla, flb)
    else:
        if w is None:
            bins = NmtBin.from_lmax_linear(fla.ainfo.lmax, max(fla.ainfo.lmax // 10, 1))
            w = NmtWorkspace.from_fields(fla, flb, bins)
        coupled = w.couple_cell(cl_guess)
    return coupled / fsky
