"""MASTER workspaces and pseudo-spectra (the counterpart of gmaster/workspaces.py).

`compute_coupled_cell` forms the coupled pseudo-C_ell (workspaces.py:86-125);
`NmtWorkspace` builds the mode-coupling matrix from the masks' pseudo-spectrum with
the FP64 Wigner-3j recursion kernel, bins it and LU-factors the binned matrix on the
GPU, and `decouple_cell` returns bandpowers (workspaces.py:1593-2147).
"""

import numpy as np
import torch

from . import _lib, fits
from .bins import NmtBin
from .utils import as_device

_BLOCK_TT, _BLOCK_TE, _BLOCK_PP, _BLOCK_MM = 0, 1, 2, 3


def pseudo_cl(alm1, alm2, lmax):
    """(n1, nelem) x (n2, nelem) complex128 -> (n1 n2, lmax+1) float64 on the GPU."""
    a = alm1 if alm1.ndim == 2 else alm1[None]
    b = alm2 if alm2.ndim == 2 else alm2[None]
    a = a.contiguous()
    b = b.contiguous()
    out = torch.empty((a.shape[0] * b.shape[0], lmax + 1), dtype=torch.float64, device=a.device)
    _lib.call("gm_pseudo_cl", lmax, a.shape[0], _lib.ptr(a), b.shape[0], _lib.ptr(b),
              _lib.ptr(out), _lib.stream_handle(a.device))
    return out


def compute_coupled_cell(f1, f2):
    """Coupled pseudo-C_ell of two fields: (n1 n2, lmax+1) (workspaces.py:98-125)."""
    if not f1.is_compatible(f2, strict=False):
        raise ValueError("You're trying to correlate incompatible fields")
    lmax = min(f1.ainfo.lmax, f2.ainfo.lmax)
    return pseudo_cl(f1.get_alms(), f2.get_alms(), lmax)


def coupling_blocks(window, lmax, which):
    """(4, lmax+1, lmax+1) coupling blocks [tt, te, pp, mm] from a mask spectrum."""
    w = as_device(window, torch.float64)
    blocks = torch.empty((4, lmax + 1, lmax + 1), dtype=torch.float64, device=w.device)
    queue = torch.zeros(1, dtype=torch.int64, device=w.device)
    _lib.call("gm_coupling_blocks", lmax, _lib.ptr(w), w.shape[0], which, _lib.ptr(blocks),
              _lib.ptr(queue), _lib.stream_handle(w.device))
    return blocks


def coupling_blocks_multi(windows, lmaxs, whiches):
    """Coupling blocks of many workspaces of different lmax in one persistent launch.

    ``windows`` is a list of float64 device mask spectra, ``lmaxs`` and ``whiches`` the
    lmax and block mask of each workspace.  Returns a list of (4, lmax+1, lmax+1) blocks,
    bit-identical to ``coupling_blocks`` of each workspace in turn (unused blocks are
    zero).  The jobs are queued by decreasing lmax so the longest recursions start first.
    """
    if len(windows) == 0:
        return []
    dev = windows[0].device
    wins = [as_device(w, torch.float64).contiguous() for w in windows]
    # workspaces with equal windows and lmax (the 0x0, 0x2 and 2x2 workspaces of one mask)
    # share one job computing the union of their blocks: each (l1, l2) recursion then runs
    # once, and every block equals the one of a separate job bit for bit
    groups = []   # [lmax, window, which, members]
    for i, w in enumerate(wins):
        lmax = int(lmaxs[i])
        for g in groups:
            if g[0] == lmax and g[1].shape == w.shape and torch.equal(g[1], w):
                g[2] |= int(whiches[i])
                g[3].append(i)
                break
        else:
            groups.append([lmax, w, int(whiches[i]), [i]])
    order = sorted(range(len(groups)), key=lambda k: -groups[k][0])
    rows, wparts, woff, boff, first = [], [], 0, 0, 0
    offsets = [None] * len(groups)
    for k in order:
        lmax, w, which, _ = groups[k]
        n = lmax + 1
        rows.append([lmax, woff, w.shape[0], which, boff, first])
        offsets[k] = boff
        wparts.append(w)
        woff += w.shape[0]
        boff += 4 * n * n
        first += int(_lib.load().gm_coupling_units(lmax))
    jobs = torch.tensor(rows, dtype=torch.int64).to(dev)
    allw = torch.cat(wparts) if woff else torch.zeros(1, dtype=torch.float64, device=dev)
    blocks = torch.zeros(boff, dtype=torch.float64, device=dev)
    queue = torch.zeros(1, dtype=torch.int64, device=dev)
    _lib.call("gm_coupling_blocks_multi", len(rows), _lib.ptr(jobs), first, _lib.ptr(allw),
              _lib.ptr(blocks), _lib.ptr(queue), _lib.stream_handle(dev))
    out = [None] * len(windows)
    for k, (lmax, _, _, members) in enumerate(groups):
        n = lmax + 1
        shared = blocks[offsets[k]:offsets[k] + 4 * n * n].view(4, n, n)
        # every workspace gets its own blocks (a Toeplitz fill edits them in place), with
        # the blocks it did not ask for zero
        for i in members[1:]:
            own = torch.zeros_like(shared)
            for x in range(4):
                if int(whiches[i]) & (1 << x):
                    own[x] = shared[x]
            out[i] = own
        for x in range(4):
            if not int(whiches[members[0]]) & (1 << x):
                shared[x].zero_()
        out[members[0]] = shared
    return out


def toeplitz_sanity(l_toeplitz, l_exact, dl_band, lmax):
    """Toeplitz parameter checks of the reference (workspaces.py:1125-1138); a no-op when
    ``l_toeplitz <= 0``."""
    if l_toeplitz <= 0:
        return
    if l_exact <= 0 or dl_band < 0:
        raise ValueError("`l_exact` and `dl_band` must be positive numbers")
    if l_exact > l_toeplitz:
        raise ValueError("`l_exact` must be `<= l_toeplitz")
    if l_toeplitz >= lmax or l_exact >= lmax or dl_band >= lmax:
        raise ValueError("`l_toeplitz`, `l_exact` and `dl_band` must be smaller than `l_max`")


def toeplitz_exact_pairs(n, l_toeplitz, l_exact, dl_band):
    """(npairs, 2) int32 array of the (l1 <= l2) pairs whose exact coupling the Toeplitz
    fill reads: the diagonal, column l_toeplitz, columns 0..l_exact and the dl_band
    off-diagonals (the pair set of workspaces.py:521-538)."""
    ell = np.arange(n)
    parts = [np.stack([ell, ell], 1), np.stack([ell, np.full(n, l_toeplitz)], 1)]
    for c in range(l_exact + 1):
        parts.append(np.stack([ell, np.full(n, c)], 1))
    for off in range(1, dl_band + 1):
        parts.append(np.stack([ell[: n - off], ell[: n - off] + off], 1))
    p = np.concatenate(parts)
    p = np.sort(p, axis=1)
    return np.unique(p, axis=0).astype(np.int32)


def toeplitz_fill(S, lmax, l_toeplitz, l_exact, dl_band):
    """Toeplitz approximation (times 2 l' + 1) from a symmetric S = block / (2 l' + 1)."""
    out = torch.empty_like(S)
    _lib.call("gm_toeplitz_fill", lmax, l_toeplitz, l_exact, dl_band, _lib.ptr(S.contiguous()),
              _lib.ptr(out), _lib.stream_handle(S.device))
    return out


def coupling_tt_toeplitz(window, lmax, l_toeplitz, l_exact, dl_band):
    """Scalar (TT) coupling block under the Toeplitz approximation: only the entries the
    fill reads are computed by the 3j recursion (workspaces.py:546-590)."""
    w = as_device(window, torch.float64)
    n = lmax + 1
    pairs = torch.from_numpy(toeplitz_exact_pairs(n, l_toeplitz, l_exact, dl_band)).to(w.device)
    S = torch.zeros((n, n), dtype=torch.float64, device=w.device)
    _lib.call("gm_coupling_pairs_tt", lmax, _lib.ptr(w), w.shape[0], _lib.ptr(pairs), pairs.shape[0],
              _lib.ptr(S), _lib.stream_handle(w.device))
    return toeplitz_fill(S, lmax, l_toeplitz, l_exact, dl_band)


def _blocks_from_dense(dense, lmax, ncls, device):
    """(4, L, L) blocks [tt, te, pp, mm] of a dense (ncls L)^2 coupling matrix in
    ``l * ncls + c`` order; the inverse of ``NmtWorkspace.get_coupling_matrix``.  Raises if
    the matrix does not have the structure of a spin 0x0, 0x2, 2x2 or joint TEB workspace."""
    n = lmax + 1
    d = np.asarray(dense, dtype=np.float64)
    if d.shape != (ncls * n, ncls * n):
        raise ValueError(f"coupling matrix of shape {d.shape}, expected {(ncls * n, ncls * n)}")
    if ncls not in (1, 2, 4, 7):
        raise ValueError(f"unsupported number of spectra {ncls}")
    q = d.reshape(n, ncls, n, ncls)
    blocks = np.zeros((4, n, n))
    seen = set()
    for x, r, c, sign in _slots(ncls):
        if x not in seen:
            blocks[x] = sign * q[:, r, :, c]
            seen.add(x)
    rebuilt = np.zeros_like(q)
    for x, r, c, sign in _slots(ncls):
        rebuilt[:, r, :, c] += sign * blocks[x]
    rebuilt = rebuilt.reshape(ncls * n, ncls * n)
    if not np.array_equal(rebuilt, d):
        raise NotImplementedError("the coupling matrix is not that of a standard spin 0x0, 0x2, "
                                  "2x2 or joint TEB workspace")
    return torch.from_numpy(blocks).to(device)


def _slot_blocks_from_dense(dense, lmax, ncls, device):
    """A block per standard slot of a dense (ncls L)^2 coupling matrix (purified workspaces,
    whose slots hold different blocks); raises if the matrix has entries off the slots."""
    n = lmax + 1
    d = np.asarray(dense, dtype=np.float64)
    if d.shape != (ncls * n, ncls * n):
        raise ValueError(f"coupling matrix of shape {d.shape}, expected {(ncls * n, ncls * n)}")
    q = d.reshape(n, ncls, n, ncls)
    rebuilt = np.zeros_like(q)
    out = []
    for _, r, c, sign in _slots(ncls):
        blk = sign * q[:, r, :, c]
        rebuilt[:, r, :, c] += sign * blk
        out.append((torch.from_numpy(np.ascontiguousarray(blk)).to(device), r, c, sign))
    if not np.array_equal(rebuilt.reshape(d.shape), d):
        raise NotImplementedError("the coupling matrix is not that of a spin 0x2, 2x2 or joint "
                                  "TEB workspace")
    return out


def _which(ncls):
    return {1: 1, 2: 2, 4: 12, 7: 15}[ncls]


_MM_SIGNS = (1.0, -1.0, -1.0, 1.0)


def _slots(ncls):
    """(block, row channel, column channel, sign) of every block placement in the
    (ncls L)^2 coupling matrix (workspaces.py:1856-1903): spin 0x0 [TT]; 0x2 [TE, TB];
    2x2 [EE, EB, BE, BB]; joint TEB [TT, TE, TB, EE, EB, BE, BB].  The EE..BB part takes
    M+ on its diagonal and M- on its anti-diagonal."""
    if ncls == 1:
        return [(_BLOCK_TT, 0, 0, 1.0)]
    if ncls == 2:
        return [(_BLOCK_TE, 0, 0, 1.0), (_BLOCK_TE, 1, 1, 1.0)]
    off = 3 if ncls == 7 else 0
    out = [(_BLOCK_TT, 0, 0, 1.0), (_BLOCK_TE, 1, 1, 1.0), (_BLOCK_TE, 2, 2, 1.0)] if ncls == 7 else []
    out += [(_BLOCK_PP, off + c, off + c, 1.0) for c in range(4)]
    out += [(_BLOCK_MM, off + c, off + 3 - c, _MM_SIGNS[c]) for c in range(4)]
    return out


class LUFactor:
    """FP64 LU factorisation with partial pivoting of a square device matrix."""

    # matrices above this order are factored in panels of _PANEL columns (the trailing
    # updates by the FP64 tile kernel gm_lu_update); smaller ones in one single-CTA kernel
    _BLOCKED_FROM = 256
    _PANEL = 64

    def __init__(self, a):
        self.n = a.shape[0]
        self.lu = a.contiguous().clone()
        self.piv = torch.empty(self.n, dtype=torch.int32, device=a.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=a.device)
        st = _lib.stream_handle(a.device)
        if self.n <= self._BLOCKED_FROM:
            _lib.call("gm_lu_factor", self.n, _lib.ptr(self.lu), _lib.ptr(self.piv),
                      _lib.ptr(self.status), st)
            return
        n, A = self.n, self.lu
        for k0 in range(0, n, self._PANEL):
            k1 = min(n, k0 + self._PANEL)
            _lib.call("gm_lu_panel", n, _lib.ptr(A), k0, k1, _lib.ptr(self.piv), _lib.ptr(self.status), st)
            if k1 < n:
                _lib.call("gm_lu_trsm", n, _lib.ptr(A), k0, k1, st)
                _lib.call("gm_lu_update", n, _lib.ptr(A), k0, k1, st)

    def check(self):
        st = int(self.status.item())
        if st:
            raise np.linalg.LinAlgError(f"binned coupling matrix is singular (pivot {st - 1})")

    def solve(self, b):
        """Solve A x = b for b of shape (n,) or (n, nrhs)."""
        x = b.contiguous().clone()
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        _lib.call("gm_lu_solve", self.n, _lib.ptr(self.lu), _lib.ptr(self.piv), nrhs, _lib.ptr(x),
                  _lib.stream_handle(b.device))
        return x


class NmtWorkspace:
    """Curved-sky MASTER workspace (gmaster/workspaces.py:1593-2255)."""

    def __init__(self, fl1=None, fl2=None, bins=None, is_teb=False, l_toeplitz=-1, l_exact=-1,
                 dl_band=-1, fname=None, normalization="MASTER"):
        self.mcm_blocks = self.mcm_binned = self._lu = None
        self._slot_blocks = self._dense = self._bpws = None
        self.pure_e1 = self.pure_b1 = self.pure_e2 = self.pure_b2 = False
        if fname is not None:
            self.read_from(fname)
            return
        if fl1 is not None or fl2 is not None or bins is not None:
            self.compute_coupling_matrix(fl1, fl2, bins, is_teb=is_teb, l_toeplitz=l_toeplitz,
                                         l_exact=l_exact, dl_band=dl_band,
                                         normalization=normalization)

    @classmethod
    def from_fields(cls, fl1, fl2, bins, **kwargs):
        return cls(fl1, fl2, bins, **kwargs)

    @classmethod
    def from_file(cls, fname):
        """Workspace read from a NaMaster-compatible FITS file (workspaces.py:1674-1676)."""
        return cls(fname=fname)

    def write_to(self, fname):
        """Write the workspace to a NaMaster-compatible FITS file (workspaces.py:2211-2255):
        the dense coupling matrix with the workspace keywords in the primary HDU, then the
        BEAMS, PCL_MASKS and BANDPOWERS tables.  An existing file is overwritten."""
        if self._lu is None:
            raise RuntimeError("the workspace holds no coupling matrix")
        header = {
            "LMAX": self.lmax, "LMAX_MASK": self.lmax_mask, "IS_TEB": bool(getattr(self, "is_teb", False)),
            "NCLS": self.ncls,
            "NORM_TYPE": 0 if self.normalization == "MASTER" else 1, "WAWB": float(self.wawb),
            "SPIN1": self.spin1, "SPIN2": self.spin2, "ANISO1": False, "ANISO2": False,
            "PURE_E1": bool(self.pure_e1), "PURE_B1": bool(self.pure_b1),
            "PURE_E2": bool(self.pure_e2), "PURE_B2": bool(self.pure_b2),
            "L_TOEPLITZ": self.l_toeplitz, "L_EXACT": self.l_exact, "DL_BAND": self.dl_band,
        }
        ell = np.arange(self.lmax + 1, dtype=np.int32)
        pcl = self.pcl_mask.cpu().numpy()
        fits.write(fname, [
            {"kind": "image", "name": "WSP_PRIMARY", "data": self.get_coupling_matrix().cpu().numpy(),
             "header": header},
            {"kind": "table", "name": "BEAMS",
             "columns": [("L", ell), ("BEAM1", self.beam1.cpu().numpy()),
                         ("BEAM2", self.beam2.cpu().numpy())]},
            {"kind": "table", "name": "PCL_MASKS",
             "columns": [("L", np.arange(len(pcl), dtype=np.int32)), ("PCL_MASKS", pcl)]},
            self.bins._fits_table("BANDPOWERS"),
        ])

    def read_from(self, fname, device=None):
        """Read a workspace from a NaMaster-compatible FITS file (workspaces.py:2162-2209)
        onto `device` (the current CUDA device by default), then bin and LU-factor it."""
        hdus = {h["name"]: h for h in fits.read(fname)}
        prim = hdus.get("WSP_PRIMARY") or fits.read(fname)[0]
        h = prim["header"]
        if any(bool(h.get(k, False)) for k in ("ANISO1", "ANISO2")):
            raise NotImplementedError("anisotropic workspaces are not part of this build")
        self.pure_e1, self.pure_b1 = bool(h.get("PURE_E1", False)), bool(h.get("PURE_B1", False))
        self.pure_e2, self.pure_b2 = bool(h.get("PURE_E2", False)), bool(h.get("PURE_B2", False))
        self._slot_blocks = None
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.lmax = int(h["LMAX"])
        self.lmax_mask = int(h["LMAX_MASK"])
        self.ncls = int(h["NCLS"])
        self.is_teb = bool(h.get("IS_TEB", False))
        self.normalization = "MASTER" if int(h.get("NORM_TYPE", 0)) == 0 else "FKP"
        self.wawb = float(h.get("WAWB", 0.0))
        self.spin1 = int(h.get("SPIN1", 0 if self.ncls == 1 else 2))
        self.spin2 = int(h.get("SPIN2", 0 if self.ncls == 1 else 2))
        self.nmaps1 = 1 if self.spin1 == 0 else 2
        self.nmaps2 = 1 if self.spin2 == 0 else 2
        self.l_toeplitz = int(h.get("L_TOEPLITZ", -1))
        self.l_exact = int(h.get("L_EXACT", -1))
        self.dl_band = int(h.get("DL_BAND", -1))
        self._dense = None
        try:
            if self.pure_e1 or self.pure_b1 or self.pure_e2 or self.pure_b2:
                # purified channels take different blocks per slot: keep each slot's block
                self.mcm_blocks = None
                self._slot_blocks = _slot_blocks_from_dense(prim["data"], self.lmax, self.ncls, dev)
            else:
                self.mcm_blocks = _blocks_from_dense(prim["data"], self.lmax, self.ncls, dev)
        except NotImplementedError:
            # a matrix without the slot structure (e.g. one set by update_coupling_matrix):
            # keep it dense
            self.mcm_blocks = self._slot_blocks = None
            self._dense = torch.from_numpy(np.ascontiguousarray(prim["data"], dtype=np.float64)).to(dev)
        beams = hdus["BEAMS"]["data"]
        if "BEAMS" in beams:
            b1 = b2 = np.sqrt(beams["BEAMS"].astype(np.float64))
        else:
            b1, b2 = beams["BEAM1"].astype(np.float64), beams["BEAM2"].astype(np.float64)
        self.beam1 = torch.from_numpy(np.ascontiguousarray(b1)).to(dev)
        self.beam2 = torch.from_numpy(np.ascontiguousarray(b2)).to(dev)
        self.pcl_mask = torch.from_numpy(
            np.ascontiguousarray(hdus["PCL_MASKS"]["data"]["PCL_MASKS"], dtype=np.float64)).to(dev)
        nw = min(self.pcl_mask.shape[0], 2 * self.lmax + 1)
        self.window = self.pcl_mask[:nw].contiguous()
        self.bins = NmtBin._from_fits_table(hdus["BINS"] if "BINS" in hdus else hdus["BANDPOWERS"])
        self.nbands = self.bins.get_n_bands()
        self._postprocess()

    def compute_coupling_matrix(self, fl1, fl2, bins, is_teb=False, l_toeplitz=-1, l_exact=-1,
                                dl_band=-1, normalization="MASTER"):
        self._prepare(fl1, fl2, bins, is_teb, l_toeplitz, l_exact, dl_band, normalization)
        self._compute_blocks()
        self._postprocess()

    def _prepare(self, fl1, fl2, bins, is_teb=False, l_toeplitz=-1, l_exact=-1, dl_band=-1,
                 normalization="MASTER"):
        """Checks, mask pseudo-spectrum and normalisation: everything but the blocks."""
        if not fl1.is_compatible(fl2, strict=False):
            raise ValueError("Fields have incompatible pixelizations")
        if fl1.ainfo.lmax != bins.lmax:
            raise ValueError(f"Maximum multipoles in bins ({bins.lmax}) and fields "
                             f"({fl1.ainfo.lmax}) are not the same")
        if is_teb and (fl1.spin != 0 or fl2.spin == 0):
            raise ValueError("If is_teb=True, fl1 must be spin-0 and fl2 non-zero spin")
        self.pure_e1, self.pure_b1 = bool(fl1.pure_e), bool(fl1.pure_b)
        self.pure_e2, self.pure_b2 = bool(fl2.pure_e), bool(fl2.pure_b)
        self._pure_any = self.pure_e1 or self.pure_b1 or self.pure_e2 or self.pure_b2
        if self._pure_any and l_toeplitz > 0:
            raise ValueError("Can't use Toeplitz approximation with purification.")
        toeplitz_sanity(l_toeplitz, l_exact, dl_band, fl1.ainfo.lmax)
        if normalization not in ("MASTER", "FKP"):
            raise ValueError(f"Unknown normalization type {normalization}. "
                             "Allowed options are 'MASTER' and 'FKP'")
        self.spin1, self.spin2 = fl1.spin, fl2.spin
        self.nmaps1 = 1 if self.spin1 == 0 else 2
        self.nmaps2 = 1 if self.spin2 == 0 else 2
        self.ncls = 7 if is_teb else self.nmaps1 * self.nmaps2
        self.is_teb = bool(is_teb)
        self.lmax = fl1.ainfo.lmax
        self.lmax_mask = fl1.ainfo_mask.lmax
        self.bins = bins
        self.nbands = bins.get_n_bands()
        self.normalization = normalization
        self.beam1 = fl1.beam
        self.beam2 = fl2.beam
        alm1 = fl1.get_mask_alms()
        alm2 = alm1 if fl2 is fl1 else fl2.get_mask_alms()
        self.pcl_mask = pseudo_cl(alm1[None], alm2[None], self.lmax_mask)[0]
        if fl2 is fl1:
            self.pcl_mask = self.pcl_mask - fl1.Nw
        nw = min(self.pcl_mask.shape[0], 2 * self.lmax + 1)
        self.window = self.pcl_mask[:nw].contiguous()
        self.l_toeplitz, self.l_exact, self.dl_band = int(l_toeplitz), int(l_exact), int(dl_band)
        self.wawb = 0.0
        if normalization == "FKP":
            self.wawb = float((fl1.get_mask() * fl2.get_mask()).sum() * fl1.minfo.weight / (4 * np.pi))

    def _compute_blocks(self, blocks=None):
        """Coupling blocks, or the exact ``blocks`` given (from a multi-workspace launch),
        then the Toeplitz fill when it is enabled."""
        l_toeplitz, l_exact, dl_band = self.l_toeplitz, self.l_exact, self.dl_band
        self._slot_blocks = self._dense = None
        if getattr(self, "_pure_any", False):
            self._compute_pure_blocks()
            return
        if self.spin1 not in (0, 2) or self.spin2 not in (0, 2):
            self._compute_general_spin_blocks()
            return
        if blocks is not None:
            self.mcm_blocks = blocks
        elif l_toeplitz > 0 and self.ncls == 1:
            # only the entries the Toeplitz fill reads are computed exactly
            n = self.lmax + 1
            self.mcm_blocks = torch.zeros((4, n, n), dtype=torch.float64, device=self.window.device)
            self.mcm_blocks[_BLOCK_TT] = coupling_tt_toeplitz(self.window, self.lmax, l_toeplitz,
                                                              l_exact, dl_band)
            return
        else:
            self.mcm_blocks = coupling_blocks(self.window, self.lmax, _which(self.ncls))
        if l_toeplitz > 0:
            # exact blocks, then the Toeplitz fill (workspaces.py:1833-1844)
            col = (2.0 * torch.arange(self.lmax + 1, dtype=torch.float64,
                                      device=self.window.device) + 1.0)[None, :]
            slots = sorted({x for x, _, _, _ in _slots(self.ncls)})
            for x in slots:
                self.mcm_blocks[x] = toeplitz_fill((self.mcm_blocks[x] / col).contiguous(),
                                                   self.lmax, l_toeplitz, l_exact, dl_band)

    def _compute_general_spin_blocks(self):
        """Blocks of workspaces with fields of spins other than 0 and 2 (workspaces.py:
        1811-1831, 1856-1897): the spin-0 x spin-s block and the spin-s1 x spin-s2 M+ / M-
        from the Gauss-Legendre quadrature of the general coupling matrix, the scalar block
        of a TEB workspace from the 3j kernel; the slot signs depend on the spins."""
        s1, s2, L = self.spin1, self.spin2, self.lmax
        lm = self.lmax_mask
        te = even = odd = None
        if s1 == 0 or s2 == 0:
            te = general_coupling_matrix(self.pcl_mask, s1, s2, s1, s2, L, lm).sum(0)
        else:
            even, odd = general_coupling_matrix(self.pcl_mask, s1, s2, s1, s2, L, lm)
        if self.is_teb:
            even, odd = general_coupling_matrix(self.pcl_mask, s2, s2, s2, s2, L, lm)
        col = (2.0 * torch.arange(L + 1, dtype=torch.float64, device=self.window.device)
               + 1.0)[None, :]
        if self.l_toeplitz > 0:
            def approx(x):
                return None if x is None else toeplitz_fill((x / col).contiguous(), L,
                                                             self.l_toeplitz, self.l_exact,
                                                             self.dl_band)
            te, even, odd = approx(te), approx(even), approx(odd)
        slots = []
        if self.ncls == 2:
            sign = -1.0 if (s1 + s2) % 2 else 1.0
            slots += [(te, 0, 0, sign), (te, 1, 1, sign)]
        else:
            offset = 3 if self.ncls == 7 else 0
            if self.ncls == 7:
                if self.l_toeplitz > 0:
                    tt = coupling_tt_toeplitz(self.window, L, self.l_toeplitz, self.l_exact,
                                              self.dl_band)
                else:
                    tt = coupling_blocks(self.window, L, 1)[_BLOCK_TT]
                mixed = -1.0 if s2 % 2 else 1.0
                slots += [(tt, 0, 0, 1.0), (te, 1, 1, mixed), (te, 2, 2, mixed)]
                spin_sign = 1.0
            else:
                spin_sign = -1.0 if (s1 + s2) % 2 else 1.0
            for index in range(4):
                slots.append((even, offset + index, offset + index, spin_sign))
            for index in range(4):
                slots.append((odd, offset + index, offset + 3 - index,
                              -spin_sign if index in (1, 2) else spin_sign))
        self._slot_blocks = [(b.contiguous(), r, c, sg) for b, r, c, sg in slots]
        self.mcm_blocks = None

    def _compute_pure_blocks(self):
        """Blocks of a workspace with purified fields (workspaces.py:1782-1897): all spin-2
        blocks from the Gauss-Legendre quadrature, each slot taking the standard block or
        the one with one or two purified fields according to how many of its two channels
        are purified."""
        from .pure import coupling_blocks_pure

        std_te, std_e, std_o, pure_te, e1, o1, e2, o2 = coupling_blocks_pure(self.window, self.lmax)
        te_levels, even_levels, odd_levels = (std_te, pure_te), (std_e, e1, e2), (std_o, o1, o2)
        slots = []
        if self.ncls == 2:
            pe, pb = int(self.pure_e1) + int(self.pure_e2), int(self.pure_b1) + int(self.pure_b2)
            for index, level in enumerate((pe, pb)):
                slots.append((te_levels[level], index, index, 1.0))
        else:
            offset = 3 if self.ncls == 7 else 0
            if self.ncls == 7:
                tt = coupling_blocks(self.window, self.lmax, 1)[_BLOCK_TT]
                slots.append((tt, 0, 0, 1.0))
                for index, level in enumerate((int(self.pure_e2), int(self.pure_b2))):
                    slots.append((te_levels[level], 1 + index, 1 + index, 1.0))
                pe1 = pe2 = int(self.pure_e2)
                pb1 = pb2 = int(self.pure_b2)
            else:
                pe1, pb1 = int(self.pure_e1), int(self.pure_b1)
                pe2, pb2 = int(self.pure_e2), int(self.pure_b2)
            levels = (pe1 + pe2, pe1 + pb2, pb1 + pe2, pb1 + pb2)
            for index, level in enumerate(levels):
                slots.append((even_levels[level], offset + index, offset + index, 1.0))
            for index, level in enumerate(levels):
                slots.append((odd_levels[level], offset + index, offset + 3 - index,
                              _MM_SIGNS[index]))
        self._slot_blocks = [(b.contiguous(), r, c, sg) for b, r, c, sg in slots]
        self.mcm_blocks = None

    def _postprocess(self):
        self._bpws = None
        if self._dense is not None:
            dev = self._dense.device
        elif self.mcm_blocks is not None:
            dev = self.mcm_blocks.device
        else:
            dev = self._slot_blocks[0][0].device
        ops = self.bins.device_operators(dev)
        beam = (self.beam1 * self.beam2).contiguous()
        N = self.ncls * self.nbands
        if self.normalization == "FKP":
            self.mcm_binned = self.wawb * torch.eye(N, dtype=torch.float64, device=dev)
        elif self._dense is not None:
            # B M diag(beam) T with kron(., I_ncls) operators, as FP64 GEMMs
            B, T = self._dense_operators(dev)
            rep = beam.repeat_interleave(self.ncls)[None, :]
            self.mcm_binned = (B @ (self._dense * rep)) @ T
        elif self._slot_blocks is not None:
            # a block per slot: each distinct block binned once, then placed with its sign
            nb = self.nbands
            binned = {}
            full = torch.zeros((nb, self.ncls, nb, self.ncls), dtype=torch.float64, device=dev)
            for blk, r, c, sign in self._slot_blocks:
                key = id(blk)
                if key not in binned:
                    scratch = torch.empty(2 * nb * nb, dtype=torch.float64, device=dev)
                    out = torch.empty((nb, nb), dtype=torch.float64, device=dev)
                    _lib.call("gm_bin_coupling_csr", self.lmax, nb, 1, _lib.ptr(blk),
                              _lib.ptr(ops["ptr"]), _lib.ptr(ops["ells"]), _lib.ptr(ops["wfl"]),
                              _lib.ptr(ops["inv_fl"]), _lib.ptr(beam), _lib.ptr(scratch),
                              _lib.ptr(out), _lib.stream_handle(dev))
                    binned[key] = out
                full[:, r, :, c] += sign * binned[key]
            self.mcm_binned = full.reshape(N, N)
        elif self.ncls == 7:
            # joint TEB: each distinct block binned on its own, then placed with its sign
            nb = self.nbands
            binned = {}
            for x in sorted({x for x, _, _, _ in _slots(7)}):
                scratch = torch.empty(2 * nb * nb, dtype=torch.float64, device=dev)
                out = torch.empty((nb, nb), dtype=torch.float64, device=dev)
                blk = self.mcm_blocks[x].contiguous()
                _lib.call("gm_bin_coupling_csr", self.lmax, nb, 1, _lib.ptr(blk), _lib.ptr(ops["ptr"]),
                          _lib.ptr(ops["ells"]), _lib.ptr(ops["wfl"]), _lib.ptr(ops["inv_fl"]),
                          _lib.ptr(beam), _lib.ptr(scratch), _lib.ptr(out), _lib.stream_handle(dev))
                binned[x] = out
            full = torch.zeros((nb, 7, nb, 7), dtype=torch.float64, device=dev)
            for x, r, c, sign in _slots(7):
                full[:, r, :, c] += sign * binned[x]
            self.mcm_binned = full.reshape(N, N)
        else:
            scratch = torch.empty(2 * self.nbands * self.nbands, dtype=torch.float64, device=dev)
            self.mcm_binned = torch.empty((N, N), dtype=torch.float64, device=dev)
            _lib.call("gm_bin_coupling_csr", self.lmax, self.nbands, self.ncls,
                      _lib.ptr(self.mcm_blocks), _lib.ptr(ops["ptr"]), _lib.ptr(ops["ells"]),
                      _lib.ptr(ops["wfl"]), _lib.ptr(ops["inv_fl"]), _lib.ptr(beam),
                      _lib.ptr(scratch), _lib.ptr(self.mcm_binned), _lib.stream_handle(dev))
        self._lu = LUFactor(self.mcm_binned)

    def get_coupling_matrix(self):
        """Dense (ncls (lmax+1))^2 MCM in ``l * ncls + c`` order (workspaces.py:2005-2025)."""
        n = self.lmax + 1
        if self._dense is not None:
            return self._dense.clone()
        if self._slot_blocks is not None:
            dev = self._slot_blocks[0][0].device
            out = torch.zeros((n, self.ncls, n, self.ncls), dtype=torch.float64, device=dev)
            for blk, r, c, sign in self._slot_blocks:
                out[:, r, :, c] += sign * blk
            return out.reshape(self.ncls * n, self.ncls * n)
        b = self.mcm_blocks
        if self.ncls == 1:
            return b[_BLOCK_TT].clone()
        out = torch.zeros((n, self.ncls, n, self.ncls), dtype=torch.float64, device=b.device)
        for x, r, c, sign in _slots(self.ncls):
            out[:, r, :, c] += sign * b[x]
        return out.reshape(self.ncls * n, self.ncls * n)

    def update_beams(self, beam1, beam2):
        n = self.lmax + 1
        if np.shape(beam1) != (n,) or np.shape(beam2) != (n,):
            raise ValueError(f"The new beams must go up to ell = {self.lmax}")
        self.beam1 = as_device(beam1, torch.float64)
        self.beam2 = as_device(beam2, torch.float64)
        self._postprocess()

    def update_bins(self, bins):
        if bins.lmax != self.lmax:
            raise ValueError("The new binning scheme has a different maximum multipole")
        self.bins = bins
        self.nbands = bins.get_n_bands()
        self._postprocess()

    def couple_cell(self, cl_in):
        """Theory spectra (ncls, >= lmax+1) -> expected coupled spectra (workspaces.py:2060-2104)."""
        cl = as_device(cl_in, torch.float64)
        if cl.ndim != 2 or cl.shape[0] != self.ncls or cl.shape[1] < self.lmax + 1:
            raise ValueError(f"Input power spectrum has wrong shape. Expected "
                             f"({self.ncls}, {self.lmax + 1}), but got {tuple(cl.shape)}")
        theory = cl[:, : self.lmax + 1] * (self.beam1 * self.beam2)[None, :]
        flat = theory.T.reshape(-1)
        return (self.get_coupling_matrix() @ flat).reshape(self.lmax + 1, self.ncls).T

    def decouple_cell(self, cl_in, cl_bias=None, cl_noise=None):
        """Bin and decouple coupled spectra into bandpowers (workspaces.py:2106-2147)."""
        cl = as_device(cl_in, torch.float64)
        if cl.ndim != 2 or cl.shape[0] != self.ncls or cl.shape[1] < self.lmax + 1:
            raise ValueError(f"Input power spectrum has wrong shape. Expected "
                             f"({self.ncls}, {self.lmax + 1}), but got {tuple(cl.shape)}")
        total = cl[:, : self.lmax + 1]
        for name, bias in (("bias", cl_bias), ("noise", cl_noise)):
            if bias is not None:
                bias = as_device(bias, torch.float64)
                if bias.ndim != 2 or bias.shape[0] != self.ncls or bias.shape[1] < self.lmax + 1:
                    raise ValueError(f"Input {name} power spectrum has wrong shape")
                total = total - bias[:, : self.lmax + 1]
        binned = self.bins.bin_cell(total.contiguous())
        vec = binned.T.reshape(-1).contiguous()
        self._lu.check()
        sol = self._lu.solve(vec)
        return sol.reshape(self.nbands, self.ncls).T

    def _dense_operators(self, dev):
        """kron(B, I_ncls) (nbands ncls, L ncls) and kron(T, I_ncls) (L ncls, nbands ncls):
        B averages a spectrum into bands with weight x f_ell, T spreads a bandpower over its
        multipoles divided by f_ell (workspaces.py:1452-1470)."""
        n = self.lmax + 1
        ops = self.bins.device_operators(dev)
        ells = torch.from_numpy(self.bins._ells_np.astype(np.int64)).to(dev)
        bp = torch.from_numpy(self.bins._bpws_np.astype(np.int64)).to(dev)
        B = torch.zeros((self.nbands, n), dtype=torch.float64, device=dev)
        B[bp, ells] = ops["wfl"][ells]
        T = torch.zeros((n, self.nbands), dtype=torch.float64, device=dev)
        T[ells, bp] = ops["inv_fl"][ells]
        eye = torch.eye(self.ncls, dtype=torch.float64, device=dev)
        return torch.kron(B, eye), torch.kron(T, eye)

    @property
    def bpws(self):
        """Bandpower windows solve(mcm_binned, B M diag(beam)), (nbands ncls, (lmax+1) ncls),
        computed on first access (workspaces.py:1629-1638)."""
        if self._bpws is None and self._lu is not None:
            dev = self.mcm_binned.device
            M = self.get_coupling_matrix() * (self.beam1 * self.beam2).repeat_interleave(self.ncls)[None]
            B, _ = self._dense_operators(dev)
            self._lu.check()
            self._bpws = self._lu.solve((B @ M).contiguous())
        return self._bpws

    def get_bandpower_windows(self):
        """(ncls, nbands, ncls, lmax+1) windows W with <C_b> = sum W C_l (workspaces.py:2149-2160)."""
        n = self.lmax + 1
        return self.bpws.reshape(self.nbands, self.ncls, n, self.ncls).permute(1, 0, 3, 2)

    def update_coupling_matrix(self, new_matrix):
        """Replace the unbinned coupling matrix ((ncls (lmax+1))^2, the ordering of
        `get_coupling_matrix`) and recompute the binned matrix and its LU factors
        (workspaces.py:2023-2040).  The matrix is kept dense."""
        size = self.ncls * (self.lmax + 1)
        if tuple(np.shape(new_matrix)) != (size, size):
            raise ValueError(f"Input matrix has an inconsistent shape. Expected {(size, size)}, "
                             f"but got {tuple(np.shape(new_matrix))}")
        dev = self.mcm_binned.device if self.mcm_binned is not None else None
        self._dense = as_device(new_matrix, torch.float64, dev).clone()
        self.mcm_blocks = self._slot_blocks = None
        self._postprocess()


# ----------------------------------------------------------------------------- general couplings

# Coupling operands are FP64 in this build at every size; the reference's switch between
# FP32 and FP64 operands (workspaces.py:40-84) is kept as a recorded setting.
_COUPLING_PRECISION = {"name": "auto"}


def set_coupling_precision(name):
    """Record the coupling operand precision ("fp64", "fp32" or "auto";
    workspaces.py:56-78).  This build computes every coupling block in FP64 (the 3j
    recursion and the quadrature alike), which is at least as accurate as either choice."""
    if name not in ("fp64", "fp32", "auto"):
        raise KeyError("GMaster coupling precision must be 'fp64', 'fp32' or 'auto'")
    _COUPLING_PRECISION["name"] = name


def coupling_precision():
    """The recorded coupling-precision setting (workspaces.py:81-84)."""
    return _COUPLING_PRECISION["name"]


def general_coupling_matrix(mask_cl, s1, s2, n1, n2, lmax, lmax_mask, table_bytes=None):
    """Even and odd general coupling matrices ``(2, lmax+1, lmax+1)`` by Gauss-Legendre
    quadrature (workspaces.py:683-747, 878-905): with the mask correlation
    xi(x) = sum_L (2L+1)/(4 pi) C_L d^L_{s1-n1, s2-n2}(x) (and its (-1)^L-signed twin),
    M[l1, l2] = (2 l2 + 1)/2 sum_i w_i d^l1_{n1 n2}(x_i) xi(x_i) d^l2_{-s1,-s2}(x_i), split
    by the parity of l1 + l2 + L.  Nodes are processed in chunks whose rows fit
    `table_bytes` (4 GB by default)."""
    from .pure import PURE_TABLE_BYTES, gl_nodes, wigner_corr, wigner_table

    c = as_device(mask_cl, torch.float64)
    dev = c.device
    L, Lm = lmax + 1, lmax_mask + 1
    cm = torch.zeros(Lm, dtype=torch.float64, device=dev)
    k = min(c.shape[0], Lm)
    cm[:k] = c[:k]
    ell = torch.arange(Lm, dtype=torch.float64, device=dev)
    coef = (2 * ell + 1) * cm / (4 * np.pi)
    sign = 1.0 - 2.0 * (torch.arange(Lm, device=dev) % 2).to(torch.float64)
    order = (2 * lmax + lmax_mask) // 2 + 1
    x_all, w_all = gl_nodes(order, dev)
    budget = PURE_TABLE_BYTES if table_bytes is None else int(table_bytes)
    chunk = max(1, min(order, budget // (2 * 8 * L)))
    tot = torch.zeros((L, L), dtype=torch.float64, device=dev)
    sig = torch.zeros((L, L), dtype=torch.float64, device=dev)
    vecs = torch.stack([coef, coef * sign])
    for a in range(0, order, chunk):
        x, w = x_all[a:a + chunk].contiguous(), w_all[a:a + chunk]
        xi = wigner_corr(x, lmax_mask, s1 - n1, s2 - n2, vecs)
        first = wigner_table(x, lmax, n1, n2)
        second = wigner_table(x, lmax, -s1, -s2)
        tot += (first * (w * xi[0])[None, :]) @ second.T
        sig += (first * (w * xi[1])[None, :]) @ second.T
    row = torch.arange(L, dtype=torch.float64, device=dev)
    cols = ((2 * row + 1) / 2)[None, :]
    pair_sign = 1.0 - 2.0 * ((row[:, None] + row[None, :]) % 2)
    tot = tot * cols
    sig = sig * cols * pair_sign
    return torch.stack([(tot + sig) / 2, (tot - sig) / 2])


def get_general_coupling_matrix(pcl_mask, s1, s2, n1, n2, parity="all"):
    """General mode-coupling matrix as in pymaster (workspaces.py:1069-1122):
    M[l, l'] = sum_l'' (2l'+1)(2l''+1)/(4 pi) C_l'' P (l l' l''; n1 -s1 s1-n1)
    (l l' l''; n2 -s2 s2-n2) with P = 1 ("all"), the even or odd parity of l + l' + l''
    ("even" / "odd"), or both stacked ("both").  Rows and columns below
    max(s1, s2, n1, n2) are zero."""
    if parity not in ("all", "even", "odd", "both"):
        raise ValueError('`parity` must be "all", "even", "odd", or "both".')
    c = as_device(pcl_mask, torch.float64)
    if c.ndim != 1:
        raise ValueError("pcl_mask must be one-dimensional")
    lmax = c.shape[0] - 1
    mats = general_coupling_matrix(c, int(s1), int(s2), int(n1), int(n2), lmax, lmax)
    lstart = max(int(s1), int(s2), int(n1), int(n2))
    keep = torch.arange(lmax + 1, device=c.device) >= lstart
    mats = torch.where(keep[None, :, None] & keep[None, None, :], mats, torch.zeros_like(mats))
    if parity == "both":
        return mats
    if parity == "even":
        return mats[0]
    if parity == "odd":
        return mats[1]
    return mats.sum(dim=0)


def get_master_coefficients(pcl_mask, lmax, spin1, spin2, is_teb=False, pure_any=False,
                            l_toeplitz=-1, l_exact=-1, dl_band=-1):
    """The distinct MASTER coupling blocks of a spin pair, divided by 2 l' + 1
    (workspaces.py:1197-1352): "00", "0s", "pp", "mm" (None when not applicable); "0s",
    "pp", "mm" carry a leading purification-level axis (1 without purification, 2 or 3
    with it) and a mask axis before the last two when `pcl_mask` is 2-D.  Spin-0/2
    blocks come from the 3j recursion (the quadrature with purification), other spins
    from `general_coupling_matrix`."""
    from .pure import coupling_blocks_pure

    spin1, spin2, lmax = int(spin1), int(spin2), int(lmax)
    if is_teb and not (spin1 == 0 and spin2 != 0):
        raise ValueError("is_teb is only valid for spin1=0 and spin2!=0")
    if pure_any and spin1 != 2 and spin2 != 2:
        raise ValueError("pure_any is only valid for spin 2")
    if pure_any and (spin1 not in (0, 2) or spin2 not in (0, 2)):
        raise ValueError("Purification is only implemented for spin 2")
    toeplitz_sanity(l_toeplitz, l_exact, dl_band, lmax)
    masks = as_device(pcl_mask, torch.float64)
    one_d = masks.ndim == 1
    if one_d:
        masks = masks[None]
    if masks.ndim != 2:
        raise ValueError("pcl_mask must be one- or two-dimensional")
    lmax_mask = masks.shape[1] - 1
    dev = masks.device
    cols = (2 * torch.arange(lmax + 1, dtype=torch.float64, device=dev) + 1)[None, :]
    has_00 = (spin1 == spin2 == 0) or is_teb
    has_0s = ((spin1 != spin2) and (spin1 == 0 or spin2 == 0)) or is_teb
    has_ss = (spin1 != 0 and spin2 != 0) or is_teb

    def toeplitz(S):
        return toeplitz_fill(S.contiguous(), lmax, l_toeplitz, l_exact, dl_band) / cols

    def standard(mask):
        nw = min(mask.shape[0], 2 * lmax + 1)
        window = mask[:nw].contiguous()
        pure8 = coupling_blocks_pure(window, lmax) if pure_any else None
        res = {}
        if has_00:
            if l_toeplitz > 0:
                res["00"] = coupling_tt_toeplitz(window, lmax, l_toeplitz, l_exact, dl_band) / cols
            else:
                res["00"] = coupling_blocks(window, lmax, 1)[_BLOCK_TT] / cols
        if has_0s:
            if spin1 in (0, 2) and spin2 in (0, 2):
                te = pure8[0] if pure8 is not None else coupling_blocks(window, lmax, 2)[_BLOCK_TE]
                res["0s"] = te / cols
            else:
                p0, p1 = (0, spin2) if spin1 == 0 else (spin1, 0)
                res["0s"] = general_coupling_matrix(mask, p0, p1, p0, p1, lmax, lmax_mask).sum(0) / cols
        if has_ss:
            a, b = (spin2, spin2) if is_teb else (spin1, spin2)
            if a == b == 2:
                if pure8 is not None:
                    ev, od = pure8[1], pure8[2]
                else:
                    blk = coupling_blocks(window, lmax, 12)
                    ev, od = blk[_BLOCK_PP], blk[_BLOCK_MM]
                res["pp"], res["mm"] = ev / cols, od / cols
            else:
                mats = general_coupling_matrix(mask, a, b, a, b, lmax, lmax_mask) / cols
                res["pp"], res["mm"] = mats[0], mats[1]
        if l_toeplitz > 0:
            for name in ("0s", "pp", "mm"):
                if name in res:
                    res[name] = toeplitz(res[name])
        if pure_any:
            p = [mtx / cols for mtx in pure8[3:]]
            if has_0s:
                res["0s"] = torch.stack([res["0s"], p[0]])
            if has_ss:
                res["pp"] = torch.stack([res["pp"], p[1], p[3]])
                res["mm"] = torch.stack([res["mm"], p[2], p[4]])
        else:
            for name in ("0s", "pp", "mm"):
                if name in res:
                    res[name] = res[name][None]
        return res

    values = [standard(m) for m in masks]
    out = {}
    for name, present in (("00", has_00), ("0s", has_0s), ("pp", has_ss), ("mm", has_ss)):
        if not present:
            out[name] = None
            continue
        arrs = [v[name] for v in values]
        out[name] = arrs[0] if one_d else torch.stack(arrs, dim=-3)
    out.update(pure_any=bool(pure_any),
               toeplitz={"l_toeplitz": l_toeplitz, "l_exact": l_exact, "dl_band": dl_band},
               spins=(spin1, spin2), lmax=lmax, lmax_mask=lmax_mask)
    return out


def deprojection_bias(f1, f2, cl_guess, n_iter=None):
    """Coupled bias from contaminant-template deprojection (workspaces.py:2268-2386).  Fields
    of this build carry no templates (deprojection is outside it), so after the
    reference's checks the bias is zero."""
    if not f1.is_compatible(f2):
        raise ValueError("Fields have incompatible pixelizations")
    shape = (f1.nmaps * f2.nmaps, f1.ainfo.lmax + 1)
    guess = as_device(cl_guess, torch.float64)
    if tuple(guess.shape) != shape:
        raise ValueError(f"Guess Cl should have shape {shape}")
    if f1.lite or f2.lite:
        raise ValueError("Can't compute deprojection bias for lightweight fields")
    return torch.zeros(shape, dtype=torch.float64, device=guess.device)


def uncorr_noise_deprojection_bias(f1, map_var, n_iter=None):
    """Deprojection bias for uncorrelated noise (workspaces.py:2389-2454): zero for fields
    without templates, which are all the fields of this build."""
    if f1.lite:
        raise ValueError("Can't compute deprojection bias for lightweight fields")
    var = as_device(map_var, torch.float64).reshape(-1)
    if var.shape[0] != f1.minfo.npix:
        raise ValueError("Variance map doesn't match map resolution")
    return torch.zeros((f1.nmaps * f1.nmaps, f1.ainfo.lmax + 1), dtype=torch.float64,
                       device=var.device)


def compute_full_master(f1, f2, b=None, cl_noise=None, cl_guess=None, workspace=None,
                        l_toeplitz=-1, l_exact=-1, dl_band=-1, normalization="MASTER"):
    """The full MASTER estimator for two fields (workspaces.py:2457-2517): coupled
    pseudo-C_ell minus the deprojection and noise biases, decoupled into bandpowers with
    `workspace` (built from `b` if not given)."""
    if b is None and workspace is None:
        raise SyntaxError("Must supply either workspace or bins")
    if not f1.is_compatible(f2, strict=False):
        raise ValueError("Fields have incompatible pixelizations")
    coupled = compute_coupled_cell(f1, f2)
    shape = (f1.nmaps * f2.nmaps, f1.ainfo.lmax + 1)
    dev = coupled.device
    noise = (torch.zeros(shape, dtype=torch.float64, device=dev) if cl_noise is None
             else as_device(cl_noise, torch.float64, dev))
    guess = (torch.zeros(shape, dtype=torch.float64, device=dev) if cl_guess is None
             else as_device(cl_guess, torch.float64, dev))
    if tuple(noise.shape) != shape:
        raise ValueError(f"Noise Cl should have shape {shape}")
    if tuple(guess.shape) != shape:
        raise ValueError(f"Guess Cl should have shape {shape}")
    bias = deprojection_bias(f1, f2, guess)
    if workspace is None:
        workspace = NmtWorkspace.from_fields(f1, f2, b, l_toeplitz=l_toeplitz, l_exact=l_exact,
                                             dl_band=dl_band, normalization=normalization)
    return workspace.decouple_cell(coupled - bias - noise)
