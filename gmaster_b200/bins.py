"""Bandpower binning (`NmtBin`), the counterpart of gmaster/bins.py:40-302."""

import numpy as np
import torch

from . import _lib


def _linear_bands(lmax, nlb):
    """Bands of `nlb` multipoles from l = 2; l < 2 and an incomplete last band get -1
    (gmaster/bins.py:30-37)."""
    ells = np.arange(lmax + 1, dtype=np.int32)
    bpws = ((ells - 2) // nlb).astype(np.int32)
    bpws[:2] = -1
    if np.sum(bpws == bpws[-1]) != nlb:
        bpws[bpws == bpws[-1]] = -1
    return ells, bpws


class NmtBin:
    """Bandpower definition (keyword-only arguments, as in the reference).

    ``C_b = sum_{l in b} w_l f_l C_l`` with the weights normalised to one per band.
    """

    def __init__(self, *, bpws, ells, lmax=None, weights=None, f_ell=None):
        # The definition: entries (l, b, w, f) with b >= 0 and l <= lmax take part; within a
        # band the weights are divided by their sum; f <= 0 means "no factor" (f = 1).
        table = self._entry_table(ells, bpws, weights, f_ell)
        if lmax is None:
            lmax = table["l"].max()
        self.lmax = self.ell_max = int(lmax)
        table = table[(table["b"] >= 0) & (table["l"] <= self.lmax)]
        self.n_bands = int(table["b"].max()) + 1 if len(table) else 1
        band_sum = np.zeros(self.n_bands)
        np.add.at(band_sum, table["b"], table["w"])
        empty = np.nonzero(~(band_sum > 0))[0]
        if len(empty):
            raise RuntimeError(f"Weights in band {int(empty[0])} are wrong")
        self._ells_np = np.ascontiguousarray(table["l"])
        self._bpws_np = np.ascontiguousarray(table["b"])
        self._weights_np = table["w"] / band_sum[table["b"]]
        self._f_ell_np = np.where(table["f"] > 0, table["f"], 1.0)
        self._dev = {}

    @staticmethod
    def _entry_table(ells, bpws, weights, f_ell):
        """The constructor's inputs as one structured array (l, b, w, f), checked for
        shape: ells and bpws non-empty 1-D of one length, weights and f_ell (default 1)
        of that length too."""
        l_arr = np.asarray(ells, dtype=np.int32)
        b_arr = np.asarray(bpws, dtype=np.int32)
        n = l_arr.shape[0] if l_arr.ndim == 1 else -1
        if n <= 0 or b_arr.shape != (n,):
            raise ValueError("ells and bpws must be non-empty 1-D arrays of equal size")
        cols = []
        for extra in (weights, f_ell):
            col = np.ones(n) if extra is None else np.asarray(extra)
            if col.shape != (n,):
                raise ValueError("weights and f_ell must have the same shape as ells")
            cols.append(col.astype(np.float64))
        table = np.empty(n, dtype=[("l", np.int32), ("b", np.int32), ("w", np.float64),
                                   ("f", np.float64)])
        table["l"], table["b"], table["w"], table["f"] = l_arr, b_arr, cols[0], cols[1]
        return table

    def _fits_table(self, extname="BANDPOWERS"):
        """The bandpower table of workspace files (gmaster/bins.py:288-302): one row per l
        with its band (-1 outside every band), weight and f_l."""
        bands = np.full(self.lmax + 1, -1, dtype=np.int32)
        weights = np.zeros(self.lmax + 1)
        f_ell = np.zeros(self.lmax + 1)
        bands[self._ells_np] = self._bpws_np
        weights[self._ells_np] = self._weights_np
        f_ell[self._ells_np] = self._f_ell_np
        return {"kind": "table", "name": extname,
                "columns": [("BAND", bands), ("ELLS", np.arange(self.lmax + 1, dtype=np.int32)),
                            ("WEIGHTS", weights), ("F_ELL", f_ell)],
                "header": {"ELL_MAX": self.lmax, "N_BANDS": self.n_bands}}

    @classmethod
    def _from_fits_table(cls, hdu):
        """Inverse of ``_fits_table`` (gmaster/bins.py:276-286)."""
        d = hdu["data"]
        return cls(lmax=int(hdu["header"]["ELL_MAX"]), bpws=d["BAND"], ells=d["ELLS"],
                   weights=d["WEIGHTS"].astype(np.float64), f_ell=d["F_ELL"].astype(np.float64))

    @classmethod
    def from_nside_linear(cls, nside, nlb, is_Dell=False, f_ell=None):
        return cls.from_lmax_linear(3 * nside - 1, nlb, is_Dell, f_ell)

    @classmethod
    def from_lmax_linear(cls, lmax, nlb, is_Dell=False, f_ell=None):
        ells, bpws = _linear_bands(lmax, nlb)
        if is_Dell and f_ell is None:
            f_ell = ells * (ells + 1) / (2 * np.pi)
        return cls(bpws=bpws, ells=ells, lmax=lmax, f_ell=f_ell)

    @classmethod
    def from_edges(cls, ell_ini, ell_end, is_Dell=False, f_ell=None):
        ells = np.concatenate([np.arange(a, b) for a, b in zip(ell_ini, ell_end)])
        bpws = np.concatenate([np.full(b - a, k) for k, (a, b) in enumerate(zip(ell_ini, ell_end))])
        weights = np.concatenate([np.full(b - a, 1 / (b - a)) for a, b in zip(ell_ini, ell_end)])
        if is_Dell and f_ell is None:
            f_ell = ells * (ells + 1) / (2 * np.pi)
        return cls(bpws=bpws, ells=ells, lmax=np.max(ells), weights=weights, f_ell=f_ell)

    def get_n_bands(self):
        return self.n_bands

    def get_nell_list(self):
        return np.bincount(self._bpws_np, minlength=self.n_bands)

    def get_ell_list(self, b):
        return self._ells_np[self._bpws_np == int(b)].copy()

    def get_ell_min(self, b):
        return self.get_ell_list(b)[0]

    def get_ell_max(self, b):
        return self.get_ell_list(b)[-1]

    def get_weight_list(self, b):
        return self._weights_np[self._bpws_np == int(b)].copy()

    def get_fell_list(self, b):
        return self._f_ell_np[self._bpws_np == int(b)].copy()

    def get_effective_ells(self):
        return np.bincount(self._bpws_np, weights=self._ells_np * self._weights_np,
                           minlength=self.n_bands)

    # ------------------------------------------------------------- device operators

    def device_operators(self, device):
        """CSR band lists and per-l factors on the device, for the binning kernels."""
        dev = torch.device(device)
        key = (dev.type, dev.index)
        ops = self._dev.get(key)
        if ops is None:
            order = np.lexsort((self._ells_np, self._bpws_np))
            ells = self._ells_np[order].astype(np.int32)
            counts = np.bincount(self._bpws_np, minlength=self.n_bands)
            ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
            wfl = np.zeros(self.lmax + 1)
            inv_fl = np.zeros(self.lmax + 1)
            wfl[self._ells_np] = self._weights_np * self._f_ell_np
            inv_fl[self._ells_np] = 1.0 / self._f_ell_np
            ops = {
                "ptr": torch.from_numpy(ptr).to(dev),
                "ells": torch.from_numpy(ells).to(dev),
                "wfl": torch.from_numpy(wfl).to(dev),
                "inv_fl": torch.from_numpy(inv_fl).to(dev),
            }
            self._dev[key] = ops
        return ops

    def bin_cell(self, cls_in):
        """Bin spectra (n_cls, lmax+1) -> (n_cls, n_bands) on the GPU (bins.py:228-250)."""
        from .utils import as_device

        cls = as_device(cls_in, torch.float64)
        oned = cls.ndim != 2
        if oned:
            cls = cls[None]
        if cls.ndim > 2 or cls.shape[1] != self.lmax + 1:
            raise ValueError("Input Cl has wrong size")
        cls = cls.contiguous()
        ops = self.device_operators(cls.device)
        out = torch.empty((cls.shape[0], self.n_bands), dtype=torch.float64, device=cls.device)
        _lib.call("gm_bin_cells_csr", self.lmax, self.n_bands, cls.shape[0], _lib.ptr(cls),
                  _lib.ptr(ops["ptr"]), _lib.ptr(ops["ells"]), _lib.ptr(ops["wfl"]), _lib.ptr(out),
                  _lib.stream_handle(cls.device))
        return out[0] if oned else out

    def unbin_cell(self, cls_in):
        """Bandpowers -> piecewise-constant spectra divided by f_ell (bins.py:252-275)."""
        from .utils import as_device

        cls = as_device(cls_in, torch.float64)
        oned = cls.ndim != 2
        if oned:
            cls = cls[None]
        if cls.ndim > 2 or cls.shape[1] != self.n_bands:
            raise ValueError("Input Cl has wrong size")
        out = torch.zeros((cls.shape[0], self.lmax + 1), dtype=torch.float64, device=cls.device)
        ells = torch.from_numpy(self._ells_np.astype(np.int64)).to(cls.device)
        bp = torch.from_numpy(self._bpws_np.astype(np.int64)).to(cls.device)
        fl = torch.from_numpy(self._f_ell_np).to(cls.device)
        out[:, ells] = cls[:, bp] / fl
        return out[0] if oned else out
