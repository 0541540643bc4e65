"""E/B purification: purified field alms and the coupling blocks of purified fields.

`purify_alms` adds to a spin-2 field's alms the counter-terms built from the spin-1 and
spin-2 derivatives of its mask (Smith 2006; gmaster/field.py:433-499), with this build's
spin-1, spin-2 and spin-0 transforms.  `coupling_blocks_pure` evaluates the eight spin-2
coupling blocks of gmaster/workspaces.py:927-1061 (standard TE, M+, M- and the purified TE,
M+/M- with one and with two purified fields) by Gauss-Legendre quadrature of products of
Wigner d-functions: the nodes, the d-function rows and the mask's correlation functions
come from the CUDA kernels of `wigner.cu`, the integrals are FP64 matrix products.
"""

import math

import numpy as np
import torch

from . import _lib, sht

__all__ = ["purify_alms", "coupling_blocks_pure", "gl_nodes", "wigner_table", "wigner_corr"]


def gl_nodes(n, device):
    """Ascending Gauss-Legendre nodes and weights of the n-point rule, the weights scaled to
    sum to 2 as the reference does (workspaces.py:593-605)."""
    x = torch.empty(n, dtype=torch.float64, device=device)
    w = torch.empty(n, dtype=torch.float64, device=device)
    _lib.call("gm_gl_nodes", n, _lib.ptr(x), _lib.ptr(w), _lib.stream_handle(device))
    return x, w * (2.0 / w.sum())


def _jacobi_norm(m, n, lmax, device):
    """sqrt(k! (k+mu+nu)! / ((k+mu)! (k+nu)!)) for k = 0 .. lmax - max(|m|, |n|)."""
    mu, nu = abs(m - n), abs(m + n)
    kmax = max(lmax - max(abs(m), abs(n)), 1)
    lg = [0.5 * (math.lgamma(k + 1) + math.lgamma(k + mu + nu + 1) - math.lgamma(k + mu + 1)
                 - math.lgamma(k + nu + 1)) for k in range(kmax + 1)]
    return torch.from_numpy(np.exp(np.asarray(lg))).to(device)


def wigner_table(x, lmax, m, n):
    """(lmax + 1, len(x)) rows d^l_mn(arccos x) (workspaces.py:608-679)."""
    out = torch.empty((lmax + 1, x.shape[0]), dtype=torch.float64, device=x.device)
    norm = _jacobi_norm(m, n, lmax, x.device)
    _lib.call("gm_wigner_table", x.shape[0], _lib.ptr(x), lmax, m, n, _lib.ptr(norm), _lib.ptr(out),
              _lib.stream_handle(x.device))
    return out


def wigner_corr(x, lmax, m, n, vecs):
    """(nvec, len(x)) sums sum_l d^l_mn(arccos x) vecs[v, l] for one or two vectors."""
    vecs = vecs.contiguous()
    out = torch.empty((vecs.shape[0], x.shape[0]), dtype=torch.float64, device=x.device)
    norm = _jacobi_norm(m, n, lmax, x.device)
    _lib.call("gm_wigner_corr", x.shape[0], _lib.ptr(x), lmax, m, n, _lib.ptr(norm), vecs.shape[0],
              _lib.ptr(vecs), _lib.ptr(out), _lib.stream_handle(x.device))
    return out


# Wigner rows of one chunk of quadrature nodes stay below this many bytes (nine row tables
# of (lmax + 1) x chunk doubles); the integrals accumulate over the chunks.
PURE_TABLE_BYTES = 4 << 30


def coupling_blocks_pure(window, lmax, table_bytes=None):
    """The eight (lmax+1)^2 spin-2 coupling blocks (standard TE, standard M+, standard M-,
    purified TE, M+ and M- with one purified field, M+ and M- with two) of a mask
    pseudo-spectrum `window` (zero-padded to 2 lmax + 1), following
    workspaces.py:927-1061 step by step.  The quadrature nodes are processed in chunks
    whose Wigner rows fit `table_bytes` (default `PURE_TABLE_BYTES`)."""
    dev = window.device
    L, L2 = lmax + 1, 2 * lmax + 1
    w2 = torch.zeros(L2, dtype=torch.float64, device=dev)
    nw = min(window.shape[0], L2)
    w2[:nw] = window[:nw]
    x_all, wt_all = gl_nodes(L2, dev)
    ell = torch.arange(L2, dtype=torch.float64, device=dev)
    first = torch.sqrt(ell * (ell + 1))
    second = torch.sqrt(torch.clamp((ell + 2) * (ell + 1) * ell * (ell - 1), min=0))
    row = torch.arange(L, dtype=torch.float64, device=dev)
    big = row > 1
    row_first = torch.where(big, 2 / torch.sqrt(torch.clamp((row + 2) * (row - 1), min=1)),
                            torch.zeros_like(row))
    row_second = torch.where(big, 1 / torch.sqrt(torch.clamp((row + 2) * (row + 1) * row * (row - 1),
                                                             min=1)), torch.zeros_like(row))
    coef = (2 * ell + 1) * w2 / (4 * np.pi)
    sign = 1.0 - 2.0 * (torch.arange(L2, device=dev) % 2).to(torch.float64)
    rf, rs = row_first[:, None], row_second[:, None]
    budget = PURE_TABLE_BYTES if table_bytes is None else int(table_bytes)
    chunk = max(1, min(L2, budget // (9 * 8 * L)))
    names = ("t", "std_t", "std", "std_s", "one", "one_s", "two", "two_s")
    acc = {k: torch.zeros((L, L), dtype=torch.float64, device=dev) for k in names}
    for a in range(0, L2, chunk):
        x, wt = x_all[a:a + chunk].contiguous(), wt_all[a:a + chunk]

        def corr(m, n, factor=None):
            c = coef if factor is None else coef * factor
            return wigner_corr(x, L2 - 1, m, n, torch.stack([c, c * sign]))

        c00, s00 = corr(0, 0)
        c10, s10 = corr(1, 0, first)
        c20, s20 = corr(2, 0, second)
        c11, s11 = corr(1, 1, first ** 2)
        c12, s12 = corr(1, 2, first * second)
        c22, s22 = corr(2, 2, second ** 2)
        c01 = corr(0, 1, first)[0]
        c02 = corr(0, 2, second)[0]
        d = {(m, n): wigner_table(x, lmax, m, n)
             for m, n in ((0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2), (2, 2))}
        right_t = wigner_table(x, lmax, 0, -2)
        right_s = wigner_table(x, lmax, -2, -2)

        def add(key, left_t, right):
            # sum over this chunk's nodes of left(x_i, l1) w_i right(x_i, l2)
            acc[key] += (left_t * wt[None, :]) @ right.T

        add("t", d[0, 2] * c00 + d[0, 1] * c01 * rf + d[0, 0] * c02 * rs, right_t)
        add("std_t", d[0, 2] * c00, right_t)
        add("std", d[2, 2] * c00, right_s)
        add("std_s", d[2, 2] * s00, right_s)
        add("one", d[2, 2] * c00 + d[1, 2] * c10 * rf + d[0, 2] * c20 * rs, right_s)
        add("one_s", d[2, 2] * s00 + d[1, 2] * s10 * rf + d[0, 2] * s20 * rs, right_s)
        add("two", d[2, 2] * c00 + 2 * d[1, 2] * c10 * rf + 2 * d[0, 2] * c20 * rs
            + d[1, 1] * c11 * rf ** 2 + 2 * d[1, 0] * c12 * rf * rs + d[0, 0] * c22 * rs ** 2, right_s)
        add("two_s", d[2, 2] * s00 + 2 * d[1, 2] * s10 * rf + 2 * d[0, 2] * s20 * rs
            + d[1, 1] * s11 * rf ** 2 + 2 * d[1, 0] * s12 * rf * rs + d[0, 0] * s22 * rs ** 2, right_s)
        del d, right_t, right_s
    cols = (2 * row + 1)[None, :] / 2
    pair_sign = 1.0 - 2.0 * ((row[:, None] + row[None, :]) % 2)

    def parity(total_key, signed_key):
        total = acc[total_key] * cols
        signed = acc[signed_key] * cols * pair_sign
        return (total + signed) / 2, (total - signed) / 2

    standard_e, standard_o = parity("std", "std_s")
    one_e, one_o = parity("one", "one_s")
    two_e, two_o = parity("two", "two_s")
    return (acc["std_t"] * cols, standard_e, standard_o, acc["t"] * cols, one_e, one_o, two_e, two_o)


def purify_alms(field, alm_mask, maps_unmasked, task, n_iter=None):
    """Pure E/B alms of a spin-2 field (gmaster/field.py:433-499): the masked alms plus, for
    the components selected by ``task = (purify_e, purify_b)``, the counter-terms of the
    spin-1 and spin-2 derivatives of the mask."""
    n_iter = field.n_iter if n_iter is None else int(n_iter)
    nside, prec = field.minfo.nside, field.precision
    lmax = field.ainfo.lmax
    dev = maps_unmasked.device
    ell_np, _ = field.ainfo.ell_m()
    ell = torch.from_numpy(ell_np.astype(np.float64)).to(dev)
    q, u = maps_unmasked[0], maps_unmasked[1]
    alms = sht.map2alm_device((maps_unmasked * field.mask[None, :]).contiguous(), 2, nside,
                              field.ainfo_mask.lmax, n_iter, prec)
    walm = torch.stack([alm_mask * (-torch.sqrt((ell + 1) * ell)), torch.zeros_like(alm_mask)])
    wmap = sht.alm2map_device(walm, 1, nside, field.ainfo_mask.lmax, prec)
    maps = torch.stack([wmap[0] * q + wmap[1] * u, wmap[0] * u - wmap[1] * q])
    palm = sht.map2alm_device(maps, 1, nside, lmax, n_iter, prec)
    big = ell >= 2
    f = torch.where(big, 2 / torch.sqrt(torch.clamp((ell + 2) * (ell - 1), min=1)), torch.zeros_like(ell))
    for ipol, on in enumerate(task):
        if on:
            alms[ipol] += palm[ipol] * f
    f = torch.where(big, -torch.sqrt(torch.clamp((ell + 2) * (ell - 1), min=0)), torch.zeros_like(ell))
    walm[0] = walm[0] * f
    wmap = sht.alm2map_device(walm, 2, nside, field.ainfo_mask.lmax, prec)
    maps = torch.stack([wmap[0] * q + wmap[1] * u, wmap[0] * u - wmap[1] * q])
    palm = sht.map2alm_device(maps, 0, nside, lmax, n_iter, prec)
    f = torch.where(big, 1 / torch.sqrt(torch.clamp((ell + 2) * (ell + 1) * ell * (ell - 1), min=1)),
                    torch.zeros_like(ell))
    for ipol, on in enumerate(task):
        if on:
            alms[ipol] += palm[ipol] * f
    return alms
