"""Monte-Carlo batches: many simulations that share one mask and one workspace.

A NaMaster-style Monte-Carlo loop builds one ``NmtField`` per simulated map and decouples
each spectrum with the same workspace (the reference does exactly this, one field at a
time: gmaster/field.py:78-98, gmaster/workspaces.py:2106-2147).  The helpers here run
that loop for a whole batch at once:

* ``fields_from_maps`` builds the (lite) fields of a batch.  In mixed precision the
  spherical-harmonic analyses, ``n_iter`` Jacobi iterations included, run as batched
  tensor-core transforms: up to 32 spin-0 maps or 32 spin-2 (Q, U) pairs share every
  generated Legendre row.  In FP64 each field goes through the FP64 transform.
* ``compute_coupled_cells`` returns the coupled spectra of field pairs.
* ``decouple_cells`` bins and decouples many spectra at once (one FP64 product with the
  LU factors of the binned coupling matrix, one right-hand side per simulation).
* ``workspaces_from_fields`` builds many workspaces -- of uneven lmax too -- whose
  coupling blocks come from one persistent FP64 Wigner-3j launch sharing a device work
  queue, instead of one launch per workspace.
* ``SimulationGraph`` captures the whole per-simulation estimator (masking, the two
  field transforms with their Jacobi iterations, three pseudo-spectra, binning and the
  three LU solves) as one CUDA graph and replays it for each simulation, so a loop over
  simulations issues one graph launch instead of some hundred kernel launches.
* ``mc_bandpowers`` runs the whole estimator for a batch of TQU simulations; maps given
  in (pinned) host memory are copied on a side stream, so that the copy of the (Q, U)
  maps overlaps the T transforms.
"""

import numpy as np
import torch

from . import _lib, sht, sht_tc
from ._config import get_precision, nmt_params
from .field import NmtField
from .utils import as_device
from .workspaces import (NmtWorkspace, _which, compute_coupled_cell, coupling_blocks_multi,
                         pseudo_cl)


def fields_from_maps(mask, maps, *, spin=None, n_iter=None, beam=None, lmax=None,
                     masked_on_input=False, precision=None, ring_spectra=None):
    """Lite fields of a batch of simulations sharing one mask.

    ``maps`` is (nsims, npix) or (nsims, 1, npix) for spin 0 and (nsims, 2, npix) for
    spin 2 (Q, U), float64 on the host or the device.  Returns a list of ``nsims``
    ``NmtField`` objects whose alms equal those of ``NmtField(mask, maps[i], ...)``
    up to the precision of the chosen transform.  ``ring_spectra`` (mixed precision, one
    tensor-core launch) may hand over the ring spectra of the masked maps already
    computed, in a one-element list that is emptied so the spectra can be released early.
    """
    precision = precision or get_precision()
    n_iter = nmt_params.n_iter_default if n_iter is None else int(n_iter)
    mask_t = as_device(mask, torch.float64)
    maps_t = as_device(maps, torch.float64)
    if maps_t.ndim == 2:
        maps_t = maps_t[:, None, :]
    if maps_t.ndim != 3 or maps_t.shape[1] not in (1, 2):
        raise ValueError("maps must be (nsims, npix), (nsims, 1, npix) or (nsims, 2, npix)")
    if maps_t.shape[2] != mask_t.shape[0]:
        raise ValueError("Maps and mask have different sizes")
    nmaps = maps_t.shape[1]
    if spin is None:
        spin = 0 if nmaps == 1 else 2
    if (spin == 0) != (nmaps == 1):
        raise ValueError("Spin-zero fields are associated with a single map")
    if spin not in (0, 2):
        raise NotImplementedError("only spin-0 and spin-2 fields are implemented")

    # one template field carries the geometry, lmax and beam checks of NmtField
    proto = NmtField(mask_t, None, spin=spin, n_iter=n_iter, beam=beam, lmax=lmax, lite=True,
                     precision=precision)
    nside, lm = proto.minfo.nside, proto.ainfo.lmax
    nsims = maps_t.shape[0]
    per_launch = sht_tc.MAX_MAPS_SPIN0 if spin == 0 else sht_tc.MAX_FIELDS_SPIN2
    alms = []
    for s0 in range(0, nsims, per_launch):
        chunk = maps_t[s0:s0 + per_launch]
        flat = chunk.reshape(-1, chunk.shape[2]).contiguous()
        if precision == "fp64":
            if not masked_on_input:
                flat = flat * mask_t[None, :]
            a = torch.cat([sht.map2alm_device(flat[i * nmaps:(i + 1) * nmaps], spin, nside, lm,
                                              n_iter, "fp64") for i in range(chunk.shape[0])])
        else:
            # the ring stage multiplies by the mask as it reads the maps: no masked copy
            spec = None
            if ring_spectra and s0 == 0 and nsims <= per_launch:
                spec = ring_spectra.pop()
            a = sht_tc.map2alm_tc(flat, spin, nside, lm, n_iter,
                                  mask=None if masked_on_input else mask_t, ring_spectra=spec)
            del spec
        del flat, chunk
        alms.append(a.reshape(-1, nmaps, a.shape[1]))
    # one launch's alms are used as they are (a concatenation would hold a second copy)
    alms = alms[0] if len(alms) == 1 else torch.cat(alms)
    fields = []
    for i in range(nsims):
        f = NmtField(mask_t, None, spin=spin, n_iter=n_iter, beam=beam, lmax=lmax, lite=True,
                     precision=precision)
        f.alm = alms[i]
        fields.append(f)
    return fields


def compute_coupled_cells(fields1, fields2):
    """Coupled pseudo-C_ell of each pair (fields1[i], fields2[i])."""
    if len(fields1) != len(fields2):
        raise ValueError("the two field lists must have the same length")
    return [compute_coupled_cell(a, b) for a, b in zip(fields1, fields2)]


def decouple_cells(workspace, cls, cl_bias=None, cl_noise=None):
    """Bandpowers of many coupled spectra (each (ncls, lmax+1)) with one LU solve of the
    binned coupling matrix for all of them (one right-hand side per spectrum).

    Equivalent to ``[workspace.decouple_cell(c, cl_bias, cl_noise) for c in cls]``.
    """
    w = workspace
    if len(cls) == 0:
        return []
    stack = []
    for c in cls:
        c = as_device(c, torch.float64)
        if c.ndim != 2 or c.shape[0] != w.ncls or c.shape[1] < w.lmax + 1:
            raise ValueError(f"Input power spectrum has wrong shape. Expected "
                             f"({w.ncls}, {w.lmax + 1}), but got {tuple(c.shape)}")
        c = c[:, : w.lmax + 1]
        for name, bias in (("bias", cl_bias), ("noise", cl_noise)):
            if bias is not None:
                bias = as_device(bias, torch.float64)
                if bias.ndim != 2 or bias.shape[0] != w.ncls or bias.shape[1] < w.lmax + 1:
                    raise ValueError(f"Input {name} power spectrum has wrong shape")
                c = c - bias[:, : w.lmax + 1]
        stack.append(c)
    allcl = torch.cat(stack).contiguous()                      # (nsims ncls, L)
    binned = w.bins.bin_cell(allcl)                            # (nsims ncls, nb)
    nb = binned.shape[1]
    rhs = binned.reshape(len(cls), w.ncls, nb).permute(2, 1, 0).reshape(nb * w.ncls, len(cls))
    w._lu.check()
    # every simulation is one right-hand side of the LU solve (the factors of the binned
    # coupling matrix, as decouple_cell uses them), all in one launch
    sol = w._lu.solve(rhs)                                     # (nb ncls, nsims)
    out = sol.reshape(nb, w.ncls, len(cls)).permute(2, 1, 0)
    return [out[i] for i in range(len(cls))]


def workspaces_from_fields(field_pairs, bins, **kwargs):
    """``[NmtWorkspace.from_fields(f1, f2, b, **kwargs) for (f1, f2), b in ...]`` with all
    coupling blocks built in one launch.

    ``field_pairs`` is a list of (fl1, fl2); ``bins`` one NmtBin for every pair or a list
    of them.  The workspaces may differ in lmax and spins.  Scalar workspaces with the
    Toeplitz approximation keep their own launch (they compute only the entries the fill
    reads), workspaces of purified fields their quadrature; every other workspace takes its
    exact blocks from the shared launch.
    """
    pairs = list(field_pairs)
    if not isinstance(bins, (list, tuple)):
        bins = [bins] * len(pairs)
    if len(bins) != len(pairs):
        raise ValueError("one NmtBin per field pair is needed")
    wss = []
    for (f1, f2), b in zip(pairs, bins):
        w = NmtWorkspace()
        w._prepare(f1, f2, b, **kwargs)
        wss.append(w)
    # scalar Toeplitz workspaces compute only the entries their fill reads, and purified
    # ones take all their blocks from the quadrature: neither needs the shared launch
    shared = [w for w in wss if not (w.l_toeplitz > 0 and w.ncls == 1) and not w._pure_any
              and w.spin1 in (0, 2) and w.spin2 in (0, 2)]
    blocks = coupling_blocks_multi([w.window for w in shared], [w.lmax for w in shared],
                                   [_which(w.ncls) for w in shared])
    given = {id(w): bl for w, bl in zip(shared, blocks)}
    for w in wss:
        w._compute_blocks(given.get(id(w)))
        w._postprocess()
    return wss


class SimulationGraph:
    """The estimator of one TQU simulation, captured once as a CUDA graph.

    ``SimulationGraph(mask, w00, w02, w22)(t, qu)`` returns the bandpowers TT (1, nb),
    TE/TB (2, nb) and EE/EB/BE/BB (4, nb) of ``w.decouple_cell(compute_coupled_cell(...))``
    for fields ``NmtField(mask, t)`` and ``NmtField(mask, qu)``, using the one-field
    transforms of ``precision`` (the SIMT kernels).  The first call runs the pipeline twice
    on a side stream (plans, tables and workspace operators are built there) and then
    captures it; every call copies the maps into the graph's static input buffers and
    replays the graph on the current stream.  The graph keeps its own memory pool; the
    returned tensors are copies.  The workspaces' LU factors are checked once, before the
    capture (a singular binned matrix raises there).
    """

    def __init__(self, mask, w00, w02, w22, *, n_iter=None, precision=None):
        self.precision = precision or get_precision()
        self.n_iter = nmt_params.n_iter_default if n_iter is None else int(n_iter)
        self.mask = as_device(mask, torch.float64).contiguous()
        npix = self.mask.shape[0]
        self.nside = int(round(np.sqrt(npix / 12)))
        if 12 * self.nside ** 2 != npix:
            raise ValueError("mask is not a HEALPix map")
        self.ws = (w00, w02, w22)
        if (w00.ncls, w02.ncls, w22.ncls) != (1, 2, 4):
            raise ValueError("workspaces must be spin 0x0, 0x2 and 2x2")
        self.lmax = w00.lmax
        for w in self.ws:
            w._lu.check()
        dev = self.mask.device
        self.t = torch.zeros((1, npix), dtype=torch.float64, device=dev)
        self.qu = torch.zeros((2, npix), dtype=torch.float64, device=dev)
        self.graph = None
        self.out = None

    def _step(self):
        at = sht.map2alm_device(self.t * self.mask[None, :], 0, self.nside, self.lmax, self.n_iter,
                                self.precision)
        aq = sht.map2alm_device(self.qu * self.mask[None, :], 2, self.nside, self.lmax, self.n_iter,
                                self.precision)
        out = []
        for w, (a, b) in zip(self.ws, ((at, at), (at, aq), (aq, aq))):
            binned = w.bins.bin_cell(pseudo_cl(a, b, self.lmax))
            sol = w._lu.solve(binned.T.reshape(-1).contiguous())
            out.append(sol.reshape(w.nbands, w.ncls).T)
        return out

    def capture(self):
        dev = self.mask.device
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            for _ in range(2):
                self._step()
        torch.cuda.current_stream(dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, capture_error_mode="relaxed"):
            self.out = self._step()

    def __call__(self, t, qu):
        t = as_device(t, torch.float64).reshape(1, -1)
        qu = as_device(qu, torch.float64).reshape(2, -1)
        if t.shape[1] != self.t.shape[1] or qu.shape[1] != self.qu.shape[1]:
            raise ValueError("Maps and mask have different sizes")
        if self.graph is None:
            self.capture()
        self.t.copy_(t)
        self.qu.copy_(qu)
        self.graph.replay()
        return [o.clone() for o in self.out]


_COPY_STREAMS = {}


def _copy_stream(dev):
    st = _COPY_STREAMS.get(dev.index)
    if st is None:
        st = torch.cuda.Stream(device=dev)
        _COPY_STREAMS[dev.index] = st
    return st


def _upload(x, dev):
    """Start the host-to-device copy of x on the side stream; returns (tensor, event)."""
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x, None
    h = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
    if h.dtype != torch.float64:
        h = h.to(torch.float64)
    side = _copy_stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        d = h.to(dev, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(side)
    d.record_stream(torch.cuda.current_stream(dev))
    return d, ev


def _stream_ring_spectra(t_maps, mask_t, dev, parts=4):
    """Copy host T maps (nsims, npix) to the device in `parts` pieces on the side stream and
    compute each piece's masked single-precision ring spectra on the current stream once
    it has arrived.  Returns (device maps, [spectra])."""
    h = t_maps if isinstance(t_maps, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(t_maps))
    if h.dtype != torch.float64:
        h = h.to(torch.float64)
    h = h.reshape(h.shape[0], -1)
    nsims, npix = h.shape
    nside = int(round(np.sqrt(npix / 12)))
    plan = sht.get_plan(nside, 3 * nside - 1, dev)
    d = torch.empty((nsims, npix), dtype=torch.float64, device=dev)
    spec = torch.empty((nsims, plan.nring, plan.L), dtype=torch.complex64, device=dev)
    main = torch.cuda.current_stream(dev)
    side = _copy_stream(dev)
    side.wait_stream(main)
    bounds = np.linspace(0, nsims, min(parts, nsims) + 1).astype(int)
    events = []
    with torch.cuda.stream(side):
        for a, b in zip(bounds[:-1], bounds[1:]):
            d[a:b].copy_(h[a:b], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(side)
            events.append(ev)
    for (a, b), ev in zip(zip(bounds[:-1], bounds[1:]), events):
        main.wait_event(ev)
        sht.ring_analysis(plan, d[a:b], _lib.MIXED, mask=mask_t, out=spec[a:b])
    return d, [spec]


def mc_bandpowers(mask, t_maps, qu_maps, w00, w02, w22, *, n_iter=None, precision=None):
    """Bandpowers of a batch of TQU simulations sharing one mask and three workspaces.

    ``t_maps`` (nsims, npix) and ``qu_maps`` (nsims, 2, npix), float64 on the device or in
    host memory (pinned host memory lets the copies run asynchronously: the (Q, U) maps
    are copied while the T fields are transformed).  Returns three lists over the
    simulations: TT (1, nb); TE, TB (2, nb); EE, EB, BE, BB (4, nb) -- the per-simulation
    result of ``w.decouple_cell(compute_coupled_cell(f1, f2))``.
    """
    dev = torch.device("cuda", torch.cuda.current_device())
    mask_t = as_device(mask, torch.float64)
    precision = precision or get_precision()
    main = torch.cuda.current_stream(dev)
    streamed = (precision != "fp64" and not (isinstance(t_maps, torch.Tensor) and t_maps.is_cuda)
                and 1 <= len(t_maps) <= sht_tc.MAX_MAPS_SPIN0)
    spec_box = None
    if streamed:
        # T maps in parts: the ring transform of each part runs as soon as it has arrived,
        # behind the copies of the next parts and of the (Q, U) maps
        t_dev, spec_box = _stream_ring_spectra(t_maps, mask_t, dev)
        qu_dev, ev_qu = _upload(qu_maps, dev)
    else:
        t_dev, ev_t = _upload(t_maps, dev)
        qu_dev, ev_qu = _upload(qu_maps, dev)
        if ev_t is not None:
            main.wait_event(ev_t)
    ft = fields_from_maps(mask_t, t_dev, spin=0, n_iter=n_iter, precision=precision,
                          ring_spectra=spec_box)
    del t_dev, spec_box
    if ev_qu is not None:
        main.wait_event(ev_qu)
    fp = fields_from_maps(mask_t, qu_dev, spin=2, n_iter=n_iter, precision=precision)
    del qu_dev
    return (decouple_cells(w00, compute_coupled_cells(ft, ft)),
            decouple_cells(w02, compute_coupled_cells(ft, fp)),
            decouple_cells(w22, compute_coupled_cells(fp, fp)))
