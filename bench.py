#!/usr/bin/env python
"""Throughput of the pseudo-C_ell MASTER estimator on B200 GPUs.

Workload (the Nside 2048 configuration): T, Q, U maps at Nside 2048 (lmax 6143) drawn
from C_TT = 1e3/(l+10)^2, C_EE = 0.05 C_TT, C_BB = 0.005 C_TT, C_TE = 0.3 sqrt(C_TT C_EE);
binary mask |b| > 20 deg about a pole tilted to (theta, phi) = (30, 45) deg with 2000
point-source holes of 5 arcmin (seeded), C1-apodised at 1 deg; n_iter = 3; bands of 16.

One step = one batch of Monte-Carlo simulations (32 by default) through the estimator
with shared, precomputed workspaces: fields_from_maps for T and for (Q, U) (map2alm with
3 Jacobi iterations, batched on the tensor cores), compute_coupled_cells for TT, TE/TB
and EE/EB/BE/BB, and decouple_cells with the three binned coupling matrices.  `value` is
sims/s with the maps resident on the device; `e2e` is the same through the public API
from pinned host maps (host->device copy of the maps and device->host copy of the
bandpowers inside the timed region).  Inputs (400 MB per map) are larger than the
126 MB L2, so no explicit flush is needed.  The plain FP64 GPU path (one simulation at
a time) is timed beside it, and the mixed/FP64 bandpowers of the same simulation are
compared.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--batch S] [--impl reference]
Under torchrun each rank runs independent simulations (replicas, no collective on the
data path); value is the total over ranks divided by the max-over-ranks device time.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MASTER sims/s, Nside 2048 TQU (shared workspace, n_iter=3), mixed precision"
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")


# Kernel behind each timed Legendre pass (the checkpointed kernels of legendre_ck.cu when
# the geometry's checkpoint tables are in use, else the carried-state ones of
# legendre_tc.cu).
KERNEL_OF = {"tc_analysis_s2": "k_ana_ck<2>", "tc_analysis_s0": "k_ana_ck<0>",
             "tc_synthesis_s2": "k_syn_ck<2>", "tc_synthesis_s0": "k_syn_ck<0>"}
KERNEL_OF_CARRIED = {"tc_analysis_s2": "k_ana_tc<2>", "tc_analysis_s0": "k_ana_tc<0>",
                     "tc_synthesis_s2": "k_syn_tc<2>", "tc_synthesis_s0": "k_syn_tc<0>"}

# DRAM traffic of one checkpointed analysis launch: ncu measured 1.545 GB (dram__bytes_read.sum
# + dram__bytes_write.sum) for the spin-2 launch of 8 fields at Nside 512, 1.029 x the byte
# model below (operand images read once, alm accumulator read and written once, checkpoint
# states read once); the launch at the benchmark size is given as that model x 1.029.
# DRAM bytes ncu measured for one k_ana_ck<2> launch (row variant s' = -2) at Nside 512 with
# 8 fields (1.061 GB read + 0.293 GB written), over the byte model below evaluated on the
# same launch's unit masks (1.3298 GB)
CK_TRAFFIC_RATIO = 1.354e9 / 1.3298e9


def ck_unit_activity(nside, lmax, spin=2, sp=-2):
    """(active 64-lane groups per analysis unit, unit offsets per order) of the row variant,
    from the zero-group masks the geometry's checkpoint tables were built with; None when
    the masks do not exist."""
    from gmaster_b200 import sht_tc
    tp = sht_tc.get_tc_plan(nside, lmax)
    mk = sht_tc.ck_masks(tp, spin, sp)
    if mk is None:
        return None
    um = mk[1].cpu().numpy().view(np.uint64)
    return um, tp.ck_uoff[spin].cpu().numpy()


def ck_analysis_bytes(nside, lmax, nrows, activity=None):
    """Byte model of one checkpointed analysis launch (one row variant).  Without masks: a 64 KB
    operand image per (order, 128-lane group), nrows FP64 alm rows read and written, 9 B
    checkpoint state per (128-row segment, lane).  With the unit masks (`ck_unit_activity`):
    32 KB per (order, 64-lane group) active in some unit of the order, the alm rows of the
    units with an active group, and the states of the active (unit, group) pairs."""
    L, nlanes = lmax + 1, 2 * nside
    groups = (nlanes + 127) // 128
    if activity is None:
        nelem = L * (L + 1) // 2
        segs = sum((L - max(m, 2) + 127) // 128 for m in range(L))
        return L * groups * 65536 + 2 * nelem * nrows * 8 + segs * nlanes * 9
    um, uoff = activity
    per_order = np.bitwise_or.reduceat(um, uoff[:-1].astype(np.int64))
    img = int(np.bitwise_count(per_order).sum()) * 32768
    first = np.maximum(np.arange(L), 2)
    rows = 0
    for m in range(L):
        n_m = int(uoff[m + 1] - uoff[m])
        live = um[uoff[m]:uoff[m + 1]] != 0
        full = np.minimum(256, L - first[m] - 256 * np.arange(n_m))
        rows += int(full[live].sum())
    states = int(np.bitwise_count(um).sum()) * 64 * 2 * 9
    return img + 2 * rows * nrows * 8 + states


def ck_issued_flops(activity, nrows_mma=128):
    """Tensor-pipe flops one k_ana_ck launch issues: three f16 products of M = 128, N = 256,
    K = 64 per active (unit, 64-lane group)."""
    um, _ = activity
    return 3 * 2 * nrows_mma * 256 * 64 * int(np.bitwise_count(um).sum())


def traffic_per_launch(kernel, nside, lmax, sims, activity=None):
    """(model bytes, DRAM bytes scaled by the measured ratio) of one launch, or (None, None)."""
    if kernel == "k_ana_ck<2>":
        model = ck_analysis_bytes(nside, lmax, 4 * sims, activity)
        return model, CK_TRAFFIC_RATIO * model
    return None, None


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nside", type=int, default=2048)
    p.add_argument("--nlb", type=int, default=16)
    p.add_argument("--batch", type=int, default=32)
    p.add_argument("--fp64-steps", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--workload", default="mc",
                   choices=["mc", "uneven_workspaces", "nside4096", "mc1024", "nside8192", "apodize",
                            "covariance", "purify"],
                   help="mc: the Monte-Carlo estimator (default); uneven_workspaces: TT "
                        "coupling matrices of 32 masks of mixed Nside in one launch; nside4096: "
                        "batched map2alm (n_iter=0) and alm2map at Nside 4096; mc1024: 512 TQU "
                        "simulations at Nside 1024, batched and per simulation as a CUDA graph; "
                        "nside8192: one spin-2 spectrum at Nside 8192 with the exact and the "
                        "Toeplitz coupling matrix; apodize: C1 apodisation of the binary "
                        "Nside 2048 and 8192 config masks on the GPU; covariance: Gaussian "
                        "(NKA) covariance workspaces and bandpower covariances at Nside 2048; "
                        "purify: a purified-B spin-2 field and its 2x2 workspace at Nside 2048")
    p.add_argument("--apo-nsides", default="2048,8192",
                   help="apodize workload: the Nside values to run (the first is the headline)")
    p.add_argument("--nmasks", type=int, default=32)
    return p.parse_args()


# ----------------------------------------------------------------------------- inputs

def config_spectra(lmax):
    ell = np.arange(lmax + 1, dtype=np.float64)
    tt = 1e3 / (ell + 10.0) ** 2
    tt[:2] = 0
    ee, bb = 0.05 * tt, 0.005 * tt
    te = 0.3 * np.sqrt(tt * ee)
    return tt, ee, bb, te


def make_mask(nside, device, seed=4, nholes=2000, hole_arcmin=5.0, cut_deg=20.0, apo_deg=1.0):
    """Analytic C1-apodised mask of the Nside 2048 recipe, built on the GPU.

    The angular distance of each observed pixel to the masked region is the smaller of
    (|b| - cut) and (distance to the nearest hole centre - hole radius); the C1 factor
    x - sin(2 pi x)/(2 pi), x = sqrt((1 - cos d)/(1 - cos apo)), is applied within apo.
    """
    import torch

    from gmaster_b200.utils import pix2vec_ring

    vec = torch.from_numpy(pix2vec_ring(nside)).to(device)
    th, ph = np.radians(30.0), np.radians(45.0)
    pole = torch.tensor([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)],
                        dtype=torch.float64, device=device)
    rng = np.random.default_rng(seed)
    centres = rng.normal(size=(nholes, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    cen = torch.from_numpy(centres).to(device)
    blat = torch.arcsin((vec @ pole).abs().clamp(max=1.0))
    d = blat - np.radians(cut_deg)
    r = np.radians(hole_arcmin / 60.0)
    chunk = 1 << 20
    for s in range(0, vec.shape[0], chunk):
        cosang = (vec[s:s + chunk] @ cen.T).max(dim=1).values.clamp(-1.0, 1.0)
        d[s:s + chunk] = torch.minimum(d[s:s + chunk], torch.arccos(cosang) - r)
    mask = (d > 0).to(torch.float64)
    apo = np.radians(apo_deg)
    x = torch.sqrt((1 - torch.cos(d.clamp(min=0))) / (1 - np.cos(apo)))
    c1 = x - torch.sin(2 * np.pi * x) / (2 * np.pi)
    mask = torch.where((d > 0) & (d < apo), c1, mask)
    return mask.contiguous()


def make_sims(nside, nsims, seed, device):
    """T maps (nsims, npix) and Q, U maps (nsims, 2, npix), float64 on the device, of
    `nsims` seeded Gaussian TQU simulations of the configuration spectra.  The alms are
    drawn on the GPU (unit complex normals, real at m = 0, mixed through the Cholesky
    factor of the (T, E, B) covariance at each l) and synthesised with the batched
    tensor-core alm2map."""
    import torch

    from gmaster_b200 import sht_tc
    from gmaster_b200.utils import NmtAlmInfo

    lmax = 3 * nside - 1
    tt, ee, bb, te = config_spectra(lmax)
    l00 = np.sqrt(tt)
    l10 = np.divide(te, l00, out=np.zeros_like(te), where=l00 > 0)
    l11 = np.sqrt(np.maximum(ee - l10 ** 2, 0.0))
    l22 = np.sqrt(bb)
    ell, order = NmtAlmInfo(lmax).ell_m()
    ell_t = torch.from_numpy(ell).to(device)
    m0 = torch.from_numpy(order == 0).to(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    dev_f = lambda a: torch.from_numpy(a).to(device)[ell_t]

    def unit():
        re = torch.randn((nsims, ell.shape[0]), generator=gen, device=device, dtype=torch.float64)
        im = torch.randn((nsims, ell.shape[0]), generator=gen, device=device, dtype=torch.float64)
        re[:, m0] *= np.sqrt(2.0)
        im[:, m0] = 0.0
        return torch.complex(re, im) / np.sqrt(2.0)

    step0, step2 = sht_tc.MAX_MAPS_SPIN0, sht_tc.MAX_FIELDS_SPIN2
    z0 = unit()
    a_t = z0 * dev_f(l00)
    t = torch.cat([sht_tc.alm2map_tc(a_t[i:i + step0], 0, nside, lmax) for i in range(0, nsims, step0)])
    del a_t
    a_e = z0 * dev_f(l10)
    del z0
    a_e += unit() * dev_f(l11)
    a_b = unit() * dev_f(l22)
    eb = torch.stack([a_e, a_b], dim=1)                       # (nsims, 2, nelem)
    del a_e, a_b
    qu = torch.cat([sht_tc.alm2map_tc(eb[i:i + step2].reshape(-1, eb.shape[2]), 2, nside, lmax)
                    for i in range(0, nsims, step2)])
    del eb
    return t.contiguous(), qu.reshape(nsims, 2, -1).contiguous()


# ----------------------------------------------------------------------------- ranks

def max_over_ranks(value, device):
    """Maximum of a per-rank float over all ranks of the process group (the value itself
    when there is no group or one rank)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(world, steps, per_step, ms):
    """Whole-job units per second: every rank processes steps x per_step units, the job
    lasts the slowest rank's ms."""
    return world * steps * per_step / (ms / 1e3)


# ----------------------------------------------------------------------------- estimator

def build_workspaces(mask, nside, nlb, precision):
    import gmaster_b200 as nmt

    f0 = nmt.NmtField(mask, None, spin=0, precision=precision)
    f2 = nmt.NmtField(mask, None, spin=2, precision=precision)
    f2.alm_mask = f0.get_mask_alms()
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    return b, {
        "00": nmt.NmtWorkspace.from_fields(f0, f0, b),
        "02": nmt.NmtWorkspace.from_fields(f0, f2, b),
        "22": nmt.NmtWorkspace.from_fields(f2, f2, b),
    }


def estimator_step(mask, t, qu, ws, precision):
    """One simulation through fields, coupled spectra and decoupling."""
    import gmaster_b200 as nmt

    ft = nmt.NmtField(mask, t, n_iter=3, lite=True, precision=precision)
    fp = nmt.NmtField(mask, qu, n_iter=3, lite=True, precision=precision)
    return (ws["00"].decouple_cell(nmt.compute_coupled_cell(ft, ft)),
            ws["02"].decouple_cell(nmt.compute_coupled_cell(ft, fp)),
            ws["22"].decouple_cell(nmt.compute_coupled_cell(fp, fp)))


def batch_step(mask, t, qu, ws, precision="mixed"):
    """A batch of simulations through the Monte-Carlo batch API (shared workspaces):
    fields_from_maps for T and (Q, U), compute_coupled_cells and decouple_cells, with the
    host-to-device copy of host maps overlapping the transforms."""
    import gmaster_b200 as nmt

    return nmt.mc_bandpowers(mask, t, qu, ws["00"], ws["02"], ws["22"], n_iter=3,
                             precision=precision)


def full_estimator(mask, t, qu, nside, nlb, precision, stages=None):
    """The whole estimator from the maps: fields with their mask transforms, three
    workspaces (pseudo-C_ell of the mask, 3j coupling, binning, LU), spectra.  With a dict
    `stages`, the device time of each stage (ms, CUDA events) is added to it."""
    import torch

    import gmaster_b200 as nmt

    marks = []

    def mark(name):
        if stages is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks.append((name, ev))

    # a fresh mask tensor: the mask alms are computed once per call (shared by the two
    # fields of the call), not served from an earlier call
    mask = mask.clone()
    mark("start")
    ft = nmt.NmtField(mask, t, n_iter=3, precision=precision)
    mark("T field (map and mask transforms)")
    fp = nmt.NmtField(mask, qu, n_iter=3, precision=precision)
    mark("QU field")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    pairs = ((ft, ft), (ft, fp), (fp, fp))
    # the three workspaces in one coupling launch (the fields share the mask, so one 3j
    # recursion per (l1, l2) serves the TT, TE and EE/BB blocks)
    wss = nmt.workspaces_from_fields(pairs, b)
    mark("workspaces 00, 02, 22")
    out = []
    for name, (f1, f2), w in zip(("00", "02", "22"), pairs, wss):
        out.append(w.decouple_cell(nmt.compute_coupled_cell(f1, f2)))
        mark(f"spectra {name}")
    if stages is not None:
        torch.cuda.synchronize()
        for (_, a), (name, b_) in zip(marks[:-1], marks[1:]):
            stages[name] = stages.get(name, 0.0) + a.elapsed_time(b_)
    return out


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(np.max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU legs

def cpu_oracle_sample(nside):
    """One bounded sample of the FP64 oracle's work for one simulation, timed, and the
    sims/s it implies.  The sample is a ring FFT of every ring plus the Legendre sums of
    a sample of orders, for spin 0 and spin 2; every part of it runs inside the timed
    region.  One simulation is 7 passes of each spin (4 analyses + 3 syntheses of map2alm
    with n_iter = 3; in the oracle a synthesis costs what an analysis costs), and a pass
    is the ring FFTs plus the Legendre sums of all orders, whose cost per order scales with
    (L - m): the full pass time is extrapolated as ring time + sampled Legendre time x
    sum_m (L - m) / sum_sample (L - m).  Returns the sample's wall time, the share of one
    simulation's modelled work it covered and the extrapolated sims/s (marked as such)."""
    import oracle

    oracle.build()
    lmax = 3 * nside - 1
    L = lmax + 1
    rng = np.random.default_rng(0)
    npix = 12 * nside ** 2
    m0 = rng.normal(size=npix)
    qu = rng.normal(size=(2, npix))
    orders = np.arange(0, L, max(1, L // 8))
    t0 = time.perf_counter()
    oracle.ring_analysis(nside, L, m0.astype(np.complex128))
    t_ring0 = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.ana0_orders(m0, nside, lmax, orders)
    t_a0 = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.ana2_orders(qu, nside, lmax, orders)
    t_a2 = time.perf_counter() - t0
    t_ring2 = 2 * t_ring0  # the spin-2 ring stage transforms Q + iU over m in (-L, L)
    w_all = L * (L + 1) / 2
    w_s = float(np.sum(L - orders))
    leg0 = max(t_a0 - t_ring0, 0.0) * w_all / w_s
    leg2 = max(t_a2 - t_ring2, 0.0) * w_all / w_s
    sim_seconds = 7 * (t_ring0 + leg0) + 7 * (t_ring2 + leg2)
    wall = t_ring0 + t_a0 + t_a2
    return {
        "value": 1.0 / sim_seconds,
        "unit": "sims/s",
        "cores": os.cpu_count(),
        "kind": "port",
        "extrapolated": True,
        "sample_fraction": wall / sim_seconds,
        "sample": (f"FP64 C oracle (OpenMP, {os.cpu_count()} threads): ring FFT of all "
                   f"{4 * nside - 1} rings + spin-0 and spin-2 Legendre sums for {len(orders)} of "
                   f"{L} orders at Nside {nside} ({wall:.1f} s, timed); sims/s extrapolated by "
                   f"sum(L-m) to the 7 spin-0 + 7 spin-2 passes of one simulation "
                   f"(the sample is {wall / sim_seconds:.2e} of one simulation's work)"),
        "sample_wall_s": wall,
        "seconds_per_sim": sim_seconds,
    }


def cpu_oracle_config1():
    """The FP64 oracle's complete scalar estimator at Nside 64 (lmax 191, the CPU-runnable
    configuration), timed as it runs, nothing extrapolated: field and mask transforms with
    n_iter = 3, the mask pseudo-spectrum, the exact coupling matrix, its binning (bands of
    16), the map's pseudo-spectrum and the decoupled bandpowers.  The mask (a 60 deg cap
    with 20 holes of 1 deg, C1-apodised at 2 deg) and the map are made outside the timing."""
    import oracle

    oracle.build()
    nside, nlb = 64, 16
    lmax = 3 * nside - 1
    vec = oracle.pix2vec(nside)
    rng = np.random.default_rng(2)
    mask = (vec[:, 2] > np.cos(np.radians(60.0))).astype(np.float64)
    centres = rng.normal(size=(20, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(1.0))] = 0.0
    mask = oracle.mask_apodization(mask, 2.0, "C1")
    m = np.random.default_rng(1).normal(size=(1, 12 * nside ** 2))
    t0 = time.perf_counter()
    alm = oracle.map2alm(m * mask, 0, nside, lmax, 3)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    mcm = oracle.coupling_tt_closed(oracle.pcl(am, am, lmax)[0], lmax)
    bp = oracle.decouple(oracle.binned_mcm(mcm, lmax, nlb, 1), oracle.pcl(alm, alm, lmax), lmax, nlb)
    sec = time.perf_counter() - t0
    assert np.all(np.isfinite(bp))
    return {"value": 1.0 / sec, "unit": "spectra/s", "seconds": sec, "cores": os.cpu_count(),
            "workload": "Nside 64 spin-0 MASTER estimator from the maps (field and mask transforms "
                        "n_iter=3, exact coupling, binning, decouple), FP64 oracle, not extrapolated"}


def run_reference(args):
    """The CPU arm: each step is one bounded, timed sample of the FP64 oracle's work for
    one Nside 2048 simulation (cpu_oracle_sample); ms_per_step is the sample's measured
    time and `value` the sims/s extrapolated from it (marked `extrapolated`, with the
    sample's share of a simulation), so value * ms_per_step / 1000 is the fraction of a
    simulation one step covered.  The oracle's complete Nside 64 estimator is timed once
    beside it without extrapolation."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = []
    for _ in range(args.warmup + args.steps):
        steps.append(cpu_oracle_sample(args.nside))
    timed = steps[args.warmup:]
    value = float(np.median([s["value"] for s in timed]))
    step_s = float(np.median([s["sample_wall_s"] for s in timed]))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "sims/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * step_s, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "extrapolated": True, "sims_per_step": value * step_s,
        "config": {"workload": f"Nside {args.nside} TQU MASTER simulation, n_iter=3 (a timed sample of "
                               "its transform work per step, extrapolated to sims/s)",
                   "nside": args.nside, "lmax": 3 * args.nside - 1},
        "cpu_baseline": {k: timed[-1][k] for k in ("kind", "cores", "sample", "extrapolated",
                                                   "sample_fraction")} | {"value": value, "unit": "sims/s"},
        "exact_config1": cpu_oracle_config1(),
        "e2e": {"value": value, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU leg

def coupling_triples(lmax):
    """(l1, l2, l3) triples one coupling block visits: every l1 <= l2 pair runs its l3
    recursion over [l2 - l1, l1 + l2], 2 l1 + 1 values."""
    l1 = np.arange(lmax + 1, dtype=np.float64)
    return float(np.sum((2 * l1 + 1) * (lmax - l1 + 1)))


def run_uneven_workspaces(args):
    """Scalar coupling matrices of `nmasks` masks whose Nside is drawn from
    {256, 512, 1024, 2048} (seed 5), lmax = 3 Nside - 1: all blocks from one persistent
    FP64 Wigner-3j launch (coupling_blocks_multi), beside one launch per workspace.  The
    mask spectra are computed before the timed region; a step is the blocks of all masks."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib
    from gmaster_b200 import workspaces as ws

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(5)
    nsides = [int(x) for x in rng.choice([256, 512, 1024, 2048], size=args.nmasks)]
    windows, lmaxs = [], []
    for k, ns in enumerate(nsides):
        mask = make_mask(ns, dev, seed=100 + k, nholes=200 + 10 * k)
        f0 = nmt.NmtField(mask, None, spin=0, precision="mixed")
        pcl = ws.pseudo_cl(f0.get_mask_alms()[None], f0.get_mask_alms()[None],
                           f0.ainfo_mask.lmax)[0] - f0.Nw
        lmax = 3 * ns - 1
        windows.append(pcl[: min(pcl.shape[0], 2 * lmax + 1)].contiguous())
        lmaxs.append(lmax)
        del mask, f0
    torch.cuda.synchronize()
    triples = sum(coupling_triples(l) for l in lmaxs)

    def one_launch(i):
        return ws.coupling_blocks_multi(windows, lmaxs, [1] * len(lmaxs))

    def per_workspace(i):
        return [ws.coupling_blocks(w, l, 1) for w, l in zip(windows, lmaxs)]

    def timed(fn, warmup, steps):
        for i in range(warmup):
            out = fn(i)
            del out
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for i in range(steps):
            out = fn(i)
            del out
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    calls0 = dict(_lib.CALLS)
    sampler = ClockSampler(0)
    sampler.start()
    ms = timed(one_launch, args.warmup, args.steps)
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    ms_each = timed(per_workspace, 1, max(1, args.steps // 2))
    # bit-identical blocks either way
    multi = one_launch(0)
    same = all(torch.equal(m[0], ws.coupling_blocks(w, l, 1)[0])
               for m, w, l in zip(multi, windows, lmaxs))
    line = {
        "metric": "coupling matrices/s, 32 masks of uneven lmax in one FP64 Wigner-3j launch",
        "value": args.nmasks * 1e3 / ms, "unit": "matrices/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded analytic masks)",
        "config": {"workload": f"{args.nmasks} scalar coupling matrices, Nside drawn from "
                               "{256, 512, 1024, 2048} (seed 5), lmax = 3 Nside - 1",
                   "nsides": nsides, "l2_flush": "none needed (the kernel is FP64-bound, "
                                                 "its inputs are windows of a few KB)"},
        "per_workspace_launches": {"ms_per_step": ms_each,
                                   "value": args.nmasks * 1e3 / ms_each},
        "blocks_bit_identical": bool(same),
        "triples_per_s": triples / (ms / 1e3),
        "clocks": clocks,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def run_nside4096(args):
    """Batched transforms at Nside 4096 (lmax 12287): FP32 maps of Gaussian alms with
    C_l = 1/(l+10)^2 (seeds 10 + i), spin 0 and spin 2 (E and B from the same C_l), batches
    of 1, 8 (and 16 spin-0 maps); one step = map2alm with n_iter = 0, or alm2map, of the
    batch.  The transforms run over windows of orders (their single-window operand images
    alone would take 51.5 GB per row variant).  Batch 1 of each spin is also transformed
    by the SIMT mixed-precision path as a cross-check (the FP64 ring stage is limited to
    Nside 2048 by shared memory)."""
    import torch

    from gmaster_b200 import _lib, sht, sht_tc
    from gmaster_b200.utils import NmtAlmInfo

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside = 4096
    lmax = 3 * nside - 1
    ell, order = NmtAlmInfo(lmax).ell_m()
    ell_t = torch.from_numpy(ell).to(dev)
    m0 = torch.from_numpy(order == 0).to(dev)
    amp = torch.from_numpy(1.0 / (np.arange(lmax + 1) + 10.0)).to(dev)[ell_t]

    def alms(n, seed, spin):
        out = torch.empty((n, ell.shape[0]), dtype=torch.complex128, device=dev)
        for i in range(n):
            gen = torch.Generator(device=dev)
            gen.manual_seed(10 + seed + i)
            re = torch.randn(ell.shape[0], generator=gen, device=dev, dtype=torch.float64)
            im = torch.randn(ell.shape[0], generator=gen, device=dev, dtype=torch.float64)
            re[m0] *= np.sqrt(2.0)
            im[m0] = 0.0
            a = torch.complex(re, im) * (amp / np.sqrt(2.0))
            if spin:
                a[ell_t < 2] = 0
            out[i] = a
        return out

    def timed(fn, warmup, steps):
        for _ in range(warmup):
            out = fn()
            del out
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            out = fn()
            del out
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps / 1e3

    cases = []
    calls0 = dict(_lib.CALLS)
    sampler = ClockSampler(0)
    sampler.start()
    for spin, batches in ((0, (1, 8, 16)), (2, (1, 8))):
        for batch in batches:
            ncomp = batch if spin == 0 else 2 * batch
            torch.cuda.reset_peak_memory_stats(dev)
            a = alms(ncomp, 1000 * spin + 100 * batch, spin)
            maps = sht_tc.alm2map_tc(a, spin, nside, lmax).to(torch.float32)
            torch.cuda.empty_cache()
            t_ana = timed(lambda: sht_tc.map2alm_tc(maps, spin, nside, lmax, 0), 1, args.steps)
            t_syn = timed(lambda: sht_tc.alm2map_tc(a, spin, nside, lmax), 1, args.steps)
            case = {"spin": spin, "batch": batch, "maps": ncomp,
                    "map2alm_s": t_ana, "alm2map_s": t_syn,
                    "map2alm_maps_per_s": ncomp / t_ana, "alm2map_maps_per_s": ncomp / t_syn,
                    "window_orders": sht_tc.window_orders(sht_tc.get_tc_plan(nside, lmax, dev), spin, ncomp),
                    "peak_gb": torch.cuda.max_memory_allocated(dev) / 1e9}
            if batch == 1:
                tc = sht_tc.map2alm_tc(maps, spin, nside, lmax, 0)
                simt = sht.map2alm_device(maps.to(torch.float64), spin, nside, lmax, 0, "mixed")
                case["map2alm_rel_diff_vs_simt_mixed"] = float((tc - simt).abs().max() / simt.abs().max())
                del tc, simt
            cases.append(case)
            del a, maps
            torch.cuda.empty_cache()
            print(json.dumps(case), file=sys.stderr, flush=True)
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    best = max(cases, key=lambda c: c["map2alm_maps_per_s"] if c["spin"] == 0 else 0)
    line = {
        "metric": "batched map2alm (n_iter=0) maps/s at Nside 4096, lmax 12287",
        "value": best["map2alm_maps_per_s"], "unit": "maps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": 1, "ms_per_step": best["map2alm_s"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f16x3 tensor-core products (f32 accumulate), f64 recurrence, f32 ring FFTs",
        "data": "synthetic (Gaussian alms, C_l = 1/(l+10)^2, seeds 10+i)",
        "config": {"workload": "Nside 4096 batched transforms, spin 0 batches 1/8/16, spin 2 "
                               "batches 1/8 fields, FP32 maps, windows of orders",
                   "l2_flush": "inputs (0.8 GB per map) larger than L2"},
        "cases": cases, "clocks": clocks, "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def run_mc1024(args):
    """Monte-Carlo loop at Nside 1024 (lmax 3071): 512 TQU simulations (batches of 32, seeds
    1000 + 32 b for batch b) of the configuration spectra through shared workspaces, with
    the config mask recipe at Nside 1024.  Timed three ways on the device: the batched
    estimator (mc_bandpowers, tensor-core transforms, 64 maps per spin-2 launch), the
    per-simulation estimator replayed as one CUDA graph (SimulationGraph, SIMT mixed
    transforms), and the same per-simulation estimator launched eagerly."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside, nlb, S, nsims = 1024, args.nlb, 32, 512
    mask = make_mask(nside, dev)
    _, ws = build_workspaces(mask, nside, nlb, "mixed")
    torch.cuda.synchronize()

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # batched: maps of each batch generated outside the timed region
    calls0 = dict(_lib.CALLS)
    sampler = ClockSampler(0)
    sampler.start()
    t0, qu0 = make_sims(nside, S, 1000, dev)
    for _ in range(args.warmup):
        batch_step(mask, t0, qu0, ws)
    ms_batched = 0.0
    for bi in range(nsims // S):
        t, qu = make_sims(nside, S, 1000 + S * bi, dev)
        torch.cuda.synchronize()
        a, b = events()
        a.record()
        batch_step(mask, t, qu, ws)
        b.record()
        torch.cuda.synchronize()
        ms_batched += a.elapsed_time(b)
        del t, qu
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    # per simulation: graph replays and eager launches of the same pipeline
    graph = nmt.SimulationGraph(mask, ws["00"], ws["02"], ws["22"], n_iter=3, precision="mixed")
    graph(t0[0], qu0[0])
    nper = 32
    torch.cuda.synchronize()
    a, b = events()
    a.record()
    for i in range(nper):
        graph(t0[i], qu0[i])
    b.record()
    torch.cuda.synchronize()
    ms_graph = a.elapsed_time(b) / nper
    estimator_step(mask, t0[:1], qu0[0], ws, "mixed")
    torch.cuda.synchronize()
    a, b = events()
    a.record()
    for i in range(nper):
        estimator_step(mask, t0[i:i + 1], qu0[i], ws, "mixed")
    b.record()
    torch.cuda.synchronize()
    ms_eager = a.elapsed_time(b) / nper
    got = graph(t0[3], qu0[3])
    want = estimator_step(mask, t0[3:4], qu0[3], ws, "mixed")
    gdiff = max(float((g - w).abs().max() / w.abs().max()) for g, w in zip(got, want))
    clocks = sampler.stop()
    line = {
        "metric": "MASTER sims/s, Nside 1024 TQU (shared workspace, n_iter=3), 512 simulations",
        "value": nsims * 1e3 / ms_batched, "unit": "sims/s", "n_gpus": 1, "steps": nsims // S,
        "warmup": args.warmup, "ms_per_step": ms_batched / (nsims // S), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f16x3 tensor-core products (f32 accumulate), f32 difference-form rows restarted "
                 "from f64 checkpoints every 128 rows, f64 alm accumulation, f32 ring FFTs",
        "data": "synthetic (seeded Gaussian TQU sims, config mask recipe at Nside 1024)",
        "config": {"workload": "512 Nside 1024 TQU simulations in batches of 32 through "
                               "mc_bandpowers; per-simulation CUDA graph and eager timings on 32",
                   "nside": nside, "lmax": 3 * nside - 1, "nlb": nlb,
                   "l2_flush": "inputs (100 MB maps, 32 x 3 per batch) larger than L2"},
        "per_simulation_graph": {"ms_per_sim": ms_graph, "value": 1e3 / ms_graph, "unit": "sims/s"},
        "per_simulation_eager": {"ms_per_sim": ms_eager, "value": 1e3 / ms_eager, "unit": "sims/s"},
        "graph_vs_eager_max_rel_diff": gdiff,
        "clocks": clocks, "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def make_mask_gpu(nside, device, seed=4, nholes=10000, hole_arcmin=2.0, cut_deg=20.0, apo_deg=0.5,
                  chunk=1 << 16):
    """The analytic mask recipe of `make_mask` with the pixel centres computed on the GPU in
    chunks (for Nside 8192, where the host pixel vectors would take 19 GB)."""
    import torch

    from gmaster_b200 import sht

    theta, phi0, nphi, offsets = sht.ring_geometry(nside)
    th_t = torch.from_numpy(theta).to(device)
    ph_t = torch.from_numpy(phi0).to(device)
    nphi_t = torch.from_numpy(nphi.astype(np.int64)).to(device)
    off_t = torch.from_numpy(offsets.astype(np.int64)).to(device)
    th, ph = np.radians(30.0), np.radians(45.0)
    pole = torch.tensor([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)],
                        dtype=torch.float64, device=device)
    rng = np.random.default_rng(seed)
    centres = rng.normal(size=(nholes, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    cen = torch.from_numpy(centres).to(device)
    npix = 12 * nside * nside
    r = np.radians(hole_arcmin / 60.0)
    apo = np.radians(apo_deg)
    mask = torch.empty(npix, dtype=torch.float64, device=device)
    for s0 in range(0, npix, chunk):
        pix = torch.arange(s0, min(npix, s0 + chunk), dtype=torch.int64, device=device)
        ring = torch.searchsorted(off_t, pix, right=True) - 1
        phi = ph_t[ring] + 2 * np.pi * (pix - off_t[ring]).to(torch.float64) / nphi_t[ring].to(torch.float64)
        t = th_t[ring]
        vec = torch.stack([torch.sin(t) * torch.cos(phi), torch.sin(t) * torch.sin(phi), torch.cos(t)], 1)
        d = torch.arcsin((vec @ pole).abs().clamp(max=1.0)) - np.radians(cut_deg)
        cosang = (vec @ cen.T).max(dim=1).values.clamp(-1.0, 1.0)
        d = torch.minimum(d, torch.arccos(cosang) - r)
        m = (d > 0).to(torch.float64)
        if apo > 0:
            x = torch.sqrt((1 - torch.cos(d.clamp(min=0))) / (1 - np.cos(apo)))
            m = torch.where((d > 0) & (d < apo), x - torch.sin(2 * np.pi * x) / (2 * np.pi), m)
        mask[s0:s0 + len(pix)] = m
    return mask


def run_nside8192(args):
    """One spin-2 MASTER spectrum at Nside 8192 (lmax 24575): the config mask recipe with
    10000 holes of 2 arcmin and 0.5 deg apodisation, (Q, U) maps of Gaussian E and B alms
    (C_EE = 0.05 C_TT, C_BB = 0.005 C_TT, C_TT = 1e3/(l+10)^2), n_iter = 3, bands of 16; the
    field (with its mask transform), the exact FP64 3j workspace and the decoupled
    bandpowers, then the same with the Toeplitz approximation beside it.  Transforms in
    mixed precision (the one-field SIMT kernels; the ring stage's widest rings go through
    its global-memory path).  Tile tuning is off (it would time every tile at this size)."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib, autotune, sht
    from gmaster_b200.utils import NmtAlmInfo

    autotune.set_autotune(False)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside, nlb = 8192, 16
    lmax = 3 * nside - 1
    t0 = time.perf_counter()
    mask = make_mask_gpu(nside, dev)
    _, ee, bb, _ = config_spectra(lmax)
    ell, order = NmtAlmInfo(lmax).ell_m()
    ell_t = torch.from_numpy(ell).to(dev)
    m0 = torch.from_numpy(order == 0).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(3)

    def unit():
        re = torch.randn(ell.shape[0], generator=gen, device=dev, dtype=torch.float64)
        im = torch.randn(ell.shape[0], generator=gen, device=dev, dtype=torch.float64)
        re[m0] *= np.sqrt(2.0)
        im[m0] = 0.0
        return torch.complex(re, im) / np.sqrt(2.0)

    eb = torch.stack([unit() * torch.from_numpy(np.sqrt(ee)).to(dev)[ell_t],
                      unit() * torch.from_numpy(np.sqrt(bb)).to(dev)[ell_t]])
    qu = sht.alm2map_device(eb, 2, nside, lmax, "mixed")
    del eb
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    torch.cuda.reset_peak_memory_stats(dev)
    calls0 = dict(_lib.CALLS)
    sampler = ClockSampler(0)
    sampler.start()
    marks = []

    def mark(name):
        torch.cuda.synchronize()
        marks.append((name, time.perf_counter()))

    mark("start")
    f2 = nmt.NmtField(mask, qu, spin=2, n_iter=3, precision="mixed")
    f2.get_mask_alms()
    mark("field (maps and mask transforms)")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f2, f2, b)
    mark("workspace (exact 3j coupling, binning, LU)")
    pcl = nmt.compute_coupled_cell(f2, f2)
    cl = w.decouple_cell(pcl)
    mark("spectra")
    del w
    torch.cuda.empty_cache()
    kw = dict(l_toeplitz=nside, l_exact=nside // 4, dl_band=64)
    wt = nmt.NmtWorkspace.from_fields(f2, f2, b, **kw)
    cl_t = wt.decouple_cell(pcl)
    mark("Toeplitz workspace and spectra")
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    stages = {b_[0]: round(b_[1] - a[1], 3) for a, b_ in zip(marks[:-1], marks[1:])}
    s_spec = marks[3][1] - marks[0][1]
    l_eff = b.get_effective_ells()
    fsky = float((mask ** 2).mean())
    sigma = np.sqrt(2.0 / ((2.0 * l_eff + 1.0) * nlb * fsky))
    c, ct = cl.cpu().numpy(), cl_t.cpu().numpy()
    toep = {}
    for i, name in ((0, "EE"), (3, "BB")):
        toep[name] = {"max_rel": float(np.max(np.abs(ct[i] - c[i]) / np.abs(c[i]).max())),
                      "max_in_sigma_cv": float(np.max(np.abs(ct[i] - c[i]) / (sigma * np.abs(c[i]))))}
    # recovered EE against the input spectrum, binned (a sanity check, cosmic variance ~1 %)
    ee_in = b.bin_cell(torch.from_numpy(ee[None]).to(dev)).cpu().numpy()[0]
    sel = (l_eff > 100) & (l_eff < 2 * nside)
    ee_ratio = float(np.median(c[0][sel] / ee_in[sel]))
    line = {
        "metric": "MASTER s/spectrum, Nside 8192 spin 2 (exact FP64 3j workspace), mixed precision",
        "value": s_spec, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0,
        "ms_per_step": s_spec * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 transforms (f64 recurrence and alm accumulation), f64 coupling and LU",
        "data": "synthetic (config mask recipe, 10000 holes of 2 arcmin, 0.5 deg apodisation; "
                "Gaussian E/B alms)",
        "config": {"workload": "one spin-2 spectrum from the maps at Nside 8192, lmax 24575, "
                               "n_iter=3, nlb=16, plus a Toeplitz workspace beside it",
                   "nside": nside, "lmax": lmax, "nlb": nlb, "toeplitz": kw,
                   "l2_flush": "inputs (6.4 GB per map) larger than L2"},
        "stages_s": stages, "setup_s": setup_s,
        "peak_device_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
        "toeplitz_vs_exact": toep, "fsky": fsky,
        "recovered_ee_over_input_median": ee_ratio,
        "clocks": clocks, "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


APO_RECIPES = {2048: dict(nholes=2000, hole_arcmin=5.0, apo_deg=1.0),
               8192: dict(nholes=10000, hole_arcmin=2.0, apo_deg=0.5)}


def kdtree_apodization_sample(mask_np, nside, apo_deg, nquery=2_000_000, seed=0):
    """The reference's C1 apodisation step (gmaster/utils.py:130-146: a scipy k-d tree over the
    masked pixels' unit vectors, one nearest-neighbour query per pixel) timed on the host
    for a bounded sample: the tree over all masked pixels plus `nquery` random pixels,
    the query time scaled to all pixels.  Uses the oracle's pixel vectors."""
    import oracle
    from scipy.spatial import cKDTree

    vec = oracle.pix2vec(nside)
    masked = np.flatnonzero(mask_np <= 0)
    t0 = time.perf_counter()
    tree = cKDTree(vec[masked])
    t1 = time.perf_counter()
    pick = np.random.default_rng(seed).choice(len(mask_np), min(nquery, len(mask_np)), replace=False)
    tree.query(vec[pick])
    t2 = time.perf_counter()
    total = (t1 - t0) + (t2 - t1) * len(mask_np) / len(pick)
    return {"value": total, "unit": "s/mask", "cores": 1, "kind": "port",
            "sample": f"scipy cKDTree over all {len(masked)} masked pixels (built in {t1 - t0:.1f} s) "
                      f"and {len(pick)} of {len(mask_np)} pixel queries ({t2 - t1:.1f} s), "
                      f"query time scaled to all pixels"}


def run_apodize(args):
    """C1 apodisation of binary masks of the configuration recipes (|b| > 20 deg about a
    tilted pole plus holes) on the GPU: Nside 2048 (2000 holes of 5', 1 deg) and Nside
    8192 (10000 holes of 2', 0.5 deg).  One step = gm_mask_ring_runs + gm_mask_apodize
    through `mask_apodization` on a device-resident mask; e2e adds the host->device copy of
    the mask from pinned memory and the copy of the result back."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nsides = [int(x) for x in args.apo_nsides.split(",") if x]
    runs = {}
    for nside in nsides:
        rec = APO_RECIPES.get(nside, APO_RECIPES[2048])
        binary = make_mask_gpu(nside, dev, nholes=rec["nholes"], hole_arcmin=rec["hole_arcmin"],
                               apo_deg=0.0)
        apo = rec["apo_deg"]
        for _ in range(args.warmup):
            nmt.mask_apodization(binary, apo, apotype="C1")
        torch.cuda.synchronize()
        calls0 = dict(_lib.CALLS)
        sampler = ClockSampler(0)
        sampler.start()
        # per-kernel device time: events around each launch on the launching stream
        st = torch.cuda.current_stream(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(st)
        for _ in range(args.steps):
            out = nmt.mask_apodization(binary, apo, apotype="C1")
        ev[1].record(st)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / args.steps
        clocks = sampler.stop()
        launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
        host = binary.cpu().pin_memory()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            res = nmt.mask_apodization(host.to(dev, non_blocking=True), apo, apotype="C1").cpu()
        e1.record(st)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1) / args.steps
        npix = 12 * nside * nside
        tapered = int(((out > 0) & (out < 1)).sum())
        runs[nside] = {"ms": ms, "ms_e2e": ms_e2e, "clocks": clocks, "launches": launches,
                       "npix": npix, "masked": int((binary <= 0).sum()), "tapered": tapered,
                       "apo_deg": apo, "nholes": rec["nholes"], "hole_arcmin": rec["hole_arcmin"],
                       "mask_np": binary.cpu().numpy() if nside == nsides[0] else None}
        del binary, out, res, host
        torch.cuda.empty_cache()
    head = runs[nsides[0]]
    nside0 = nsides[0]
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    # algorithmic bytes per pixel: the mask read by both kernels (16 B), prev/next written
    # (8 B), the output written (8 B)
    algo = 32.0 * head["npix"]
    line = {
        "metric": "mask apodisation s/mask (C1, exact nearest masked pixel)",
        "value": head["ms"] / 1e3, "unit": "s/mask", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (binary config mask recipes, built on the GPU)",
        "config": {"workload": f"C1 apodisation of a binary Nside {nside0} mask "
                               f"({head['nholes']} holes of {head['hole_arcmin']}', |b| > 20 deg) "
                               f"at {head['apo_deg']} deg",
                   "nside": nside0, "l2_flush": f"inputs ({head['npix'] * 8 / 1e6:.0f} MB mask, "
                                                 f"{head['npix'] * 8 / 1e6:.0f} MB prev/next) larger than L2"},
        "e2e": {"value": head["ms_e2e"] / 1e3, "unit": "s/mask",
                "h2d_bytes_per_step": 8 * head["npix"], "d2h_bytes_per_step": 8 * head["npix"]},
        "roofline": {"bound": "hbm", "achieved": algo / (head["ms"] / 1e3) / 1e9, "peak": hbm,
                     "unit": "GB/s", "frac": algo / (head["ms"] / 1e3) / 1e9 / hbm, "traffic": None,
                     "note": "both kernels of one step against their algorithmic bytes (32 B per "
                             "pixel); the ring search is instruction-bound, not HBM-bound"},
        "per_nside": {str(n): {k: v for k, v in r.items() if k != "mask_np"} for n, r in runs.items()},
        "clocks": head["clocks"], "gpu_launches": int(head["launches"]),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = kdtree_apodization_sample(head["mask_np"], nside0, head["apo_deg"])
    print(json.dumps(line), flush=True)


def run_covariance(args):
    """Gaussian covariance at Nside 2048 (lmax 6143, bands of 16) on the config mask: the
    covariance workspace (mask-product transform, 3j kernels) and the decoupled bandpower
    covariance, for TT x TT (spins 0,0,0,0), TE x TE (0,2,0,2) and the spin-2 auto
    covariance (2,2,2,2) with iNKA input spectra."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside, nlb = args.nside, args.nlb
    lmax = 3 * nside - 1
    mask = make_mask(nside, dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(7)
    t = torch.randn((1, 12 * nside * nside), generator=gen, device=dev, dtype=torch.float64)
    qu = torch.randn((2, 12 * nside * nside), generator=gen, device=dev, dtype=torch.float64)
    f0 = nmt.NmtField(mask, t, n_iter=0, precision="mixed")
    f2 = nmt.NmtField(mask, qu, spin=2, n_iter=0, precision="mixed")
    f0.get_mask_alms()
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    ws = {(0, 0): nmt.NmtWorkspace.from_fields(f0, f0, b),
          (0, 2): nmt.NmtWorkspace.from_fields(f0, f2, b),
          (2, 2): nmt.NmtWorkspace.from_fields(f2, f2, b)}
    fld = {0: f0, 2: f2}
    cells = {}
    for s1, s2 in ((0, 0), (0, 2), (2, 0), (2, 2)):
        cells[(s1, s2)] = nmt.get_iNKA_cell(fld[s1], fld[s2])
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    calls0 = dict(_lib.CALLS)
    res = {}
    st = torch.cuda.current_stream(dev)
    for spins in ((0, 0, 0, 0), (0, 2, 0, 2), (2, 2, 2, 2)):
        a1, a2, b1, b2 = (fld[s] for s in spins)
        for _ in range(args.warmup):
            cw = nmt.NmtCovarianceWorkspace.from_fields(a1, a2, b1, b2)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(st)
        for _ in range(args.steps):
            cw = nmt.NmtCovarianceWorkspace.from_fields(a1, a2, b1, b2)
        e[1].record(st)
        cl = (cells[(spins[0], spins[2])], cells[(spins[0], spins[3])],
              cells[(spins[1], spins[2])], cells[(spins[1], spins[3])])
        wa, wb = ws[(spins[0], spins[1])], ws[(spins[2], spins[3])]
        for _ in range(args.steps):
            cov = cw.gaussian_covariance(*cl, wa, wb)
        e[2].record(st)
        torch.cuda.synchronize()
        res["".join(map(str, spins))] = {
            "workspace_s": e[0].elapsed_time(e[1]) / 1e3 / args.steps,
            "covariance_s": e[1].elapsed_time(e[2]) / 1e3 / args.steps,
            "shape": list(cov.shape),
            "min_diag": float(torch.diagonal(cov).min()),
        }
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    head = res["2222"]
    line = {
        "metric": "Gaussian covariance s (workspace + decoupled bandpower covariance), Nside 2048",
        "value": head["workspace_s"] + head["covariance_s"], "unit": "s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": (head["workspace_s"] + head["covariance_s"]) * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (mask transforms mixed precision)",
        "data": "synthetic (config mask recipe; iNKA spectra of Gaussian maps)",
        "config": {"workload": f"NKA covariance of the spin-2 auto spectrum (2,2,2,2), Nside "
                               f"{nside}, lmax {lmax}, bands of {nlb}; TT and TE beside it",
                   "nside": nside, "lmax": lmax, "nlb": nlb},
        "per_spins": res, "clocks": clocks, "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def run_purify(args):
    """E/B purification at Nside 2048 (lmax 6143) on the config mask: a plain and a
    purified-B spin-2 field (mixed precision, n_iter 3), their 2x2 workspaces (bands of 16;
    the purified one by Gauss-Legendre quadrature) and the purified bandpowers.  Wall
    times around synchronised steps (each stage is seconds long)."""
    import torch

    import gmaster_b200 as nmt
    from gmaster_b200 import _lib, autotune

    autotune.set_autotune(False)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside, nlb = args.nside, args.nlb
    mask = make_mask(nside, dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1)
    qu = torch.randn((2, 12 * nside * nside), generator=gen, device=dev, dtype=torch.float64)
    nmt.NmtField(mask, qu, spin=2, n_iter=3, precision="mixed")   # warm-up (plans, mask alms)
    torch.cuda.synchronize()
    calls0 = dict(_lib.CALLS)
    sampler = ClockSampler(0)
    sampler.start()
    marks = [time.perf_counter()]

    def mark():
        torch.cuda.synchronize()
        marks.append(time.perf_counter())

    f_plain = nmt.NmtField(mask, qu, spin=2, n_iter=3, precision="mixed")
    mark()
    f_pure = nmt.NmtField(mask, qu, spin=2, purify_b=True, n_iter=3, precision="mixed")
    mark()
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    nmt.NmtWorkspace.from_fields(f_plain, f_plain, b)
    mark()
    w_pure = nmt.NmtWorkspace.from_fields(f_pure, f_pure, b)
    mark()
    w_pure.decouple_cell(nmt.compute_coupled_cell(f_pure, f_pure))
    mark()
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    d = [b_ - a for a, b_ in zip(marks[:-1], marks[1:])]
    total = d[1] + d[3] + d[4]
    line = {
        "metric": "purified-B spectrum s (purified field, purified 2x2 workspace, bandpowers), Nside 2048",
        "value": total, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": total * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 transforms (f64 recurrence), f64 quadrature and LU",
        "data": "synthetic (config mask recipe; Gaussian (Q, U) maps)",
        "config": {"workload": f"purified-B spin-2 field and 2x2 workspace at Nside {nside}, "
                               f"lmax {3 * nside - 1}, n_iter 3, bands of {nlb}",
                   "nside": nside, "nlb": nlb},
        "stages_s": {"plain field": d[0], "purified field": d[1], "plain 2x2 workspace": d[2],
                     "purified 2x2 workspace": d[3], "spectra": d[4]},
        "peak_device_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
        "clocks": clocks, "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "uneven_workspaces":
        run_uneven_workspaces(args)
        return
    if args.workload == "nside4096":
        run_nside4096(args)
        return
    if args.workload == "mc1024":
        run_mc1024(args)
        return
    if args.workload == "nside8192":
        run_nside8192(args)
        return
    if args.workload == "apodize":
        run_apodize(args)
        return
    if args.workload == "covariance":
        run_covariance(args)
        return
    if args.workload == "purify":
        run_purify(args)
        return
    import torch
    import torch.distributed as dist

    from gmaster_b200 import _lib, sht

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
    nside, nlb, S = args.nside, args.nlb, args.batch
    lmax = 3 * nside - 1
    mask = make_mask(nside, dev)
    t_all, qu_all = make_sims(nside, S, 1000 + 7919 * rank, dev)
    torch.cuda.synchronize()

    # per-geometry constants of the tensor-core and one-field mixed paths (the checkpoint
    # tables of the spin-0 and spin-2 rows), built once and kept, as the reference keeps its
    # window tables (march_v2.py:388-450): their build time is reported on its own
    from gmaster_b200 import sht_tc

    tp = sht_tc.get_tc_plan(nside, lmax, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ck_built = [sht_tc.ck_tables(tp, sp) is not None for sp in (0, 2)]
    torch.cuda.synchronize()
    table_ms = 1e3 * (time.perf_counter() - t0)
    kernel_of = KERNEL_OF if all(ck_built) else KERNEL_OF_CARRIED

    # full estimator from scratch for one simulation (seconds per spectrum)
    s_per_spec = {}
    spec_stages = {}
    for prec in ("mixed", "fp64"):
        full_estimator(mask, t_all[:1], qu_all[0], nside, nlb, prec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        full_estimator(mask, t_all[:1], qu_all[0], nside, nlb, prec)
        torch.cuda.synchronize()
        s_per_spec[prec] = time.perf_counter() - t0
        stages = {}
        full_estimator(mask, t_all[:1], qu_all[0], nside, nlb, prec, stages=stages)
        spec_stages[prec] = {k: round(v, 2) for k, v in stages.items()}

    _, ws_mixed = build_workspaces(mask, nside, nlb, "mixed")
    torch.cuda.synchronize()
    # a step holds ~176 GB at this size: the cached blocks of the runs above are released
    # so the warm-up steps lay out the allocator's cache for the step's own buffers
    torch.cuda.empty_cache()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_loop(fn, warmup, steps):
        for i in range(warmup):
            fn(i)
        barrier()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record()
        for i in range(steps):
            fn(i)
        end.record()
        barrier()
        return max_over_ranks(start.elapsed_time(end), dev)

    # device-resident value (mixed, batched), with Legendre kernel events and clocks
    for i in range(args.warmup):
        batch_step(mask, t_all, qu_all, ws_mixed)
    sampler = ClockSampler(local)
    sht.TIMER = []
    calls0 = dict(_lib.CALLS)
    sampler.start()
    torch.cuda.nvtx.range_push("bench_timed")
    ms = timed_loop(lambda i: batch_step(mask, t_all, qu_all, ws_mixed), 0, args.steps)
    torch.cuda.nvtx.range_pop()
    clocks = sampler.stop()
    launches = sum(_lib.CALLS.get(k, 0) - calls0.get(k, 0) for k in _lib.CALLS)
    events = list(sht.TIMER)
    sht.TIMER = None
    torch.cuda.synchronize()
    ktime, kflops, kcount = {}, {}, {}
    for kind, a, b, fl in events:
        ktime[kind] = ktime.get(kind, 0.0) + a.elapsed_time(b)
        kflops[kind] = kflops.get(kind, 0.0) + fl
        kcount[kind] = kcount.get(kind, 0) + 1
    leg_ms = sum(ktime.values())
    leg_flops = sum(kflops.values())
    dominant = max(ktime, key=ktime.get)
    value = throughput(world, args.steps, S, ms)
    mixed_bp = [o[0].cpu().numpy() for o in batch_step(mask, t_all, qu_all, ws_mixed)]

    # plain FP64 GPU path, one simulation at a time, and the unbatched mixed path
    _, ws_fp64 = build_workspaces(mask, nside, nlb, "fp64")
    t0_dev, qu0_dev = t_all[:1].clone(), qu_all[0].clone()
    ms64 = timed_loop(lambda i: estimator_step(mask, t0_dev, qu0_dev, ws_fp64, "fp64"), 1,
                      args.fp64_steps)
    value64 = throughput(world, args.fp64_steps, 1, ms64)
    fp64_bp = [o.cpu().numpy() for o in estimator_step(mask, t0_dev, qu0_dev, ws_fp64, "fp64")]
    ms1 = timed_loop(lambda i: estimator_step(mask, t0_dev, qu0_dev, ws_mixed, "mixed"), 1, 1)
    errs = {}
    for name, a, b in zip(("00", "02", "22"), mixed_bp, fp64_bp):
        scale = np.max(np.abs(b), axis=1, keepdims=True)
        errs[name] = float(np.max(np.abs(a - b) / scale))
    auto = [(mixed_bp[0][0], fp64_bp[0][0]), (mixed_bp[2][0], fp64_bp[2][0]),
            (mixed_bp[2][3], fp64_bp[2][3])]
    rel_auto = float(max(np.max(np.abs(a - b) / np.abs(b)) for a, b in auto))
    # the same differences in units of the Gaussian cosmic variance of each band,
    # sigma_b = sqrt(2 / ((2 l_b + 1) nlb f_sky)) |C_b| (f_sky = mean of the squared mask)
    import gmaster_b200 as nmt

    l_eff = nmt.NmtBin.from_nside_linear(nside, nlb).get_effective_ells()
    fsky = float((mask ** 2).mean())
    sig_cv = {}
    for name, (a, b) in zip(("TT", "EE", "BB"), auto):
        sigma = np.sqrt(2.0 / ((2.0 * l_eff + 1.0) * nlb * fsky)) * np.abs(b)
        sig_cv[name] = float(np.max(np.abs(a - b) / sigma))

    # e2e through the public API from pinned host memory (device copies released first)
    t_host = t_all.cpu()
    qu_host = qu_all.cpu()
    del t_all, qu_all
    torch.cuda.empty_cache()
    try:
        t_host, qu_host = t_host.pin_memory(), qu_host.pin_memory()
        pinned = True
    except RuntimeError:
        pinned = False
    h2d = t_host.numel() * 8 + qu_host.numel() * 8
    d2h = [0]

    def e2e_step(i):
        out = batch_step(mask, t_host, qu_host, ws_mixed)
        d2h[0] = sum(o.numel() * 8 for group in out for o in group)
        for group in out:
            for o in group:
                o.cpu()

    ms_e2e = timed_loop(e2e_step, 1, args.steps)
    value_e2e = throughput(world, args.steps, S, ms_e2e)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    # the Legendre kernels are timed inside seconds-long steps: sustained bf16 peak
    peak = peaks.get("bf16_tflops_sustained", 1400.0)
    # a spin-2 pass is two launches of the kernel (row variants s' = -2, +2) of equal work
    per_pass = 2 if dominant.endswith("_s2") else 1
    dom_launches = kcount[dominant] * per_pass
    dom_avg_ms = ktime[dominant] / dom_launches
    dom_tflops = kflops[dominant] / (ktime[dominant] / 1e3) / 1e12
    dom_kernel = kernel_of.get(dominant, dominant)
    activity = ck_unit_activity(nside, lmax) if dom_kernel == "k_ana_ck<2>" else None
    traffic = traffic_per_launch(dom_kernel, nside, lmax, S, activity)
    if activity is not None:
        issued_tflops = ck_issued_flops(activity) / (dom_avg_ms / 1e3) / 1e12
        active_frac = float(np.bitwise_count(activity[0]).sum()) / (len(activity[0]) * ((2 * nside + 63) // 64))
    else:
        issued_tflops, active_frac = 3 * dom_tflops, 1.0
    line = {
        "metric": METRIC, "value": value, "unit": "sims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16x3 tensor-core products (f32 accumulate), f32 difference-form rows restarted "
                 "from f64 checkpoints every 128 rows, f64 alm accumulation, f32 ring FFTs",
        "data": "synthetic (seeded Gaussian TQU sims and analytic mask of the Nside 2048 recipe)",
        "config": {
            "workload": f"batch of {S} Nside {nside} TQU simulations through fields_from_maps x2, "
                        f"compute_coupled_cells x3, decouple_cells x3 (shared workspaces), "
                        f"n_iter=3, nlb={nlb}",
            "nside": nside, "lmax": lmax, "nlb": nlb, "sims_per_step": S,
            "l2_flush": "inputs (400 MB maps) larger than L2", "parallelism": f"replicas{world}",
        },
        "e2e": {"value": value_e2e, "unit": "sims/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h[0]), "pinned": pinned},
        "roofline": {
            "bound": "tensor", "kernel": dom_kernel,
            "achieved": dom_tflops, "peak": peak, "unit": "TFLOP/s",
            "frac": dom_tflops / peak,
            "traffic": traffic[1],
            "traffic_model_bytes": traffic[0],
            "note": "algorithmic flops per launch (one complex MAC = 4 flops per (l, m, lane) and "
                    "map, every (l, m, lane) counted) / CUDA-event time of the launch; the kernel "
                    "skips the 64-lane groups whose rows are exactly zero and issues three f16 "
                    "products per active group (tensor_pipe_tflops_issued); peak = measured "
                    "sustained bf16 dense (MEASURED_PEAKS.json); traffic = DRAM bytes read + "
                    f"written per launch: ncu measured {CK_TRAFFIC_RATIO:.3f}x the launch's "
                    "mask-aware byte model at Nside 512 (8 fields); the model of this workload "
                    f"x {CK_TRAFFIC_RATIO:.3f}",
            "launches": dom_launches, "avg_ms": dom_avg_ms,
            "tensor_pipe_tflops_issued": issued_tflops,
            "active_group_fraction": active_frac,
        },
        "legendre_share_of_step": leg_ms / ms,
        "legendre_tflops": leg_flops / (leg_ms / 1e3) / 1e12,
        "fp64": {"value": value64, "unit": "sims/s", "ms_per_sim": ms64 / args.fp64_steps,
                 "path": "plain FP64 GPU estimator, one simulation at a time"},
        "mixed_unbatched": {"value": world * 1e3 / ms1, "unit": "sims/s", "ms_per_sim": ms1},
        "speedup_mixed_vs_fp64": value / value64,
        "s_per_spectrum": s_per_spec,
        "s_per_spectrum_stages_ms": spec_stages,
        "geometry_tables": {"checkpoint_tables_built": all(ck_built), "build_ms": table_ms,
                            "gb": sum(sht_tc.ck_table_bytes(tp, sp) for sp in (0, 2)) / 1e9,
                            "note": "checkpoint tables of the spin-0 and spin-2 rows at this Nside, "
                                    "built once per geometry before the timed regions and kept"},
        "peak_device_gb": torch.cuda.max_memory_allocated(dev) / 1e9,
        "bandpower_err_mixed_vs_fp64": {"max_abs_over_scale": errs, "max_rel_auto": rel_auto,
                                        "max_in_sigma_cv": sig_cv, "fsky": fsky},
        "clocks": clocks,
        "gpu_launches": int(launches),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = {k: v for k, v in cpu_oracle_sample(nside).items()
                                if k in ("value", "unit", "cores", "kind", "sample", "extrapolated",
                                         "sample_fraction")}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
