"""Tile autotuner for the SIMT Legendre kernels.

The one-field (SIMT) analysis and synthesis kernels come in several compiled tile shapes
(NC, R): NC components (maps, or one (Q, U) pair) per CTA and R lanes (rings) per thread.
Which is fastest depends on the geometry, the number of maps and the precision, so the
tuner times every shape on operands of the real size, with CUDA events, the first time a
(device, kind, precision, spin, nside, lmax, ncomp) combination is transformed, and keeps
the fastest.  The reference fixes its march tiles by rule (march_v2.py:290-332).

Tuning is on by default; ``set_autotune(False)`` or ``GMASTER_B200_AUTOTUNE=0`` turns it
off, and the kernels' built-in choice runs.  Tuning launches kernels and waits on events,
so a transform captured in a CUDA graph must have run once before the capture (its choice
is then cached).  Choices live in memory; with
``GMASTER_B200_TUNE_CACHE`` naming a JSON file they are also read from and written to it.
"""

import ctypes
import json
import os
import threading

import torch

from . import _lib

_CACHE = {}
_TIMINGS = {}
_LOCK = threading.Lock()
_STATE = {"enabled": os.environ.get("GMASTER_B200_AUTOTUNE", "1") != "0", "loaded": False}


def set_autotune(flag):
    """Enable or disable tile tuning of the SIMT Legendre kernels."""
    _STATE["enabled"] = bool(flag)


def autotune_enabled():
    return _STATE["enabled"]


def tiles(spin):
    """The (NC, R) tile shapes compiled for `spin`."""
    buf = (ctypes.c_int32 * 64)()
    n = _lib.load().gm_legendre_tiles(int(spin), buf, 32)
    if n < 0:
        raise ValueError("no tiles for this spin (spins 0..8 have tiles)")
    return [(buf[2 * i], buf[2 * i + 1]) for i in range(n)]


def _cache_file():
    return os.environ.get("GMASTER_B200_TUNE_CACHE")


def _load():
    if _STATE["loaded"]:
        return
    _STATE["loaded"] = True
    path = _cache_file()
    if path and os.path.exists(path):
        with open(path) as fh:
            for k, v in json.load(fh).items():
                _CACHE[k] = int(v)


def _save():
    path = _cache_file()
    if path:
        with open(path, "w") as fh:
            json.dump(_CACHE, fh, indent=1, sort_keys=True)


def _key(plan, spin, ncomp, prec, kind, ck=False):
    name = torch.cuda.get_device_name(plan.device).replace(" ", "_").replace(":", "_")
    return f"{name}:{kind}:p{prec}:s{spin}:n{plan.nside}:l{plan.lmax}:c{ncomp}" + (":ck" if ck else "")


def tune(plan, spin, ncomp, prec, kind, reps=2):
    """Time every tile of `kind` ("ana" or "syn") on operands of the real size; returns
    (best tile index, {tile index: ms per pass})."""
    dev = plan.device
    real = torch.float64 if prec == _lib.FP64 else torch.float32
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    rhs = torch.randn((plan.L, plan.nlanes, ncomp, 4), generator=gen, dtype=real, device=dev)
    alm = torch.zeros((ncomp, plan.nelem), dtype=torch.complex128, device=dev)
    if kind == "ana":
        a, b = rhs, alm
    else:
        alm.real.normal_(generator=gen)
        a, b = alm, rhs
    from . import sht

    ck = sht.ck_args(plan, spin, prec)
    times = {}
    for t in range(len(tiles(spin))):
        sht.run_legendre(plan, spin, ncomp, prec, kind, t, a, b, ck=ck)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            sht.run_legendre(plan, spin, ncomp, prec, kind, t, a, b, ck=ck)
        e1.record()
        e1.synchronize()
        times[t] = e0.elapsed_time(e1) / reps
    del rhs, alm
    best = min(times, key=times.get)
    return best, times


def tile_for(plan, spin, ncomp, prec, kind):
    """Tile index for this transform (-1: the built-in choice when tuning is off)."""
    if not _STATE["enabled"]:
        return -1
    from . import sht

    key = _key(plan, spin, ncomp, prec, kind, sht.ck_args(plan, spin, prec) is not None)
    with _LOCK:
        _load()
        if key not in _CACHE:
            best, times = tune(plan, spin, ncomp, prec, kind)
            _CACHE[key] = best
            _TIMINGS[key] = times
            _save()
        return _CACHE[key]


def choices():
    """{key: (chosen tile (NC, R), timings in ms per tile)} of this process."""
    out = {}
    for k, v in _CACHE.items():
        spin = int(next(f for f in k.split(":") if f.startswith("s") and f[1:].isdigit())[1:])
        out[k] = (tiles(spin)[v], _TIMINGS.get(k))
    return out

