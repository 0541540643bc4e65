"""The multi-rank timing of bench.py on CPU: world size 2 over gloo (no GPU)."""

import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench = _bench()
        ms = 1000.0 + 250.0 * rank          # rank 1 is the slow one
        top = bench.max_over_ranks(ms, "cpu")
        out[rank] = (top, bench.throughput(world, 3, 32, top))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_throughput_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        top, value = out[r]
        assert top == pytest.approx(1250.0)
        assert value == pytest.approx(2 * 3 * 32 / 1.25)


def test_single_process_is_identity():
    bench = _bench()
    assert bench.max_over_ranks(7.5, "cpu") == 7.5
    assert bench.throughput(1, 4, 32, 2000.0) == pytest.approx(64.0)


def test_ck_byte_model_with_unit_masks():
    """The mask-aware byte model of the checkpointed analysis launch equals the unmasked
    model (up to the per-unit rounding of its segment count) when every lane group is
    active, and drops the images, alm rows and states of inactive units."""
    import numpy as np

    bench = _bench()
    nside, lmax, nrows = 64, 191, 32
    L = lmax + 1
    uoff = np.zeros(L + 1, dtype=np.int64)
    for m in range(L):
        uoff[m + 1] = uoff[m] + (L - max(m, 2) + 255) // 256
    ngk = (2 * nside + 63) // 64
    full = np.full(uoff[-1], (1 << ngk) - 1, dtype=np.uint64)
    plain = bench.ck_analysis_bytes(nside, lmax, nrows)
    masked = bench.ck_analysis_bytes(nside, lmax, nrows, (full, uoff))
    assert abs(masked / plain - 1.0) < 0.01
    none = np.zeros_like(full)
    assert bench.ck_analysis_bytes(nside, lmax, nrows, (none, uoff)) == 0
    half = full.copy()
    half[::2] = 0
    assert 0 < bench.ck_analysis_bytes(nside, lmax, nrows, (half, uoff)) < masked
    assert bench.ck_issued_flops((full, uoff)) == 3 * 2 * 128 * 256 * 64 * int(uoff[-1]) * ngk
