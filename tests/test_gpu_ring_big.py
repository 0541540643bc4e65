"""The global-memory ring path (rings that do not fit the shared-memory kernels: Nside
above 4096 in single precision, above 2048 in double precision) against the shared-memory
kernels, forced onto small rings with the tuning knobs: belt rings through the global
Stockham FFT, the large-prime cap rings through the global Bluestein transform (single
precision) or the mixed-radix FFT (double precision), analysis and synthesis; and the FP64
transform at Nside 4096 against the oracle."""

import numpy as np
import pytest
import torch

from gmaster_b200 import _lib, sht

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.fixture
def forced():
    def set_(hcap, bs):
        sht.RING_TUNING.update(hcap_max=hcap, bs_min=bs)
    yield set_
    sht.RING_TUNING.update(hcap_max=0, bs_min=0)


@pytest.mark.parametrize("hcap,bs", [(100, 0), (100000, 16), (100, 16)])
def test_global_ring_analysis_matches_shared(cuda, forced, hcap, bs):
    nside, lmax = 256, 767
    plan = sht.get_plan(nside, lmax)
    rng = np.random.default_rng(3)
    maps = torch.from_numpy(rng.normal(size=(3, plan.npix))).cuda()
    mask = torch.from_numpy(rng.uniform(size=plan.npix)).cuda()
    ref = sht.ring_analysis(plan, maps, _lib.MIXED, mask=mask)
    forced(hcap, bs)
    got = sht.ring_analysis(plan, maps, _lib.MIXED, mask=mask)
    assert _rel(got, ref) < 2e-6


@pytest.mark.parametrize("hcap,bs", [(100, 0), (100000, 16), (100, 16)])
def test_global_ring_synthesis_matches_shared(cuda, forced, hcap, bs):
    nside, lmax = 256, 767
    plan = sht.get_plan(nside, lmax)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4)
    syn = torch.randn((plan.L, plan.nlanes, 2, 4), generator=gen, dtype=torch.float32, device="cuda")
    ref = sht.ring_synthesis(plan, syn, _lib.MIXED)
    forced(hcap, bs)
    got = sht.ring_synthesis(plan, syn, _lib.MIXED)
    assert _rel(got, ref) < 2e-6


def test_global_ring_path_in_a_transform(cuda, forced):
    """A mixed-precision map2alm with three Jacobi iterations gives the same alms with
    every ring routed through the global path."""
    nside, lmax = 128, 383
    rng = np.random.default_rng(5)
    maps = torch.from_numpy(rng.normal(size=(2, 12 * nside ** 2))).cuda()
    ref = sht.map2alm_device(maps, 2, nside, lmax, 3, "mixed")
    forced(8, 16)
    got = sht.map2alm_device(maps, 2, nside, lmax, 3, "mixed")
    assert _rel(got, ref) < 1e-5


@pytest.mark.parametrize("hcap", [100, 513])
def test_global_ring_path_fp64_matches_shared(cuda, forced, hcap):
    """Double precision through the global path (every ring above `hcap`, large primes
    included, by the mixed-radix FFT) equals the shared-memory FP64 kernels to rounding,
    analysis and synthesis."""
    nside, lmax = 256, 767
    plan = sht.get_plan(nside, lmax)
    rng = np.random.default_rng(7)
    maps = torch.from_numpy(rng.normal(size=(2, plan.npix))).cuda()
    mask = torch.from_numpy(rng.uniform(size=plan.npix)).cuda()
    ref = sht.ring_analysis(plan, maps, _lib.FP64, mask=mask)
    syn = torch.randn((plan.L, plan.nlanes, 2, 4), dtype=torch.float64, device="cuda")
    ref_s = sht.ring_synthesis(plan, syn, _lib.FP64)
    forced(hcap, 0)
    assert _rel(sht.ring_analysis(plan, maps, _lib.FP64, mask=mask), ref) < 1e-13
    assert _rel(sht.ring_synthesis(plan, syn, _lib.FP64), ref_s) < 1e-13


def test_fp64_transform_at_nside4096_matches_oracle_orders(cuda):
    """The plain FP64 path above Nside 2048 (belt rings of 8192 complex doubles through the
    global path): map2alm without refinement at Nside 4096 against the oracle on sampled
    orders, to 1e-10 of their scale."""
    import oracle

    nside, lmax = 4096, 12287
    rng = np.random.default_rng(8)
    maps = torch.from_numpy(rng.normal(size=(1, 12 * nside ** 2))).cuda()
    orders = [0, 5, 6000, 12280]
    got = sht.map2alm_device(maps, 0, nside, lmax, 0, "fp64").cpu().numpy()[0]
    want = oracle.ana0_orders(maps[0].cpu().numpy(), nside, lmax, orders)
    L = lmax + 1
    err = 0.0
    for i, m in enumerate(orders):
        base = m * (2 * lmax + 1 - m) // 2
        err = max(err, float(np.max(np.abs(got[base + m:base + L] - want[i, m:]))))
    assert err < 1e-10 * float(np.max(np.abs(want)))
