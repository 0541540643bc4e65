"""The global-memory ring path (rings that do not fit the shared-memory kernels: Nside
above 4096) against the shared-memory kernels, forced onto small rings with the tuning
knobs: belt rings through the global Stockham FFT, the large-prime cap rings through the
global Bluestein transform (analysis and synthesis)."""

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
