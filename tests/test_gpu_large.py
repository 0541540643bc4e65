"""The transforms at the benchmark resolutions against the FP64 oracle on sampled orders.

At Nside 2048 (lmax 6143, the Monte-Carlo configuration) and Nside 4096 (lmax 12287, the
transform benchmark) the oracle's analysis of a few orders (ring FFTs of every ring, then
the Legendre sums of those orders only) is compared with the plain FP64 GPU path (1e-10 of
the sampled alms' scale), the mixed one-field path with checkpointed single-precision rows
(2e-5) and the batched tensor-core path (5e-5).  The sampled orders include m = 0 and 1,
orders near lmax whose seeds sit far below the single-precision range, and orders in
between.  Maps are seeded Gaussian realisations of C_l = 1e3 / (l + 10)^2 (l >= 2)."""

import numpy as np
import pytest
import torch

import oracle
from gmaster_b200 import sht, sht_tc

pytestmark = pytest.mark.gpu

ORDERS = {2048: [0, 1, 517, 2048, 3071, 5000, 6140], 4096: [0, 3, 4095, 9000, 12286]}


def _gaussian_maps(nside, ncomp, seed, spin=0):
    lmax = 3 * nside - 1
    L = lmax + 1
    ell = torch.cat([torch.arange(m, L) for m in range(L)]).cuda().to(torch.float64)
    order = torch.cat([torch.full((L - m,), m) for m in range(L)]).cuda()
    cl = torch.where(ell >= 2, 1e3 / (ell + 10.0) ** 2, torch.zeros_like(ell))
    g = torch.Generator(device="cuda").manual_seed(seed)
    nrows = ncomp
    re = torch.randn((nrows, len(ell)), generator=g, device="cuda", dtype=torch.float64)
    im = torch.randn((nrows, len(ell)), generator=g, device="cuda", dtype=torch.float64)
    im[:, order == 0] = 0.0
    alm = torch.complex(re, im) * torch.sqrt(cl / 2.0)[None]
    alm[:, order == 0] *= np.sqrt(2.0)
    # the FP64 ring stage stops at Nside 2048: larger maps are synthesised in mixed precision
    # (they are the common input of both sides, so their own precision does not matter)
    return sht.alm2map_device(alm, spin, nside, lmax, "fp64" if nside <= 2048 else "mixed")


def _sampled(alm, lmax, orders):
    """(nrows, len(orders), L) complex: the rows' alms of the sampled orders (0 below l = m)."""
    L = lmax + 1
    out = np.zeros((alm.shape[0], len(orders), L), dtype=np.complex128)
    for i, m in enumerate(orders):
        base = m * (2 * lmax + 1 - m) // 2   # healpy index of (l, m) = base + l
        out[:, i, m:] = alm[:, base + m:base + L]
    return out


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


def test_nside2048_spin0_paths_match_oracle_on_sampled_orders(cuda):
    nside, lmax = 2048, 6143
    orders = ORDERS[nside]
    maps = _gaussian_maps(nside, 4, 3)
    want = oracle.ana0_orders(maps[0].cpu().numpy(), nside, lmax, orders)
    errs = {}
    fp64 = sht.map2alm_device(maps[:1], 0, nside, lmax, 0, "fp64").cpu().numpy()
    errs["fp64"] = _rel(_sampled(fp64, lmax, orders)[0], want)
    mixed = sht.map2alm_device(maps[:1], 0, nside, lmax, 0, "mixed").cpu().numpy()
    errs["mixed"] = _rel(_sampled(mixed, lmax, orders)[0], want)
    tc = sht_tc.map2alm_tc(maps, 0, nside, lmax, 0).cpu().numpy()
    errs["tensor"] = _rel(_sampled(tc[:1], lmax, orders)[0], want)
    print("Nside 2048 spin 0 alm error vs oracle (of scale):", errs)
    assert errs["fp64"] < 1e-10 and errs["mixed"] < 2e-5 and errs["tensor"] < 5e-5


def test_nside2048_spin2_paths_match_oracle_on_sampled_orders(cuda):
    nside, lmax = 2048, 6143
    orders = ORDERS[nside]
    maps = _gaussian_maps(nside, 4, 4, spin=2)   # two (Q, U) fields
    want = oracle.ana2_orders(maps[:2].cpu().numpy(), nside, lmax, orders)   # (orders, 2, L)
    want = np.transpose(want, (1, 0, 2))
    errs = {}
    fp64 = sht.map2alm_device(maps[:2], 2, nside, lmax, 0, "fp64").cpu().numpy()
    errs["fp64"] = _rel(_sampled(fp64, lmax, orders), want)
    mixed = sht.map2alm_device(maps[:2], 2, nside, lmax, 0, "mixed").cpu().numpy()
    errs["mixed"] = _rel(_sampled(mixed, lmax, orders), want)
    tc = sht_tc.map2alm_tc(maps, 2, nside, lmax, 0).cpu().numpy()
    errs["tensor"] = _rel(_sampled(tc[:2], lmax, orders), want)
    print("Nside 2048 spin 2 alm error vs oracle (of scale):", errs)
    assert errs["fp64"] < 1e-10 and errs["mixed"] < 2e-5 and errs["tensor"] < 5e-5


@pytest.mark.parametrize("spin", [0, 2])
def test_nside4096_tensor_core_matches_oracle_on_sampled_orders(cuda, spin):
    nside, lmax = 4096, 12287
    orders = ORDERS[nside]
    ncomp = 1 if spin == 0 else 2
    maps = _gaussian_maps(nside, ncomp, 5 + spin, spin=spin)
    host = maps.cpu().numpy()
    if spin == 0:
        want = oracle.ana0_orders(host[0], nside, lmax, orders)[None]
    else:
        want = np.transpose(oracle.ana2_orders(host, nside, lmax, orders), (1, 0, 2))
    got = sht_tc.map2alm_tc(maps, spin, nside, lmax, 0).cpu().numpy()
    err = _rel(_sampled(got, lmax, orders), want)
    print(f"Nside 4096 spin {spin} tensor-core alm error vs oracle (of scale): {err:.2e}")
    assert err < 5e-5
