"""Batched tensor-core transforms (tcgen05, bf16x3 products, FP32 accumulation) against
the FP64 oracle.  Tolerance: 5e-5 of the result's scale per transform (the products carry
16 significant bits; the reference's own FP32 march is held to 1e-5 of scale)."""

import numpy as np
import pytest
import torch

import oracle
from gmaster_b200 import sht, sht_tc

pytestmark = pytest.mark.gpu

TOL = 5e-5


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def _rand_alm(lmax, nrows, rng, spin=0):
    L = lmax + 1
    nelem = L * (L + 1) // 2
    alm = rng.normal(size=(nrows, nelem)) + 1j * rng.normal(size=(nrows, nelem))
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    order = np.repeat(np.arange(L), L - np.arange(L))
    alm[:, order == 0] = alm[:, order == 0].real
    if spin:
        alm[:, ell < spin] = 0
    return alm


@pytest.mark.parametrize("nside,nmaps", [(8, 1), (16, 3), (32, 8), (64, 32)])
@pytest.mark.parametrize("n_iter", [0, 3])
def test_tc_map2alm_spin0(cuda, nside, nmaps, n_iter):
    lmax = 3 * nside - 1
    rng = np.random.default_rng(nside + nmaps)
    maps = rng.normal(size=(nmaps, 12 * nside ** 2))
    got = sht_tc.map2alm_tc(torch.from_numpy(maps).cuda(), 0, nside, lmax, n_iter).cpu().numpy()
    for c in range(min(nmaps, 3)):
        want = oracle.map2alm(maps[c:c + 1], 0, nside, lmax, n_iter)[0]
        assert _rel(got[c], want) < TOL
    if nmaps > 3:
        simt = sht.map2alm_device(torch.from_numpy(maps).cuda(), 0, nside, lmax, n_iter, "fp64").cpu().numpy()
        assert _rel(got, simt) < TOL


@pytest.mark.parametrize("nside,nfields", [(8, 1), (16, 2), (32, 4)])
@pytest.mark.parametrize("n_iter", [0, 3])
def test_tc_map2alm_spin2(cuda, nside, nfields, n_iter):
    lmax = 3 * nside - 1
    rng = np.random.default_rng(50 + nside + nfields)
    maps = rng.normal(size=(2 * nfields, 12 * nside ** 2))
    got = sht_tc.map2alm_tc(torch.from_numpy(maps).cuda(), 2, nside, lmax, n_iter).cpu().numpy()
    for f in range(min(nfields, 2)):
        want = oracle.map2alm(maps[2 * f:2 * f + 2], 2, nside, lmax, n_iter)
        assert _rel(got[2 * f:2 * f + 2], want) < TOL


@pytest.mark.parametrize("spin,nside,nrows", [(0, 16, 2), (2, 16, 4), (0, 64, 8)])
def test_tc_alm2map(cuda, spin, nside, nrows):
    lmax = 3 * nside - 1
    rng = np.random.default_rng(7 + spin)
    alm = _rand_alm(lmax, nrows, rng, spin)
    got = sht_tc.alm2map_tc(torch.from_numpy(alm).cuda(), spin, nside, lmax).cpu().numpy()
    step = 1 if spin == 0 else 2
    for r in range(0, min(nrows, 2 * step), step):
        want = oracle.alm2map(alm[r:r + step], spin, nside, lmax)
        assert _rel(got[r:r + step], want) < TOL


def test_tc_two_superblocks_and_groups(cuda):
    """Nside 256 (L = 768 > 512, 512 lanes = 4 groups) exercises the recurrence state
    carried across superblocks in the scratch buffer."""
    nside, lmax = 256, 767
    rng = np.random.default_rng(3)
    maps = rng.normal(size=(4, 12 * nside ** 2))
    t = torch.from_numpy(maps).cuda()
    got = sht_tc.map2alm_tc(t, 0, nside, lmax, 1).cpu().numpy()
    ref = sht.map2alm_device(t, 0, nside, lmax, 1, "fp64").cpu().numpy()
    assert _rel(got, ref) < TOL
    got2 = sht_tc.map2alm_tc(t, 2, nside, lmax, 1).cpu().numpy()
    ref2 = sht.map2alm_device(t, 2, nside, lmax, 1, "fp64").cpu().numpy()
    assert _rel(got2, ref2) < TOL
