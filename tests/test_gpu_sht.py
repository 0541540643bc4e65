"""GPU parity of the transform kernels against the FP64 oracle (through the C ABI).

Spins 1..8 run through the polarised kernels with the spin's seeds, shift coefficient and
hemisphere parity; the oracle's spin-s form is the reference's literal one
(healpix.py:800-814), pinned for spin 2 against the golden vectors.

Tolerances: the FP64 path must agree with the oracle to 1e-10 of the result's scale;
the mixed path (FP32 ring stage and contraction, FP64 recurrence) to 2e-5 of scale
per transform (the reference's own bar for its FP32 march is 1e-5 of scale,
tests/test_sht.py:1261-1279).
"""

import numpy as np
import pytest
import torch

import oracle
from gmaster_b200 import sht

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 2e-5}


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


@pytest.mark.parametrize("nside,L", [(4, 12), (8, 24), (16, 47), (16, 71), (32, 96), (2, 9),
                                     (128, 384), (96, 200)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ring_analysis_matches_direct_dft(cuda, nside, L, precision):
    """Every ring's m block is w e^{-i m phi0} sum_p x_p e^{-2 pi i p m / nphi}
    (test_sht.py:463-491), including L > 4 nside where every ring aliases."""
    rng = np.random.default_rng(nside + L)
    npix = 12 * nside ** 2
    maps = rng.normal(size=(2, npix))
    plan = sht.get_plan(nside, L - 1)
    prec = sht._prec(precision)
    spec = sht.ring_analysis(plan, torch.from_numpy(maps).cuda(), prec).cpu().numpy()
    w = 4 * np.pi / npix
    for c in range(2):
        want = w * oracle.ring_analysis(nside, L, maps[c].astype(np.complex128))
        assert _rel(spec[c], want) < TOL[precision]


def _lpf(h):
    p, q = 1, 2
    while q * q <= h:
        while h % q == 0:
            p, h = q, h // q
        q += 1
    return max(p, h)


def test_chirp_z_rings_exist_in_the_parity_cases():
    """Nside 128 and 96 (parity cases above) have polar rings whose half-length 2i has a
    prime factor above 64: the mixed-precision ring stage sends those through the chirp-z
    (Bluestein) path, so the direct-DFT check covers it."""
    assert [i for i in range(1, 128) if _lpf(2 * i) > 64] == [67, 71, 73, 79, 83, 89, 97, 101, 103,
                                                              107, 109, 113, 127]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ring_analysis_mask_on_read_equals_masked_maps(cuda, precision):
    """The mask multiplied in as the maps are read gives bit-identical ring spectra to
    pre-masked maps (one FP64 product, rounded once)."""
    nside, L = 16, 48
    rng = np.random.default_rng(77)
    npix = 12 * nside ** 2
    maps = torch.from_numpy(rng.normal(size=(3, npix))).cuda()
    mask = torch.from_numpy(rng.uniform(size=npix) * (rng.uniform(size=npix) > 0.2)).cuda()
    plan = sht.get_plan(nside, L - 1)
    prec = sht._prec(precision)
    a = sht.ring_analysis(plan, maps, prec, mask=mask)
    b = sht.ring_analysis(plan, maps * mask[None], prec)
    assert torch.equal(a, b)


@pytest.mark.parametrize("nside,lmax", [(4, 11), (8, 23), (16, 47), (8, 40)])
@pytest.mark.parametrize("spin", [0, 1, 2, 3, 8])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_alm2map_matches_oracle(cuda, nside, lmax, spin, precision):
    rng = np.random.default_rng(100 + nside + spin)
    nrows = 1 if spin == 0 else 2
    alm = _rand_alm(lmax, nrows, rng, spin)
    want = oracle.alm2map(alm, spin, nside, lmax)
    got = sht.alm2map_device(torch.from_numpy(alm).cuda(), spin, nside, lmax, precision).cpu().numpy()
    assert _rel(got, want) < TOL[precision]


@pytest.mark.parametrize("nside,lmax", [(4, 11), (8, 23), (16, 47), (8, 40)])
@pytest.mark.parametrize("spin", [0, 1, 2, 3, 8])
@pytest.mark.parametrize("n_iter", [0, 3])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_map2alm_matches_oracle(cuda, nside, lmax, spin, n_iter, precision):
    rng = np.random.default_rng(200 + nside + spin)
    nrows = 1 if spin == 0 else 2
    maps = rng.normal(size=(nrows, 12 * nside ** 2))
    want = oracle.map2alm(maps, spin, nside, lmax, n_iter)
    got = sht.map2alm_device(torch.from_numpy(maps).cuda(), spin, nside, lmax, n_iter,
                             precision).cpu().numpy()
    assert _rel(got, want) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pair_matches_two_transforms(cuda, precision):
    """A field and its mask in one shared latitudinal pass equal two transforms."""
    nside, lmax = 16, 47
    rng = np.random.default_rng(7)
    maps = rng.normal(size=(2, 12 * nside ** 2))
    t = torch.from_numpy(maps).cuda()
    both = sht.map2alm_device(t, 0, nside, lmax, 3, precision).cpu().numpy()
    for c in range(2):
        one = sht.map2alm_device(t[c:c + 1], 0, nside, lmax, 3, precision).cpu().numpy()[0]
        assert _rel(both[c], one) < (1e-13 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("nside", [8, 16])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fold_residual_is_analysis_of_synthesis(cuda, nside, precision):
    """gm_fold_residual(syn, rhs) == pack(ring_analysis(ring_synthesis(syn))) - rhs
    (test_sht.py:1282-1304: the fold is the FFT of the IFFT)."""
    lmax = 3 * nside - 1
    plan = sht.get_plan(nside, lmax)
    prec = sht._prec(precision)
    rng = np.random.default_rng(nside)
    alm = torch.from_numpy(_rand_alm(lmax, 1, rng)).cuda()
    syn = sht.legendre_synthesis(plan, 0, alm, 1, prec)
    maps = sht.ring_synthesis(plan, syn, prec)
    rhs_map = sht.pack_rhs(plan, sht.ring_analysis(plan, torch.from_numpy(
        rng.normal(size=(1, 12 * nside ** 2))).cuda(), prec), prec)
    explicit = sht.pack_rhs(plan, sht.ring_analysis(plan, maps, prec), prec) - rhs_map
    folded = sht.fold_residual(plan, syn, rhs_map, prec)
    assert _rel(folded.cpu().numpy(), explicit.cpu().numpy()) < (1e-12 if precision == "fp64" else 2e-5)


def test_large_lmax_spin0_roundtrip(cuda):
    """Band-limited round trip at lmax = 2 nside with many iterations converges (FP64)."""
    nside, lmax = 32, 64
    rng = np.random.default_rng(11)
    alm = _rand_alm(lmax, 1, rng)
    maps = sht.alm2map_device(torch.from_numpy(alm).cuda(), 0, nside, lmax, "fp64")
    back = sht.map2alm_device(maps, 0, nside, lmax, 12, "fp64").cpu().numpy()
    assert _rel(back, alm) < 1e-8
