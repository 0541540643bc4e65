"""GPU mask apodisation (gm_mask_ring_runs + gm_mask_apodize) against the oracle.

The reference apodises on the host (gmaster/utils.py:61-147): a k-d tree over the masked
pixels' unit vectors for C1 / C2, healpy's query_disc for the zeroing step of Smooth.  The
oracle restates those steps with scipy's k-d tree; the GPU kernel finds the same nearest
masked pixel by walking the HEALPix rings.
"""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle
from gmaster_b200 import _lib, utils

pytestmark = pytest.mark.gpu


def _holes_mask(nside, nholes, hole_deg, seed, cut_z=None, values=False):
    rng = np.random.default_rng(seed)
    vec = oracle.pix2vec(nside)
    mask = np.ones(len(vec)) if cut_z is None else (vec[:, 2] < cut_z).astype(float)
    centres = rng.normal(size=(nholes, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(hole_deg))] = 0.0
    if values:
        mask *= rng.uniform(0.2, 1.0, size=len(mask))
    return mask


@pytest.mark.parametrize("nside,nholes,hole,apo", [(16, 4, 10.0, 15.0), (32, 20, 3.0, 2.0),
                                                   (64, 20, 1.0, 2.0), (128, 50, 0.5, 1.0),
                                                   (256, 100, 0.3, 0.5)])
@pytest.mark.parametrize("apotype", ["C1", "C2"])
def test_c1_c2_match_oracle(cuda, nside, nholes, hole, apo, apotype):
    mask = _holes_mask(nside, nholes, hole, seed=nside, cut_z=0.6)
    got = nmt.mask_apodization(mask, apo, apotype=apotype)
    assert isinstance(got, np.ndarray)
    want = oracle.mask_apodization(mask, apo, apotype)
    # the tapers are continuous at the radius, so a pixel whose distance rounds to the
    # other side of it changes by ~1e-16; distances agree to rounding
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    assert np.count_nonzero((got > 0) & (got < 1)) > 0


def test_non_binary_values_nans_and_tensors(cuda):
    nside = 32
    mask = _holes_mask(nside, 12, 4.0, seed=7, values=True)
    mask[[5, 100, 4000]] = np.nan
    mask[[6, 7000]] = -0.5     # negative values count as masked
    want = oracle.mask_apodization(mask, 6.0, "C1")
    got = nmt.mask_apodization(torch.from_numpy(mask).cuda(), 6.0, apotype="C1")
    assert isinstance(got, torch.Tensor) and got.is_cuda
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0, atol=1e-12)
    assert np.isnan(got.cpu().numpy()[[5, 100, 4000]]).all()


def test_whole_sky_radius_and_single_masked_pixel(cuda):
    """A radius larger than the sphere's diameter (every pixel tapered) and a mask with a
    single masked pixel (rings without masked pixels everywhere else)."""
    nside = 16
    mask = np.ones(12 * nside ** 2)
    mask[1234] = 0.0
    for apo in (179.0, 20.0):
        got = nmt.mask_apodization(mask, apo, apotype="C2")
        np.testing.assert_allclose(got, oracle.mask_apodization(mask, apo, "C2"), rtol=0,
                                   atol=1e-12)


def test_trivial_masks_are_copied(cuda):
    nside = 16
    ones = np.ones(12 * nside ** 2)
    np.testing.assert_array_equal(nmt.mask_apodization(ones, 5.0), ones)
    zeros = np.zeros(12 * nside ** 2)
    np.testing.assert_array_equal(nmt.mask_apodization(zeros, 5.0), zeros)
    mask = _holes_mask(nside, 3, 10.0, seed=1)
    np.testing.assert_array_equal(nmt.mask_apodization(mask, 0.0), mask)


def test_errors(cuda):
    mask = np.ones(12 * 8 ** 2)
    with pytest.raises(ValueError, match="too small"):
        nmt.mask_apodization(mask, 0.01)
    with pytest.raises(ValueError, match="HEALPix"):
        nmt.mask_apodization(np.ones(100), 5.0)
    dev = torch.zeros(12 * 16, dtype=torch.float64, device="cuda")
    i32 = torch.zeros(12 * 16, dtype=torch.int32, device="cuda")
    tab = torch.zeros(5 * 7, dtype=torch.float64, device="cuda")
    st = _lib.stream_handle()
    lib = _lib.load()
    assert lib.gm_mask_apodize(4, _lib.ptr(tab), _lib.ptr(dev), _lib.ptr(i32), _lib.ptr(i32), 1.0,
                               0.5, 3, _lib.ptr(dev), st) == 5
    assert lib.gm_mask_apodize(0, _lib.ptr(tab), _lib.ptr(dev), _lib.ptr(i32), _lib.ptr(i32), 1.0,
                               0.5, 0, _lib.ptr(dev), st) == 1
    assert lib.gm_mask_ring_runs(4, None, _lib.ptr(i32), _lib.ptr(i32), st) == 2


@pytest.mark.parametrize("nside,apo", [(16, 6.0), (32, 4.0)])
def test_smooth_matches_oracle(cuda, nside, apo):
    mask = _holes_mask(nside, 6, 8.0, seed=11, cut_z=0.7)
    old = nmt.get_precision()
    nmt.set_precision("fp64")
    try:
        got = nmt.mask_apodization(mask, apo, apotype="Smooth")
    finally:
        nmt.set_precision(old)
    assert isinstance(got, torch.Tensor)
    want = oracle.mask_apodization(mask, apo, "Smooth")
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0, atol=1e-10)
    assert float(np.abs(want).max()) > 0.1


def test_ring_runs_layout(cuda):
    """prev / next against a direct restatement on the host."""
    nside = 8
    mask = _holes_mask(nside, 3, 15.0, seed=4, cut_z=0.8)
    m = torch.from_numpy(mask).cuda()
    prev = torch.empty(m.numel(), dtype=torch.int32, device="cuda")
    nxt = torch.empty_like(prev)
    _lib.call("gm_mask_ring_runs", nside, _lib.ptr(m), _lib.ptr(prev), _lib.ptr(nxt),
              _lib.stream_handle())
    prev, nxt = prev.cpu().numpy(), nxt.cpu().numpy()
    _, _, nphi, off = oracle.geometry(nside)
    for n, o in zip(nphi, off):
        ring = mask[o:o + n] <= 0
        idx = np.flatnonzero(ring)
        for i in range(n):
            if not len(idx):
                assert prev[o + i] == -1 and nxt[o + i] == -1
                continue
            before = idx[idx <= i]
            after = idx[idx >= i]
            assert prev[o + i] == (before[-1] if len(before) else idx[-1])
            assert nxt[o + i] == (after[0] if len(after) else idx[0])


def test_full_size_nside2048_against_brute_force(cuda):
    """Nside 2048, |b| > 20 deg about a tilted pole plus 2000 holes of 5', C1 at 1 deg (the
    Monte-Carlo configuration's recipe): the taper of 400 sampled pixels, near the cut and
    the holes, against the exact minimum chord over all masked pixels."""
    nside = 2048
    vec = torch.from_numpy(utils.pix2vec_ring(nside)).cuda()
    th, ph = np.radians(30.0), np.radians(45.0)
    pole = torch.tensor([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)],
                        dtype=torch.float64, device="cuda")
    mask = ((vec @ pole).abs() > np.sin(np.radians(20.0))).to(torch.float64)
    rng = np.random.default_rng(4)
    centres = rng.normal(size=(2000, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    cos_hole = np.cos(np.radians(5.0 / 60.0))
    for c in torch.from_numpy(centres).cuda().split(100):
        hit = ((vec @ c.T) > cos_hole).any(dim=1)
        mask[hit] = 0.0
    out = nmt.mask_apodization(mask, 1.0, apotype="C1")
    tapered = torch.nonzero((out > 0) & (out < 1)).flatten()
    assert tapered.numel() > 1000
    pick = tapered[torch.from_numpy(rng.choice(tapered.numel(), 400, replace=False)).cuda()]
    masked_vec = vec[mask <= 0]
    thr = 1 - np.cos(np.radians(1.0))
    for p in pick.tolist():
        d2 = ((masked_vec - vec[p]) ** 2).sum(dim=1).min().item()
        x = np.sqrt(0.5 * d2 / thr)
        want = x - np.sin(2 * np.pi * x) / (2 * np.pi)
        assert abs(out[p].item() - want) < 1e-12
    # pixels the search left untouched are farther than the radius from every masked pixel
    ones = torch.nonzero(out == 1).flatten()
    far = ones[torch.from_numpy(rng.choice(ones.numel(), 50, replace=False)).cuda()]
    for p in far.tolist():
        d2 = ((masked_vec - vec[p]) ** 2).sum(dim=1).min().item()
        assert 0.5 * d2 >= thr * (1 - 1e-12)
