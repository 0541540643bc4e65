"""Batched tensor-core transforms over windows of orders (the memory-bounded form used for
Nside 4096 batches and Nside 8192) against the single-window transforms and the FP64
oracle.  Windows of a few orders, not dividing L, exercise the window edges."""

import numpy as np
import pytest
import torch

import oracle
from gmaster_b200 import _lib, sht_tc

pytestmark = pytest.mark.gpu

TOL = 5e-5


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


@pytest.fixture
def carried():
    """The windowed transforms run the carried-state kernels; the single-window reference
    they are compared with bit for bit runs those kernels too."""
    old = sht_tc.USE_CHECKPOINTS
    sht_tc.USE_CHECKPOINTS = False
    yield
    sht_tc.USE_CHECKPOINTS = old


@pytest.mark.parametrize("spin,ncomp", [(0, 3), (2, 4)])
@pytest.mark.parametrize("window", [1, 7, 40])
def test_windowed_analysis_equals_single_window(cuda, carried, spin, ncomp, window):
    """n_iter = 0: the same kernels per order, so only the order of the two hemisphere
    atomics (spin 0) can differ."""
    nside = 16
    lmax = 3 * nside - 1
    rng = np.random.default_rng(7 + window)
    maps = torch.from_numpy(rng.normal(size=(ncomp, 12 * nside ** 2))).cuda()
    mask = torch.from_numpy(rng.uniform(size=12 * nside ** 2)).cuda()
    full = sht_tc.map2alm_tc(maps, spin, nside, lmax, 0, mask=mask, window=None).cpu().numpy()
    win = sht_tc.map2alm_tc(maps, spin, nside, lmax, 0, mask=mask, window=window).cpu().numpy()
    assert _rel(win, full) < 1e-12


@pytest.mark.parametrize("spin,ncomp", [(0, 2), (2, 2)])
def test_windowed_jacobi_matches_oracle(cuda, spin, ncomp):
    """n_iter = 3 with the residual taken in map space matches the oracle and the
    ring-fold refinement of the single-window path."""
    nside = 32
    lmax = 3 * nside - 1
    rng = np.random.default_rng(11 + spin)
    maps = rng.normal(size=(ncomp, 12 * nside ** 2))
    mask = rng.uniform(size=12 * nside ** 2)
    dm, dk = torch.from_numpy(maps).cuda(), torch.from_numpy(mask).cuda()
    win = sht_tc.map2alm_tc(dm, spin, nside, lmax, 3, mask=dk, window=13).cpu().numpy()
    full = sht_tc.map2alm_tc(dm, spin, nside, lmax, 3, mask=dk).cpu().numpy()
    mm = maps * mask[None, :]
    if spin == 0:
        want = np.concatenate([oracle.map2alm(mm[c:c + 1], 0, nside, lmax, 3) for c in range(ncomp)])
    else:
        want = oracle.map2alm(mm, 2, nside, lmax, 3)
    assert _rel(win, want) < TOL
    assert _rel(win, full) < TOL


@pytest.mark.parametrize("spin,nrows", [(0, 3), (2, 4)])
def test_windowed_synthesis_equals_single_window(cuda, carried, spin, nrows):
    """alm2map: the windowed synthesis writes the same values per order (no atomics)."""
    nside = 16
    lmax = 3 * nside - 1
    L = lmax + 1
    rng = np.random.default_rng(3 + spin)
    nelem = L * (L + 1) // 2
    alm = rng.normal(size=(nrows, nelem)) + 1j * rng.normal(size=(nrows, nelem))
    order = np.repeat(np.arange(L), L - np.arange(L))
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    alm[:, order == 0] = alm[:, order == 0].real
    if spin:
        alm[:, ell < 2] = 0
    da = torch.from_numpy(alm).cuda()
    full = sht_tc.alm2map_tc(da, spin, nside, lmax).cpu().numpy()
    for window in (1, 9):
        win = sht_tc.alm2map_tc(da, spin, nside, lmax, window=window).cpu().numpy()
        assert np.array_equal(win, full)


def test_bad_windows_are_rejected(cuda):
    tp = sht_tc.get_tc_plan(8, 23)
    p = tp.plan
    img = torch.empty(tp.img_bytes_per_order * 4, dtype=torch.uint8, device="cuda")
    alm = torch.zeros((p.nelem, 2), dtype=torch.float64, device="cuda")
    for m0, m1 in ((5, 5), (-1, 3), (20, 25)):
        with pytest.raises(_lib.GMError):
            _lib.call("gm_tc_analysis_window", p.nside, p.lmax, 0, 0, 1, _lib.ptr(p.geom),
                      _lib.ptr(p.seeds), _lib.ptr(tp.coef[0]), _lib.ptr(img), _lib.ptr(alm), 1.0,
                      _lib.ptr(tp.scratch), tp.nctas, m0, m1, _lib.ptr(tp.err),
                      _lib.stream_handle(p.device))
