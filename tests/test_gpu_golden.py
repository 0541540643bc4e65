"""The GPU path against outputs of the reference's own code (tests/golden/, written by
tests/golden/make_golden.py): the quadrature coupling blocks and the FP64 3j kernel's
spin-0 x 2 and M+/M- blocks against _general_coupling_matrix_quadrature, the pseudo-C_ell
kernel against _compute_coupled_cell, and the E/B alms of the spin-s transforms against the
reference's E/B combination (healpix.py:_map2alm_once_impl) of the same spin-s transform."""

import numpy as np
import pytest
import torch

from gmaster_b200 import sht, sht_tc, workspaces

pytestmark = pytest.mark.gpu

GOLD = "tests/golden/"


def _tags():
    return [k[7:] for k in np.load(GOLD + "quadrature.npz").files if k.startswith("blocks_")]


@pytest.mark.parametrize("tag", _tags())
def test_gpu_quadrature_blocks_match_reference(cuda, tag):
    g = np.load(GOLD + "quadrature.npz")
    s1, s2, n1, n2 = (int(v) for v in tag.split("_"))
    lmax, lmax_mask = int(g["lmax"]), int(g["lmax_mask"])
    want = g[f"blocks_{tag}"]
    got = workspaces.general_coupling_matrix(torch.from_numpy(g[f"window_{tag}"]).cuda(), s1, s2, n1, n2,
                                             lmax, lmax_mask).cpu().numpy()
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * scale)


def test_gpu_3j_blocks_match_reference_quadrature(cuda):
    """The FP64 Wigner-3j kernel's TT, TE and M+/M- blocks equal the reference's quadrature
    blocks of _coupling_matrices_spin2 (spin-0 x 2: even + odd; 2 x 2: even, odd) and its
    spin-0 block (s = n = 0)."""
    g = np.load(GOLD + "quadrature.npz")
    lmax = int(g["lmax"])
    for tag, pick in (("0_0_0_0", [(0, None)]), ("0_2_0_2", [(1, None)]), ("2_2_2_2", [(2, 0), (3, 1)])):
        window = torch.from_numpy(g[f"window_{tag}"]).cuda()
        blocks = workspaces.coupling_blocks(window, lmax, 15).cpu().numpy()
        ref = g[f"blocks_{tag}"]
        for block, parity in pick:
            want = ref.sum(axis=0) if parity is None else ref[parity]
            lo = 2 if block in (1, 2, 3) else 0   # rows / columns below the spin are zero
            w = want.copy()
            w[:lo, :] = 0
            w[:, :lo] = 0
            got = blocks[block].copy()
            got[:lo, :] = 0
            got[:, :lo] = 0
            np.testing.assert_allclose(got, w, rtol=0, atol=1e-11 * np.abs(want).max())


@pytest.mark.parametrize("pair", ["11", "21", "22"])
def test_gpu_pseudo_cl_matches_reference(cuda, pair):
    g = np.load(GOLD + "spectra_eb.npz")
    a1, a2 = g[f"alm1_{pair}"], g[f"alm2_{pair}"]
    lmax = int(np.sqrt(2 * a1.shape[1])) - 1
    got = workspaces.pseudo_cl(torch.from_numpy(a1).cuda(), torch.from_numpy(a2).cuda(), lmax).cpu().numpy()
    want = g[f"cl_{pair}"]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * np.abs(want).max())


@pytest.mark.parametrize("spin", [1, 2, 3])
def test_gpu_spin_analysis_eb_matches_reference(cuda, spin):
    """E/B alms of the GPU spin-s analysis (FP64 to 1e-10 of scale, mixed to 2e-5) equal the
    reference's E/B combination of the spin-s transform of the same Q, U maps; for spin 2 the
    batched tensor-core path too (5e-5)."""
    g = np.load(GOLD + "spectra_eb.npz")
    nside, lmax = 4, 11
    qu = torch.from_numpy(g[f"qu_s{spin}"]).cuda()
    want = g[f"eb_s{spin}"]
    scale = np.abs(want).max()
    for precision, tol in (("fp64", 1e-10), ("mixed", 2e-5)):
        got = sht.map2alm_device(qu, spin, nside, lmax, 0, precision).cpu().numpy()
        assert np.max(np.abs(got - want)) <= tol * scale, precision
    if spin == 2:
        got = sht_tc.map2alm_tc(qu, 2, nside, lmax, 0).cpu().numpy()
        assert np.max(np.abs(got - want)) <= 5e-5 * scale
