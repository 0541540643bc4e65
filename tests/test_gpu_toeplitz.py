"""Toeplitz approximation of the coupling matrix (workspaces.py:521-590, 1141-1194) on
the GPU against the oracle, which is pinned to the reference's _apply_toeplitz."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle
from gmaster_b200 import workspaces as ws

pytestmark = pytest.mark.gpu


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def test_toeplitz_fill_matches_reference_golden(cuda):
    g = np.load("tests/golden/toeplitz.npz")
    k = 0
    while f"case_{k}" in g:
        lmax, lt, le, db = (int(v) for v in g[f"case_{k}"])
        cols = 2.0 * np.arange(lmax + 1) + 1.0
        S = torch.from_numpy(g[f"S_{k}"]).cuda()
        got = ws.toeplitz_fill(S, lmax, lt, le, db).cpu().numpy()
        np.testing.assert_allclose(got, g[f"out_{k}"] * cols[None, :], rtol=1e-13, atol=1e-16)
        k += 1
    S = torch.from_numpy(g["random_S"]).cuda()
    cols = 2.0 * np.arange(20) + 1.0
    got = ws.toeplitz_fill(S, 19, 9, 2, 3).cpu().numpy()
    np.testing.assert_allclose(got, g["random_out"] * cols[None, :], rtol=1e-13, atol=1e-16)


@pytest.mark.parametrize("lmax,lt,le,db", [(31, 16, 4, 3), (95, 40, 8, 4), (191, 100, 20, 6)])
def test_selective_tt_toeplitz_matches_oracle(cuda, lmax, lt, le, db):
    """Only the pairs the fill reads are computed by the 3j recursion; the result equals
    the fill applied to the full exact closed-form matrix."""
    window = np.random.default_rng(lmax).uniform(size=2 * lmax + 1) * np.exp(-np.arange(2 * lmax + 1) / 40)
    got = ws.coupling_tt_toeplitz(torch.from_numpy(window).cuda(), lmax, lt, le, db).cpu().numpy()
    want = oracle.coupling_tt_toeplitz(window, lmax, lt, le, db)
    assert _rel(got, want) < 1e-12


def _mask(nside, seed=2):
    from gmaster_b200.utils import pix2vec_ring

    rng = np.random.default_rng(seed)
    vec = pix2vec_ring(nside)
    mask = (vec[:, 2] > np.cos(np.radians(60))).astype(float)
    centres = rng.normal(size=(20, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(4.0))] = 0
    return mask


def test_workspace_with_toeplitz_matches_oracle(cuda):
    nside, nlb = 32, 4
    lmax = 3 * nside - 1
    lt, le, db = 40, 8, 4
    mask = _mask(nside)
    rng = np.random.default_rng(3)
    m = rng.normal(size=(1, 12 * nside ** 2))
    f = nmt.NmtField(mask, m, n_iter=3, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f, f, b, l_toeplitz=lt, l_exact=le, dl_band=db)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    wmask = oracle.pcl(am, am, lmax)[0]
    mcm = oracle.coupling_tt_toeplitz(wmask, lmax, lt, le, db)
    assert _rel(w.get_coupling_matrix().cpu().numpy(), mcm) < 1e-10
    cl = w.decouple_cell(nmt.compute_coupled_cell(f, f)).cpu().numpy()
    alm = oracle.map2alm(m * mask, 0, nside, lmax, 3)
    want = oracle.decouple(oracle.binned_mcm(mcm, lmax, nlb, 1), oracle.pcl(alm, alm, lmax), lmax, nlb)
    assert _rel(cl, want) < 1e-9


def test_polarised_workspace_toeplitz_blocks(cuda):
    """Polarised blocks are computed exactly and then passed through the same fill
    (workspaces.py:1833-1844)."""
    nside = 16
    lmax = 3 * nside - 1
    lt, le, db = 20, 5, 2
    mask = _mask(nside, seed=4)
    f2 = nmt.NmtField(mask, None, spin=2, precision="fp64")
    f0 = nmt.NmtField(mask, None, spin=0, precision="fp64")
    f2.alm_mask = f0.get_mask_alms()
    b = nmt.NmtBin.from_nside_linear(nside, 4)
    w22 = nmt.NmtWorkspace.from_fields(f2, f2, b, l_toeplitz=lt, l_exact=le, dl_band=db)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    wmask = oracle.pcl(am, am, lmax)[0]
    pol = oracle.coupling_blocks(wmask, lmax, 2, 2)
    cols = 2.0 * np.arange(lmax + 1) + 1.0
    for slot, name in ((ws._BLOCK_PP, "pp"), (ws._BLOCK_MM, "mm")):
        want = oracle.apply_toeplitz(pol[name] / cols[None, :], lt, le, db) * cols[None, :]
        assert _rel(w22.mcm_blocks[slot].cpu().numpy(), want) < 1e-10


def test_toeplitz_bad_parameters_raise(cuda):
    mask = _mask(8)
    f = nmt.NmtField(mask, None, spin=0, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(8, 4)
    with pytest.raises(ValueError):
        nmt.NmtWorkspace.from_fields(f, f, b, l_toeplitz=10, l_exact=12, dl_band=2)
    with pytest.raises(ValueError):
        nmt.NmtWorkspace.from_fields(f, f, b, l_toeplitz=30, l_exact=3, dl_band=2)
