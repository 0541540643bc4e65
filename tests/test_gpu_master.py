"""GPU parity of pseudo-C_ell, coupling, binning and decoupling against the FP64 oracle."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle
from gmaster_b200 import workspaces as ws

pytestmark = pytest.mark.gpu


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def test_pseudo_cl_matches_oracle(cuda):
    lmax = 40
    L = lmax + 1
    nelem = L * (L + 1) // 2
    rng = np.random.default_rng(3)
    a = rng.normal(size=(2, nelem)) + 1j * rng.normal(size=(2, nelem))
    b = rng.normal(size=(2, nelem)) + 1j * rng.normal(size=(2, nelem))
    got = ws.pseudo_cl(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), lmax).cpu().numpy()
    assert _rel(got, oracle.pcl(a, b, lmax)) < 1e-13


@pytest.mark.parametrize("lmax", [15, 16, 17, 31, 40])
def test_tt_coupling_matches_golden_closed_form(cuda, lmax):
    """TT block vs the reference's own threej closed form (tests/golden/coupling_tt.npz,
    generated from tests/test_workspaces.py:_shrinking_offset_tt), atol 2e-14 as there."""
    g = np.load("tests/golden/coupling_tt.npz")
    window = g[f"window_{lmax}"]
    blocks = ws.coupling_blocks(torch.from_numpy(window).cuda(), lmax, 1).cpu().numpy()
    np.testing.assert_allclose(blocks[0], g[f"tt_{lmax}"], atol=2e-14, rtol=0)


@pytest.mark.parametrize("lmax", [20, 63, 191])
def test_polarised_coupling_matches_quadrature(cuda, lmax):
    """TE / M+ / M- blocks from the 3j recursion vs the oracle's Gauss-Legendre
    quadrature of Wigner-d products (workspaces.py:682-924); the reference pins its
    quadrature against the recurrence at 1e-10 (test_workspaces.py:270-282)."""
    rng = np.random.default_rng(lmax)
    window = rng.uniform(size=2 * lmax + 1) * np.exp(-np.arange(2 * lmax + 1) / 30)
    blocks = ws.coupling_blocks(torch.from_numpy(window).cuda(), lmax, 15).cpu().numpy()
    tt = oracle.coupling_tt_closed(window, lmax)
    te = oracle.coupling_blocks(window, lmax, 0, 2)["te"]
    pol = oracle.coupling_blocks(window, lmax, 2, 2)
    assert _rel(blocks[0], tt) < 1e-12
    assert _rel(blocks[1], te) < 1e-10
    assert _rel(blocks[2], pol["pp"]) < 1e-10
    assert _rel(blocks[3], pol["mm"]) < 1e-10


def _config1_inputs(nside, lmax, seed=1):
    """Config-1 style inputs: Gaussian map from C_l = 1e3/(l+10)^2 and a cap mask with holes."""
    rng = np.random.default_rng(seed)
    L = lmax + 1
    ell = np.arange(L)
    cl = 1e3 / (ell + 10.0) ** 2
    cl[:2] = 0
    from gmaster_b200.utils import gaussian_alm, pix2vec_ring

    alm = gaussian_alm(cl, lmax, rng)
    m = oracle.alm2map(alm, 0, nside, lmax)[0]
    vec = pix2vec_ring(nside)
    mask = (vec[:, 2] > np.cos(np.radians(60))).astype(float)
    centres = rng.normal(size=(20, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(4.0))] = 0
    return m, mask


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-4)])
def test_full_estimator_spin0_matches_oracle(cuda, precision, tol):
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    m, mask = _config1_inputs(nside, lmax)
    f = nmt.NmtField(mask, m[None], n_iter=3, precision=precision)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f, f, b)
    cl = w.decouple_cell(nmt.compute_coupled_cell(f, f)).cpu().numpy()
    # oracle
    alm = oracle.map2alm(m[None] * mask, 0, nside, lmax, 3)
    alm_mask = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    pcl = oracle.pcl(alm, alm, lmax)
    wmask = oracle.pcl(alm_mask, alm_mask, lmax)[0]
    mcm = oracle.coupling_tt_closed(wmask, lmax)
    mb = oracle.binned_mcm(mcm, lmax, nlb, 1)
    want = oracle.decouple(mb, pcl, lmax, nlb)
    np.testing.assert_allclose(w.get_coupling_matrix().cpu().numpy(), mcm, rtol=0,
                               atol=tol * np.abs(mcm).max())
    assert _rel(cl, want) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_config1_estimator_matches_oracle(cuda, precision, tol):
    """The Nside 64 parity configuration: map from C_l = 1e3/(l+10)^2 (seed 1), cap mask
    theta < 60 deg with 20 holes of 1 deg (seed 2), C1-apodised at 2 deg, n_iter = 3,
    bands of 16; coupling matrix and bandpowers against the FP64 oracle."""
    from gmaster_b200.utils import gaussian_alm, mask_apodization, pix2vec_ring

    nside, nlb = 64, 16
    lmax = 3 * nside - 1
    ell = np.arange(lmax + 1)
    cl = 1e3 / (ell + 10.0) ** 2
    cl[:2] = 0
    m = oracle.alm2map(gaussian_alm(cl, lmax, np.random.default_rng(1)), 0, nside, lmax)[0]
    vec = pix2vec_ring(nside)
    rng = np.random.default_rng(2)
    mask = (vec[:, 2] > np.cos(np.radians(60))).astype(float)
    centres = rng.normal(size=(20, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(1.0))] = 0
    mask = np.asarray(mask_apodization(mask, 2.0, apotype="C1"))
    f = nmt.NmtField(mask, m[None], n_iter=3, precision=precision)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f, f, b)
    got = w.decouple_cell(nmt.compute_coupled_cell(f, f)).cpu().numpy()
    alm = oracle.map2alm(m[None] * mask, 0, nside, lmax, 3)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    mcm = oracle.coupling_tt_closed(oracle.pcl(am, am, lmax)[0], lmax)
    want = oracle.decouple(oracle.binned_mcm(mcm, lmax, nlb, 1), oracle.pcl(alm, alm, lmax), lmax, nlb)
    assert _rel(w.get_coupling_matrix().cpu().numpy(), mcm) < tol
    assert _rel(got, want) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-4)])
def test_full_estimator_spin2_matches_oracle(cuda, precision, tol):
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    rng = np.random.default_rng(5)
    qu = rng.normal(size=(2, 12 * nside ** 2))
    _, mask = _config1_inputs(nside, lmax, seed=2)
    f0 = nmt.NmtField(mask, qu[:1], n_iter=3, precision=precision)
    f2 = nmt.NmtField(mask, qu, n_iter=3, precision=precision)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w22 = nmt.NmtWorkspace.from_fields(f2, f2, b)
    w02 = nmt.NmtWorkspace.from_fields(f0, f2, b)
    cl22 = w22.decouple_cell(nmt.compute_coupled_cell(f2, f2)).cpu().numpy()
    cl02 = w02.decouple_cell(nmt.compute_coupled_cell(f0, f2)).cpu().numpy()
    eb = oracle.map2alm(qu * mask, 2, nside, lmax, 3)
    t = oracle.map2alm(qu[:1] * mask, 0, nside, lmax, 3)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    wmask = oracle.pcl(am, am, lmax)[0]
    pol = oracle.coupling_blocks(wmask, lmax, 2, 2)
    te = oracle.coupling_blocks(wmask, lmax, 0, 2)
    m22 = oracle.assemble_mcm(pol, lmax, 2, 2)
    m02 = oracle.assemble_mcm(te, lmax, 0, 2)
    want22 = oracle.decouple(oracle.binned_mcm(m22, lmax, nlb, 4), oracle.pcl(eb, eb, lmax), lmax, nlb)
    want02 = oracle.decouple(oracle.binned_mcm(m02, lmax, nlb, 2), oracle.pcl(t, eb, lmax), lmax, nlb)
    np.testing.assert_allclose(w22.get_coupling_matrix().cpu().numpy(), m22, rtol=0,
                               atol=tol * np.abs(m22).max())
    assert _rel(cl22, want22) < tol
    assert _rel(cl02, want02) < tol


def test_lu_solve_matches_numpy(cuda):
    rng = np.random.default_rng(9)
    n = 300
    a = rng.normal(size=(n, n)) + n * np.eye(n)
    b = rng.normal(size=(n, 3))
    lu = ws.LUFactor(torch.from_numpy(a).cuda())
    x = lu.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-12)


def test_bad_shapes_raise_status(cuda):
    from gmaster_b200 import _lib

    with pytest.raises(_lib.GMError) as err:
        _lib.call("gm_pseudo_cl", -1, 1, None, 1, None, None, None)
    assert err.value.status == 1
    with pytest.raises(_lib.GMError) as err:
        _lib.call("gm_pseudo_cl", 10, 1, None, 1, None, None, None)
    assert err.value.status == 2
