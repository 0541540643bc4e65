"""E/B purification on the GPU against the oracle.

The oracle restates the reference's purified alms (gmaster/field.py:433-499) on its FP64
transforms and the eight quadrature coupling blocks (gmaster/workspaces.py:927-1061) in
numpy; the restatement is pinned on the CPU (its standard blocks equal the 3j blocks, its
Wigner rows equal the oracle's own rows up to the transposition symmetry, and on the full
sky its purified blocks equal the standard ones).  pymaster is absent, so agreement with
NaMaster's purification itself is unpinned here.
"""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle
from gmaster_b200 import pure

pytestmark = pytest.mark.gpu


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


def _mask(nside, seed=1):
    rng = np.random.default_rng(seed)
    vec = oracle.pix2vec(nside)
    m = (vec[:, 2] < 0.4).astype(float)
    c = rng.normal(size=(3, 3))
    c /= np.linalg.norm(c, axis=1)[:, None]
    for cc in c:
        m[vec @ cc > np.cos(np.radians(15.0))] = 0.0
    return np.asarray(nmt.mask_apodization(m, 10.0 if nside <= 16 else 5.0, apotype="C2"))


@pytest.mark.parametrize("n", [23, 95, 1001])
def test_gl_nodes_match_oracle(cuda, n):
    x, w = pure.gl_nodes(n, torch.device("cuda"))
    xo, wo = oracle.gauss_legendre(n)
    order = np.argsort(xo)
    xo, wo = xo[order], wo[order] * (2.0 / wo.sum())
    np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=0, atol=1e-14)
    np.testing.assert_allclose(w.cpu().numpy(), wo, rtol=1e-12, atol=0)


def test_wigner_rows_and_correlations_match_oracle(cuda):
    lmax = 60
    xo, _ = oracle.gauss_legendre(121)
    x = torch.from_numpy(np.sort(xo)).cuda()
    beta = np.arccos(np.sort(xo))
    rng = np.random.default_rng(3)
    for m, n in ((0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2), (2, 2), (0, -2), (-2, -2)):
        got = pure.wigner_table(x, lmax, m, n).cpu().numpy()
        want = oracle.wigner_d_table(beta, m, n, lmax).T
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-13)
        vec = rng.normal(size=(2, lmax + 1))
        corr = pure.wigner_corr(x, lmax, m, n, torch.from_numpy(vec).cuda()).cpu().numpy()
        assert _rel(corr, vec @ want) < 1e-12


@pytest.mark.parametrize("nside", [8, 16])
def test_pure_coupling_blocks_match_oracle(cuda, nside):
    lmax = 3 * nside - 1
    m = _mask(nside)
    am = oracle.map2alm(m[None], 0, nside, lmax, 3)
    window = oracle.pcl(am, am, lmax)[0]
    got = pure.coupling_blocks_pure(torch.from_numpy(window).cuda(), lmax)
    want = oracle.coupling_blocks_pure(window, lmax)
    # against the scale of all blocks: for a smooth mask the purified M- blocks vanish (the
    # E -> pure-B leakage purification removes) and hold only rounding noise
    scale = max(float(np.max(np.abs(w_))) for w_ in want)
    for g, w_ in zip(got, want):
        assert float(np.max(np.abs(g.cpu().numpy() - w_))) < 1e-11 * scale
    assert float(np.max(np.abs(want[5]))) < 1e-12 * scale   # one purified field: M- = 0
    # node chunks small enough to need several passes give the same blocks
    few = pure.coupling_blocks_pure(torch.from_numpy(window).cuda(), lmax,
                                    table_bytes=9 * 8 * (lmax + 1) * 7)
    for g, w_ in zip(few, want):
        assert float(np.max(np.abs(g.cpu().numpy() - w_))) < 1e-11 * scale


@pytest.mark.parametrize("task", [(True, False), (False, True), (True, True)])
@pytest.mark.parametrize("masked_on_input", [False, True])
def test_purified_alms_match_oracle(cuda, task, masked_on_input):
    nside = 16
    lmax = 3 * nside - 1
    m = _mask(nside, 2)
    rng = np.random.default_rng(4)
    qu = rng.normal(size=(2, 12 * nside ** 2))
    maps = qu * m[None] if masked_on_input else qu
    f = nmt.NmtField(m, maps, spin=2, purify_e=task[0], purify_b=task[1], n_iter=2,
                     masked_on_input=masked_on_input, precision="fp64")
    want = oracle.purify_alms(m, np.where(m[None] > 0, qu, qu if not masked_on_input else qu * m[None]),
                              nside, lmax, 2, f.n_iter_mask, task)
    assert _rel(f.get_alms().cpu().numpy(), want) < 1e-10
    if not task[0]:
        plain = oracle.map2alm(qu * m[None], 2, nside, lmax, 2)
        assert _rel(f.get_alms().cpu().numpy()[0], plain[0]) < 1e-10


@pytest.mark.parametrize("pure_flags,spins", [((False, True, False, True), (2, 2)),
                                              ((True, True, False, False), (2, 2)),
                                              ((False, False, False, True), (0, 2)),
                                              ((False, False, True, True), (0, 2))])
def test_purified_workspaces_match_oracle(cuda, pure_flags, spins):
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    m = _mask(nside, 5)
    rng = np.random.default_rng(6)
    pe1, pb1, pe2, pb2 = pure_flags
    f1 = nmt.NmtField(m, rng.normal(size=(1 if spins[0] == 0 else 2, len(m))), spin=spins[0],
                      purify_e=pe1, purify_b=pb1, n_iter=0, precision="fp64")
    f2 = nmt.NmtField(m, rng.normal(size=(2, len(m))), spin=spins[1], purify_e=pe2, purify_b=pb2,
                      n_iter=0, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f1, f2, b)
    am = oracle.map2alm(m[None], 0, nside, lmax, f1.n_iter_mask)
    window = oracle.pcl(am, am, lmax)[0]
    blocks8 = oracle.coupling_blocks_pure(window, lmax)
    ncls = 2 if spins[0] == 0 else 4
    want = oracle.assemble_pure_mcm(blocks8, None, lmax, ncls, pure_flags)
    assert _rel(w.get_coupling_matrix().cpu().numpy(), want) < 1e-10
    cl = rng.normal(size=(ncls, lmax + 1)) ** 2
    got = w.decouple_cell(cl).cpu().numpy()
    ref = oracle.decouple(oracle.binned_mcm(want, lmax, nlb, ncls), cl, lmax, nlb)
    assert _rel(got, ref) < 1e-9


def test_purified_teb_workspace_and_files(cuda, tmp_path):
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    m = _mask(nside, 7)
    rng = np.random.default_rng(8)
    f0 = nmt.NmtField(m, rng.normal(size=(1, len(m))), n_iter=0, precision="fp64")
    f2 = nmt.NmtField(m, rng.normal(size=(2, len(m))), purify_b=True, n_iter=0, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f0, f2, b, is_teb=True)
    am = oracle.map2alm(m[None], 0, nside, lmax, f0.n_iter_mask)
    window = oracle.pcl(am, am, lmax)[0]
    tt = oracle.coupling_tt_closed(window, lmax)
    want = oracle.assemble_pure_mcm(oracle.coupling_blocks_pure(window, lmax), tt, lmax, 7,
                                    (False, False, False, True))
    assert _rel(w.get_coupling_matrix().cpu().numpy(), want) < 1e-10
    path = str(tmp_path / "pure.fits")
    w.write_to(path)
    back = nmt.NmtWorkspace.from_file(path)
    assert back.pure_b2 and not back.pure_e2
    cl = rng.normal(size=(7, lmax + 1)) ** 2
    np.testing.assert_array_equal(back.decouple_cell(cl).cpu().numpy(), w.decouple_cell(cl).cpu().numpy())
    with pytest.raises(ValueError, match="Toeplitz"):
        nmt.NmtWorkspace.from_fields(f2, f2, b, l_toeplitz=20, l_exact=5, dl_band=4)
    with pytest.raises(ValueError, match="spin-2"):
        nmt.NmtField(m, rng.normal(size=(1, len(m))), purify_b=True)
    with pytest.raises(ValueError, match="lmax == lmax_mask"):
        nmt.NmtField(m, rng.normal(size=(2, len(m))), purify_b=True, lmax_mask=lmax - 4)
