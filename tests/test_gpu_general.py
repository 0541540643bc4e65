"""General coupling matrices, MASTER coefficients and the full-MASTER helpers on the GPU.

`get_general_coupling_matrix` is checked against the oracle's restatement of the
reference's quadrature (workspaces.py:683-747, oracle.c orc_coupling_quadrature, whose
spin 0/2 cases equal the 3j closed forms), and `get_master_coefficients` against the
oracle's blocks divided by 2 l' + 1.
"""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle

pytestmark = pytest.mark.gpu


def _window(nside, lmax):
    vec = oracle.pix2vec(nside)
    mask = (vec[:, 2] < 0.45) * (0.6 + 0.4 * vec[:, 0] ** 2)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    return mask, oracle.pcl(am, am, lmax)[0]


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / np.max(np.abs(want)))


@pytest.mark.parametrize("spins", [(0, 2, 0, 2), (2, 2, 2, 2), (1, 1, 1, 1), (0, 1, 0, 1),
                                   (2, 1, 2, 1), (0, 0, 0, 0)])
def test_general_coupling_matrix_matches_oracle(cuda, spins):
    nside = 8
    lmax = 3 * nside - 1
    _, w = _window(nside, lmax)
    s1, s2, n1, n2 = spins
    got = nmt.get_general_coupling_matrix(w, s1, s2, n1, n2, parity="both").cpu().numpy()
    even, odd = oracle.coupling_quadrature(w, lmax, s1, s2, n1, n2, lmax_mask=lmax)
    lo = max(spins)
    for g, o in zip(got, (even, odd)):
        o = o.copy()
        o[:lo, :] = 0
        o[:, :lo] = 0
        if np.max(np.abs(o)) > 0:
            assert np.max(np.abs(g - o)) < 1e-11 * np.max(np.abs(even) + np.abs(odd))
    allp = nmt.get_general_coupling_matrix(w, s1, s2, n1, n2).cpu().numpy()
    np.testing.assert_allclose(allp, got[0] + got[1], rtol=0, atol=1e-14)
    with pytest.raises(ValueError):
        nmt.get_general_coupling_matrix(w, s1, s2, n1, n2, parity="bad")


def test_master_coefficients_match_oracle_blocks(cuda):
    nside = 8
    lmax = 3 * nside - 1
    _, w = _window(nside, lmax)
    cols = (2.0 * np.arange(lmax + 1) + 1.0)[None, :]
    tt = oracle.coupling_tt_closed(w, lmax) / cols
    te = oracle.coupling_blocks(w, lmax, 0, 2)["te"] / cols
    pm = oracle.coupling_blocks(w, lmax, 2, 2)
    c = nmt.get_master_coefficients(w, lmax, 0, 0)
    assert _rel(c["00"].cpu().numpy(), tt) < 1e-11 and c["0s"] is None and c["pp"] is None
    c = nmt.get_master_coefficients(w, lmax, 0, 2, is_teb=True)
    assert _rel(c["00"].cpu().numpy(), tt) < 1e-11
    assert c["0s"].shape == (1, lmax + 1, lmax + 1) and _rel(c["0s"][0].cpu().numpy(), te) < 1e-11
    assert _rel(c["pp"][0].cpu().numpy(), pm["pp"] / cols) < 1e-11
    assert _rel(c["mm"][0].cpu().numpy(), pm["mm"] / cols) < 1e-11
    c = nmt.get_master_coefficients(np.stack([w, 2 * w]), lmax, 2, 2, pure_any=True)
    assert c["pp"].shape == (3, 2, lmax + 1, lmax + 1) and c["pure_any"]
    pure = oracle.coupling_blocks_pure(w, lmax)
    assert _rel(c["pp"][2, 0].cpu().numpy(), pure[6] / cols) < 1e-10
    assert _rel(c["pp"][0, 1].cpu().numpy(), 2 * pure[1] / cols) < 1e-10
    c = nmt.get_master_coefficients(w, lmax, 0, 1)
    gen = oracle.coupling_quadrature(w, lmax, 0, 1, 0, 1, lmax_mask=lmax)
    want = (gen[0] + gen[1]) / cols
    want[:1, :] = 0
    want[:, :1] = 0
    got = c["0s"][0].cpu().numpy()
    got[:1, :] = 0
    got[:, :1] = 0
    assert _rel(got, want) < 1e-10
    with pytest.raises(ValueError):
        nmt.get_master_coefficients(w, lmax, 2, 0, is_teb=True)


def test_compute_full_master_and_biases(cuda):
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    mask, _ = _window(nside, lmax)
    rng = np.random.default_rng(2)
    f = nmt.NmtField(mask, rng.normal(size=(2, len(mask))), spin=2, n_iter=0, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f, f, b)
    noise = rng.random((4, lmax + 1)) * 1e-3
    want = w.decouple_cell(nmt.compute_coupled_cell(f, f) - torch.from_numpy(noise).cuda())
    got = nmt.compute_full_master(f, f, b, cl_noise=noise)
    np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-12, atol=0)
    got_w = nmt.compute_full_master(f, f, workspace=w, cl_noise=noise)
    np.testing.assert_array_equal(got_w.cpu().numpy(), want.cpu().numpy())
    z = nmt.deprojection_bias(f, f, np.zeros((4, lmax + 1)))
    assert float(z.abs().max()) == 0.0 and tuple(z.shape) == (4, lmax + 1)
    z = nmt.uncorr_noise_deprojection_bias(f, np.ones(len(mask)))
    assert tuple(z.shape) == (4, lmax + 1)
    with pytest.raises(SyntaxError):
        nmt.compute_full_master(f, f)
    with pytest.raises(ValueError, match="Noise"):
        nmt.compute_full_master(f, f, b, cl_noise=np.zeros((3, lmax + 1)))
    with pytest.raises(ValueError, match="Guess"):
        nmt.deprojection_bias(f, f, np.zeros((4, lmax)))


def test_update_coupling_matrix_bpws_and_dense_files(cuda, tmp_path):
    """update_coupling_matrix keeps an arbitrary dense matrix (workspaces.py:2023-2040): the
    same matrix reproduces the bandpowers, a perturbed one matches the oracle's binning,
    bandpower windows map theory to bandpowers, and a dense matrix survives a file."""
    nside, nlb = 16, 4
    lmax = 3 * nside - 1
    mask, _ = _window(nside, lmax)
    rng = np.random.default_rng(3)
    f = nmt.NmtField(mask, rng.normal(size=(2, len(mask))), spin=2, n_iter=0, precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    w = nmt.NmtWorkspace.from_fields(f, f, b)
    cl = rng.random((4, lmax + 1))
    ref = w.decouple_cell(cl).cpu().numpy()
    bp = w.bpws
    assert tuple(bp.shape) == (4 * w.nbands, 4 * (lmax + 1))
    theory = w.decouple_cell(w.couple_cell(cl)).cpu().numpy()
    via_w = np.einsum("cbdl,dl->cb", w.get_bandpower_windows().cpu().numpy(), cl)
    np.testing.assert_allclose(via_w, theory, rtol=1e-10, atol=1e-14)
    M = w.get_coupling_matrix().cpu().numpy()
    w.update_coupling_matrix(M)
    np.testing.assert_allclose(w.decouple_cell(cl).cpu().numpy(), ref, rtol=1e-10, atol=0)
    M2 = M + 1e-3 * rng.normal(size=M.shape) * np.abs(M).max()
    w.update_coupling_matrix(M2)
    want = oracle.decouple(oracle.binned_mcm(M2, lmax, nlb, 4), cl, lmax, nlb)
    got = w.decouple_cell(cl).cpu().numpy()
    assert _rel(got, want) < 1e-9
    path = str(tmp_path / "dense.fits")
    w.write_to(path)
    back = nmt.NmtWorkspace.from_file(path)
    np.testing.assert_array_equal(back.get_coupling_matrix().cpu().numpy(), M2)
    np.testing.assert_allclose(back.decouple_cell(cl).cpu().numpy(), got, rtol=1e-12, atol=0)
    with pytest.raises(ValueError, match="inconsistent shape"):
        w.update_coupling_matrix(M2[:-1])


def test_moore_penrose_pinvh(cuda):
    rng = np.random.default_rng(4)
    a = rng.normal(size=(6, 6))
    spd = a @ a.T + 6 * np.eye(6)
    np.testing.assert_allclose(nmt.moore_penrose_pinvh(spd, None).cpu().numpy(), np.linalg.inv(spd),
                               rtol=1e-12, atol=1e-14)
    v = rng.normal(size=(6, 3))
    low = v @ v.T
    got = nmt.moore_penrose_pinvh(low, 1e-10).cpu().numpy()
    np.testing.assert_allclose(got, np.linalg.pinv(low, hermitian=True), rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("spins,is_teb", [((0, 1), False), ((1, 0), False), ((1, 3), False),
                                          ((3, 3), False), ((0, 3), True)])
def test_arbitrary_spin_workspaces_match_oracle(cuda, spins, is_teb):
    """Workspaces of spin-1 and spin-3 fields (the cases of the reference's
    test_workspaces.py:429-458): coupling matrix and bandpowers against the oracle's
    general quadrature and the reference's slot signs."""
    nside, nlb = 8, 2
    lmax = 3 * nside - 1
    rng = np.random.default_rng(17)
    masks = [rng.uniform(0.2, 1, 12 * nside ** 2), rng.uniform(0.2, 1, 12 * nside ** 2)]
    fields = []
    for mask, spin in zip(masks, spins):
        maps = rng.normal(size=(1 if spin == 0 else 2, len(mask)))
        fields.append(nmt.NmtField(mask, maps, spin=spin, lmax=lmax, lmax_mask=lmax, n_iter=0,
                                   n_iter_mask=0, precision="fp64"))
    b = nmt.NmtBin.from_lmax_linear(lmax, nlb)
    w = nmt.NmtWorkspace.from_fields(*fields, b, is_teb=is_teb)
    a1 = oracle.map2alm(masks[0][None], 0, nside, lmax, 0)
    a2 = oracle.map2alm(masks[1][None], 0, nside, lmax, 0)
    window = oracle.pcl(a1, a2, lmax)[0]
    s1, s2 = spins
    te = even = odd = None
    if s1 == 0 or s2 == 0:
        e, o = oracle.coupling_quadrature(window, lmax, s1, s2, s1, s2, lmax_mask=lmax)
        te = e + o
    else:
        even, odd = oracle.coupling_quadrature(window, lmax, s1, s2, s1, s2, lmax_mask=lmax)
    if is_teb:
        even, odd = oracle.coupling_quadrature(window, lmax, s2, s2, s2, s2, lmax_mask=lmax)
    tt = oracle.coupling_tt_closed(window, lmax)
    want = oracle.assemble_general_mcm(te, even, odd, tt, lmax, s1, s2, is_teb)
    assert _rel(w.get_coupling_matrix().cpu().numpy(), want) < 1e-10
    ncls = w.ncls
    cl = rng.random((ncls, lmax + 1))
    ref = oracle.decouple(oracle.binned_mcm(want, lmax, nlb, ncls), cl, lmax, nlb)
    assert _rel(w.decouple_cell(cl).cpu().numpy(), ref) < 1e-9


@pytest.mark.parametrize("spins,is_teb", [((1, 3), False), ((0, 1), False), ((0, 3), True)])
def test_arbitrary_spin_workspaces_with_toeplitz_match_oracle(cuda, spins, is_teb):
    """The Toeplitz branch of the general-spin workspaces (workspaces.py:1832-1843): every
    quadrature block is approximated as (M / (2 l' + 1)) -> Toeplitz -> x (2 l' + 1), and the
    scalar block of a TEB workspace is the Toeplitz TT block; against the oracle's quadrature
    blocks through its restatement of the reference's _apply_toeplitz (golden-pinned)."""
    nside, nlb = 8, 2
    lmax = 3 * nside - 1
    lt, le, db = 14, 4, 3
    rng = np.random.default_rng(19)
    masks = [rng.uniform(0.2, 1, 12 * nside ** 2), rng.uniform(0.2, 1, 12 * nside ** 2)]
    fields = []
    for mask, spin in zip(masks, spins):
        maps = rng.normal(size=(1 if spin == 0 else 2, len(mask)))
        fields.append(nmt.NmtField(mask, maps, spin=spin, lmax=lmax, lmax_mask=lmax, n_iter=0,
                                   n_iter_mask=0, precision="fp64"))
    b = nmt.NmtBin.from_lmax_linear(lmax, nlb)
    w = nmt.NmtWorkspace.from_fields(*fields, b, is_teb=is_teb, l_toeplitz=lt, l_exact=le, dl_band=db)
    a1 = oracle.map2alm(masks[0][None], 0, nside, lmax, 0)
    a2 = oracle.map2alm(masks[1][None], 0, nside, lmax, 0)
    window = oracle.pcl(a1, a2, lmax)[0]
    cols = (2.0 * np.arange(lmax + 1) + 1.0)[None, :]

    def approx(x):
        return None if x is None else oracle.apply_toeplitz(x / cols, lt, le, db) * cols

    s1, s2 = spins
    te = even = odd = None
    if s1 == 0 or s2 == 0:
        e, o = oracle.coupling_quadrature(window, lmax, s1, s2, s1, s2, lmax_mask=lmax)
        te = e + o
    else:
        even, odd = oracle.coupling_quadrature(window, lmax, s1, s2, s1, s2, lmax_mask=lmax)
    if is_teb:
        even, odd = oracle.coupling_quadrature(window, lmax, s2, s2, s2, s2, lmax_mask=lmax)
    te, even, odd = approx(te), approx(even), approx(odd)
    tt = oracle.coupling_tt_toeplitz(window, lmax, lt, le, db)
    want = oracle.assemble_general_mcm(te, even, odd, tt, lmax, s1, s2, is_teb)
    assert _rel(w.get_coupling_matrix().cpu().numpy(), want) < 1e-10
