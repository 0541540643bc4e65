"""Monte-Carlo batch API: batched fields, spectra and decoupling against the per-field
API and against the FP64 oracle."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle

pytestmark = pytest.mark.gpu


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


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


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-4)])
def test_batched_estimator_matches_oracle(cuda, precision, tol):
    """TQU simulations through fields_from_maps / compute_coupled_cells / decouple_cells,
    each simulation checked against the oracle's estimator (shared workspaces)."""
    nside, nlb, nsims = 16, 4, 3
    lmax = 3 * nside - 1
    rng = np.random.default_rng(11)
    t = rng.normal(size=(nsims, 12 * nside ** 2))
    qu = rng.normal(size=(nsims, 2, 12 * nside ** 2))
    mask = _mask(nside)
    ft = nmt.fields_from_maps(mask, t, n_iter=3, precision=precision)
    fp = nmt.fields_from_maps(mask, qu, n_iter=3, precision=precision)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    f0 = nmt.NmtField(mask, None, spin=0, precision=precision)
    f2 = nmt.NmtField(mask, None, spin=2, precision=precision)
    f2.alm_mask = f0.get_mask_alms()
    w00 = nmt.NmtWorkspace.from_fields(f0, f0, b)
    w02 = nmt.NmtWorkspace.from_fields(f0, f2, b)
    w22 = nmt.NmtWorkspace.from_fields(f2, f2, b)
    bp00 = nmt.decouple_cells(w00, nmt.compute_coupled_cells(ft, ft))
    bp02 = nmt.decouple_cells(w02, nmt.compute_coupled_cells(ft, fp))
    bp22 = nmt.decouple_cells(w22, nmt.compute_coupled_cells(fp, fp))

    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    wmask = oracle.pcl(am, am, lmax)[0]
    m00 = oracle.binned_mcm(oracle.coupling_tt_closed(wmask, lmax), lmax, nlb, 1)
    m02 = oracle.binned_mcm(oracle.assemble_mcm(oracle.coupling_blocks(wmask, lmax, 0, 2), lmax, 0, 2),
                            lmax, nlb, 2)
    m22 = oracle.binned_mcm(oracle.assemble_mcm(oracle.coupling_blocks(wmask, lmax, 2, 2), lmax, 2, 2),
                            lmax, nlb, 4)
    for i in range(nsims):
        at = oracle.map2alm(t[i:i + 1] * mask, 0, nside, lmax, 3)
        eb = oracle.map2alm(qu[i] * mask, 2, nside, lmax, 3)
        assert _rel(bp00[i].cpu().numpy(), oracle.decouple(m00, oracle.pcl(at, at, lmax), lmax, nlb)) < tol
        assert _rel(bp02[i].cpu().numpy(), oracle.decouple(m02, oracle.pcl(at, eb, lmax), lmax, nlb)) < tol
        assert _rel(bp22[i].cpu().numpy(), oracle.decouple(m22, oracle.pcl(eb, eb, lmax), lmax, nlb)) < tol


def test_batched_fields_match_single_fields(cuda):
    """Batched mixed-precision alms agree with one-at-a-time fields, over more simulations
    than one tensor-core launch holds (33 > 32)."""
    nside, nsims = 8, 33
    lmax = 3 * nside - 1
    rng = np.random.default_rng(12)
    t = torch.from_numpy(rng.normal(size=(nsims, 12 * nside ** 2))).cuda()
    mask = torch.from_numpy(_mask(nside, seed=3)).cuda()
    fb = nmt.fields_from_maps(mask, t, n_iter=2, precision="mixed")
    for i in (0, 31, 32):
        f = nmt.NmtField(mask, t[i:i + 1], n_iter=2, precision="fp64", lite=True)
        assert _rel(fb[i].get_alms().cpu().numpy(), f.get_alms().cpu().numpy()) < 5e-5


def test_decouple_cells_equals_decouple_cell(cuda):
    nside, nlb = 16, 4
    mask = _mask(nside, seed=4)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    f0 = nmt.NmtField(mask, None, spin=0, precision="fp64")
    w = nmt.NmtWorkspace.from_fields(f0, f0, b)
    rng = np.random.default_rng(13)
    cls = [torch.from_numpy(rng.normal(size=(1, 3 * nside))).cuda() for _ in range(5)]
    bias = torch.from_numpy(rng.normal(size=(1, 3 * nside))).cuda()
    many = nmt.decouple_cells(w, cls, cl_bias=bias)
    for c, got in zip(cls, many):
        want = w.decouple_cell(c, cl_bias=bias)
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-12, atol=1e-14)


def test_batch_shape_errors(cuda):
    mask = _mask(8)
    with pytest.raises(ValueError):
        nmt.fields_from_maps(mask, np.zeros((2, 3, 12 * 64)))
    with pytest.raises(ValueError):
        nmt.fields_from_maps(mask, np.zeros((2, 12 * 64 + 1)))
    with pytest.raises(ValueError):
        nmt.fields_from_maps(mask, np.zeros((2, 2, 12 * 64)), spin=0)


def test_mc_bandpowers_equals_step_by_step_api(cuda):
    """mc_bandpowers on device maps and on pinned host maps (copied on a side stream)
    gives the results of fields_from_maps / compute_coupled_cells / decouple_cells (to the
    last bits: the pseudo-C_ell sums order chunks with atomics)."""
    nside, nlb, nsims = 16, 4, 3
    rng = np.random.default_rng(21)
    t = torch.from_numpy(rng.normal(size=(nsims, 12 * nside ** 2)))
    qu = torch.from_numpy(rng.normal(size=(nsims, 2, 12 * nside ** 2)))
    mask = _mask(nside, seed=5)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    f0 = nmt.NmtField(mask, None, spin=0, precision="mixed")
    f2 = nmt.NmtField(mask, None, spin=2, precision="mixed")
    f2.alm_mask = f0.get_mask_alms()
    w00 = nmt.NmtWorkspace.from_fields(f0, f0, b)
    w02 = nmt.NmtWorkspace.from_fields(f0, f2, b)
    w22 = nmt.NmtWorkspace.from_fields(f2, f2, b)
    ft = nmt.fields_from_maps(mask, t.cuda(), n_iter=3, precision="mixed")
    fp = nmt.fields_from_maps(mask, qu.cuda(), n_iter=3, precision="mixed")
    want = (nmt.decouple_cells(w00, nmt.compute_coupled_cells(ft, ft)),
            nmt.decouple_cells(w02, nmt.compute_coupled_cells(ft, fp)),
            nmt.decouple_cells(w22, nmt.compute_coupled_cells(fp, fp)))
    for src in ((t.cuda(), qu.cuda()), (t.pin_memory(), qu.pin_memory())):
        got = nmt.mc_bandpowers(mask, src[0], src[1], w00, w02, w22, n_iter=3, precision="mixed")
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            for gi, wi in zip(g, w):
                np.testing.assert_allclose(gi.cpu().numpy(), wi.cpu().numpy(), rtol=1e-12,
                                           atol=1e-12 * float(wi.abs().max()))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_simulation_graph_matches_eager_pipeline(cuda, precision):
    """The graph-captured per-simulation estimator gives each simulation's
    decouple_cell(compute_coupled_cell(...)) bandpowers (pseudo-C_ell sums order chunks
    with atomics, so to the last bits), over several replays with new maps."""
    nside, nlb = 16, 4
    mask = _mask(nside, seed=6)
    b = nmt.NmtBin.from_nside_linear(nside, nlb)
    f0 = nmt.NmtField(mask, None, spin=0, precision=precision)
    f2 = nmt.NmtField(mask, None, spin=2, precision=precision)
    f2.alm_mask = f0.get_mask_alms()
    ws = [nmt.NmtWorkspace.from_fields(a, c, b) for a, c in ((f0, f0), (f0, f2), (f2, f2))]
    g = nmt.SimulationGraph(mask, *ws, n_iter=3, precision=precision)
    rng = np.random.default_rng(31)
    for _ in range(3):
        t = rng.normal(size=12 * nside ** 2)
        qu = rng.normal(size=(2, 12 * nside ** 2))
        got = g(t, qu)
        ft = nmt.NmtField(mask, t[None], n_iter=3, precision=precision)
        fp = nmt.NmtField(mask, qu, n_iter=3, precision=precision)
        for w, (a, c), gi in zip(ws, ((ft, ft), (ft, fp), (fp, fp)), got):
            want = w.decouple_cell(nmt.compute_coupled_cell(a, c))
            np.testing.assert_allclose(gi.cpu().numpy(), want.cpu().numpy(), rtol=1e-11,
                                       atol=1e-11 * float(want.abs().max()))
