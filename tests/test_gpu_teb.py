"""Joint TEB workspaces (is_teb=True; workspaces.py:1714-1731, 1856-1903): seven spectra
[TT, TE, TB, EE, EB, BE, BB] coupled by the TT, TE and M+/M- blocks of one mask."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
import oracle
from gmaster_b200 import workspaces as ws

pytestmark = pytest.mark.gpu


def _mask(nside, seed=5):
    from gmaster_b200.utils import pix2vec_ring

    rng = np.random.default_rng(seed)
    vec = pix2vec_ring(nside)
    mask = (vec[:, 2] > np.cos(np.radians(65))).astype(float)
    for c in rng.normal(size=(8, 3)):
        mask[vec @ (c / np.linalg.norm(c)) > np.cos(np.radians(6.0))] = 0
    return mask


def _fields(nside, precision="fp64"):
    mask = _mask(nside)
    rng = np.random.default_rng(9)
    f0 = nmt.NmtField(mask, rng.normal(size=(1, 12 * nside ** 2)), precision=precision)
    f2 = nmt.NmtField(mask, rng.normal(size=(2, 12 * nside ** 2)), precision=precision)
    return mask, f0, f2


def test_teb_matrix_matches_oracle_and_decouples_like_the_separate_workspaces(cuda):
    nside = 16
    lmax = 3 * nside - 1
    mask, f0, f2 = _fields(nside)
    b = nmt.NmtBin.from_nside_linear(nside, 4)
    teb = nmt.NmtWorkspace.from_fields(f0, f2, b, is_teb=True)
    assert teb.ncls == 7
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    wmask = oracle.pcl(am, am, lmax)[0]
    tt = oracle.coupling_tt_closed(wmask, lmax)
    te = oracle.coupling_blocks(wmask, lmax, 0, 2)["te"]
    pol = oracle.coupling_blocks(wmask, lmax, 2, 2)
    n = lmax + 1
    want = np.zeros((n, 7, n, 7))
    want[:, 0, :, 0] = tt
    want[:, 1, :, 1] = want[:, 2, :, 2] = te
    for c in range(4):
        want[:, 3 + c, :, 3 + c] += pol["pp"]
    for c, sg in zip(range(4), (1, -1, -1, 1)):
        want[:, 3 + c, :, 6 - c] += sg * pol["mm"]
    got = teb.get_coupling_matrix().cpu().numpy()
    assert np.max(np.abs(got - want.reshape(7 * n, 7 * n))) / np.max(np.abs(want)) < 1e-10

    cl00 = nmt.compute_coupled_cell(f0, f0)
    cl02 = nmt.compute_coupled_cell(f0, f2)
    cl22 = nmt.compute_coupled_cell(f2, f2)
    got = teb.decouple_cell(torch.cat([cl00, cl02, cl22])).cpu().numpy()
    sep = [nmt.NmtWorkspace.from_fields(a, c, b).decouple_cell(cl).cpu().numpy()
           for (a, c), cl in (((f0, f0), cl00), ((f0, f2), cl02), ((f2, f2), cl22))]
    want = np.concatenate(sep)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10 * np.max(np.abs(want)))
    win = teb.get_bandpower_windows()
    assert tuple(win.shape) == (7, b.get_n_bands(), 7, n)


def test_teb_file_round_trip_and_checks(cuda, tmp_path):
    nside = 8
    _, f0, f2 = _fields(nside)
    b = nmt.NmtBin.from_nside_linear(nside, 4)
    teb = nmt.NmtWorkspace.from_fields(f0, f2, b, is_teb=True)
    path = str(tmp_path / "teb.fits")
    teb.write_to(path)
    r = nmt.NmtWorkspace.from_file(path)
    assert r.is_teb and r.ncls == 7
    assert torch.equal(r.get_coupling_matrix(), teb.get_coupling_matrix())
    cl = torch.cat([nmt.compute_coupled_cell(f0, f0), nmt.compute_coupled_cell(f0, f2),
                    nmt.compute_coupled_cell(f2, f2)])
    assert torch.equal(r.decouple_cell(cl), teb.decouple_cell(cl))
    with pytest.raises(ValueError):
        nmt.NmtWorkspace.from_fields(f2, f0, b, is_teb=True)
    with pytest.raises(ValueError):
        nmt.NmtWorkspace.from_fields(f0, f0, b, is_teb=True)
    assert ws._which(7) == 15
