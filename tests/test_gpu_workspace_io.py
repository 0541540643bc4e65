"""Workspace files (workspaces.py:2162-2255): a workspace written with write_to and read
back with from_file has the same coupling matrix, beams, binning and bandpowers."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt

pytestmark = pytest.mark.gpu


def _mask(nside, seed=2):
    from gmaster_b200.utils import pix2vec_ring

    rng = np.random.default_rng(seed)
    vec = pix2vec_ring(nside)
    mask = (vec[:, 2] > np.cos(np.radians(60))).astype(float)
    for c in rng.normal(size=(10, 3)):
        mask[vec @ (c / np.linalg.norm(c)) > np.cos(np.radians(5.0))] = 0
    return mask


@pytest.mark.parametrize("kw", [{}, {"l_toeplitz": 20, "l_exact": 5, "dl_band": 2}])
def test_workspace_file_round_trip(cuda, tmp_path, kw):
    nside = 16
    mask = _mask(nside)
    rng = np.random.default_rng(4)
    f0 = nmt.NmtField(mask, rng.normal(size=(1, 12 * nside ** 2)), precision="fp64",
                      beam=np.exp(-np.arange(3 * nside) / 30.0))
    f2 = nmt.NmtField(mask, rng.normal(size=(2, 12 * nside ** 2)), precision="fp64")
    b = nmt.NmtBin.from_nside_linear(nside, 4)
    for a, c in ((f0, f0), (f0, f2), (f2, f2)):
        w = nmt.NmtWorkspace.from_fields(a, c, b, **kw)
        path = tmp_path / "w.fits"
        w.write_to(str(path))
        r = nmt.NmtWorkspace.from_file(str(path))
        assert (r.lmax, r.ncls, r.spin1, r.spin2, r.l_toeplitz) == (w.lmax, w.ncls, w.spin1, w.spin2,
                                                                     w.l_toeplitz)
        assert torch.equal(r.get_coupling_matrix(), w.get_coupling_matrix())
        assert torch.equal(r.beam1, w.beam1) and torch.equal(r.beam2, w.beam2)
        assert torch.equal(r.mcm_binned, w.mcm_binned)
        cl = nmt.compute_coupled_cell(a, c)
        assert torch.equal(r.decouple_cell(cl), w.decouple_cell(cl))


def test_fkp_normalization_survives(cuda, tmp_path):
    nside = 8
    mask = _mask(nside, seed=3)
    f0 = nmt.NmtField(mask, None, spin=0, precision="fp64")
    w = nmt.NmtWorkspace.from_fields(f0, f0, nmt.NmtBin.from_nside_linear(nside, 4),
                                     normalization="FKP")
    w.write_to(str(tmp_path / "f.fits"))
    r = nmt.NmtWorkspace.from_file(str(tmp_path / "f.fits"))
    assert r.normalization == "FKP" and r.wawb == w.wawb
    assert torch.equal(r.mcm_binned, w.mcm_binned)
