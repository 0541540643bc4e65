"""Many workspaces of uneven lmax from one persistent coupling launch: the blocks equal
those of one launch per workspace (NmtWorkspace.from_fields, workspaces.py:1760-1912)."""

import numpy as np
import pytest
import torch

import gmaster_b200 as nmt
from gmaster_b200 import workspaces as ws

pytestmark = pytest.mark.gpu


def _mask(nside, seed):
    from gmaster_b200.utils import pix2vec_ring

    rng = np.random.default_rng(seed)
    vec = pix2vec_ring(nside)
    mask = (vec[:, 2] > np.cos(np.radians(rng.uniform(40, 80)))).astype(float)
    centres = rng.normal(size=(10, 3))
    centres /= np.linalg.norm(centres, axis=1)[:, None]
    for c in centres:
        mask[vec @ c > np.cos(np.radians(5.0))] = 0
    return mask


def _fields(nside, seed):
    m = _mask(nside, seed)
    f0 = nmt.NmtField(m, None, spin=0, precision="fp64")
    f2 = nmt.NmtField(m, None, spin=2, precision="fp64")
    f2.alm_mask = f0.get_mask_alms()
    return f0, f2


def test_multi_workspace_blocks_equal_single_launches(cuda):
    nsides = (8, 16, 4, 32, 16)
    pairs, bins = [], []
    for k, nside in enumerate(nsides):
        f0, f2 = _fields(nside, 100 + k)
        b = nmt.NmtBin.from_nside_linear(nside, 4)
        pair = [(f0, f0), (f0, f2), (f2, f2)][k % 3]
        pairs.append(pair)
        bins.append(b)
    many = nmt.workspaces_from_fields(pairs, bins)
    for (f1, f2), b, w in zip(pairs, bins, many):
        one = nmt.NmtWorkspace.from_fields(f1, f2, b)
        slots = {1: [ws._BLOCK_TT], 2: [ws._BLOCK_TE], 4: [ws._BLOCK_PP, ws._BLOCK_MM]}[one.ncls]
        for x in slots:
            assert torch.equal(w.mcm_blocks[x], one.mcm_blocks[x])
        assert torch.equal(w.mcm_binned, one.mcm_binned)
        cl = torch.ones((one.ncls, one.lmax + 1), dtype=torch.float64, device="cuda")
        assert torch.equal(w.decouple_cell(cl), one.decouple_cell(cl))


def test_multi_workspace_with_toeplitz(cuda):
    """Toeplitz workspaces: scalar ones keep their selective launch, polarised ones take
    their exact blocks from the shared launch before the fill."""
    f0, f2 = _fields(16, 7)
    g0, _ = _fields(8, 8)
    b16 = nmt.NmtBin.from_nside_linear(16, 4)
    kw = dict(l_toeplitz=20, l_exact=5, dl_band=2)
    many = nmt.workspaces_from_fields([(f0, f0), (f2, f2), (f0, f2)], b16, **kw)
    for (a, c), w in zip([(f0, f0), (f2, f2), (f0, f2)], many):
        one = nmt.NmtWorkspace.from_fields(a, c, b16, **kw)
        np.testing.assert_allclose(w.get_coupling_matrix().cpu().numpy(),
                                   one.get_coupling_matrix().cpu().numpy(), rtol=1e-14, atol=0)
    with pytest.raises(ValueError):
        nmt.workspaces_from_fields([(f0, f0), (g0, g0)], [b16])
