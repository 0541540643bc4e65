"""The oracle's coupling, slot, pseudo-spectrum and E/B steps pinned to outputs of the
reference's own code (tests/golden/quadrature.npz, slots.npz, spectra_eb.npz, written by
tests/golden/make_golden.py from gmaster/workspaces.py and gmaster/_sht/healpix.py).

These close the spin-2 half of the path: the oracle's Gauss-Legendre quadrature blocks
(spin 0 x 2, M+ and M- of 2 x 2, and the general spins), the (block, slot, sign) table of
the coupling matrix, the coupled pseudo-C_ell, and the E/B combinations of the spin-s
analysis and synthesis are each compared with what the reference computes from the same
inputs.  The GPU path is compared with the same fixtures in tests/test_gpu_golden.py."""

import numpy as np
import pytest

import oracle
from gmaster_b200 import workspaces

GOLD = "tests/golden/"


@pytest.fixture(scope="module")
def quad():
    return np.load(GOLD + "quadrature.npz")


def test_gauss_legendre_nodes_are_the_fixture_nodes(quad):
    """The fixture's quadrature ran on the oracle's nodes and weights (ducc0 is absent)."""
    x, w = oracle.gauss_legendre(len(quad["nodes"]))
    np.testing.assert_array_equal(x, quad["nodes"])
    np.testing.assert_array_equal(w, quad["weights"])


@pytest.mark.parametrize("mn", [k[7:] for k in np.load(GOLD + "quadrature.npz").files
                                if k.startswith("wigner_")])
def test_wigner_d_table_matches_reference(quad, mn):
    m, n = (int(v) for v in mn.split("_"))
    beta = np.arccos(quad["nodes"])
    want = quad[f"wigner_{mn}"]
    got = oracle.wigner_d_table(beta, m, n, want.shape[1] - 1)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13)


@pytest.mark.parametrize("tag", [k[7:] for k in np.load(GOLD + "quadrature.npz").files
                                 if k.startswith("blocks_")])
def test_coupling_quadrature_matches_reference(quad, tag):
    """Even/odd general coupling blocks (the spin-0 x 2 block is their sum, M+ / M- of 2 x 2
    are the pair) of _general_coupling_matrix_quadrature, reference vs oracle."""
    s1, s2, n1, n2 = (int(v) for v in tag.split("_"))
    lmax, lmax_mask = int(quad["lmax"]), int(quad["lmax_mask"])
    want = quad[f"blocks_{tag}"]
    even, odd = oracle.coupling_quadrature(quad[f"window_{tag}"], lmax, s1, s2, n1, n2, lmax_mask=lmax_mask)
    scale = np.max(np.abs(want))
    assert scale > 0
    np.testing.assert_allclose(even, want[0], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(odd, want[1], rtol=0, atol=1e-12 * scale)


def _dense_from_table(table, blocks, n, ncls):
    out = np.zeros((n, ncls, n, ncls))
    for b, r, c, sign in table:
        out[:, r, :, c] += sign * blocks[b]
    return out.reshape(n * ncls, n * ncls)


def test_slot_tables_match_reference():
    """The oracle's coupling-matrix assembly equals the reference's (block, slot, sign)
    table for spins 0, 1, 2, 3 and joint TEB workspaces; the product's spin-0/2 table
    (workspaces._slots) equals it entry for entry."""
    g = np.load(GOLD + "slots.npz")
    rng = np.random.default_rng(5)
    n = 6
    index = {0: workspaces._BLOCK_TT, 1: workspaces._BLOCK_TE, 2: workspaces._BLOCK_PP,
             3: workspaces._BLOCK_MM}
    ncases = len([k for k in g.files if k.startswith("case_")])
    for k in range(ncases):
        s1, s2, teb, ncls = (int(v) for v in g[f"case_{k}"])
        table = g[f"table_{k}"]
        tt, te, even, odd = (rng.normal(size=(n, n)) for _ in range(4))
        want = _dense_from_table(table, (tt, te, even, odd), n, ncls)
        got = oracle.assemble_general_mcm(te, even, odd, tt, n - 1, s1, s2, bool(teb))
        np.testing.assert_array_equal(got, want)
        if s1 in (0, 2) and s2 in (0, 2):
            mine = sorted((int(b), int(r), int(c), float(sg)) for b, r, c, sg in workspaces._slots(ncls))
            ref = sorted((index[int(b)], int(r), int(c), float(sg)) for b, r, c, sg in table)
            assert mine == ref, (s1, s2, teb)


@pytest.mark.parametrize("pair", ["11", "21", "22"])
def test_coupled_cell_matches_reference(pair):
    g = np.load(GOLD + "spectra_eb.npz")
    a1, a2 = g[f"alm1_{pair}"], g[f"alm2_{pair}"]
    lmax = int(np.sqrt(2 * a1.shape[1])) - 1
    want = g[f"cl_{pair}"]
    np.testing.assert_allclose(oracle.pcl(a1, a2, lmax), want, rtol=0, atol=1e-13 * np.abs(want).max())


@pytest.mark.parametrize("spin", [1, 2, 3])
def test_eb_combination_matches_reference(spin):
    """E/B of the reference's analysis combination (healpix.py:_map2alm_once_impl) applied to
    the oracle's spin-s transform of Q + iU: the oracle's restatement of the combination and
    its literal spin-s analysis give the same alms; for spin 2 so does the +-2 row form."""
    g = np.load(GOLD + "spectra_eb.npz")
    nside = 4
    lmax = 3 * nside - 1
    qu, plus, want = g[f"qu_s{spin}"], g[f"plus_s{spin}"], g[f"eb_s{spin}"]
    scale = np.abs(want).max()
    np.testing.assert_allclose(oracle.spin_plus(qu, spin, nside, lmax), plus, rtol=0, atol=1e-14 * scale)
    np.testing.assert_allclose(oracle.eb_from_plus(plus, lmax), want, rtol=0, atol=1e-14 * scale)
    got = oracle.map2alm(qu, spin, nside, lmax, 0, general=True)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * scale)
    if spin == 2:
        np.testing.assert_allclose(oracle.map2alm(qu, 2, nside, lmax, 0), want, rtol=0, atol=1e-12 * scale)


@pytest.mark.parametrize("spin", [1, 2, 3])
def test_eb_unpack_matches_reference(spin):
    """Synthesis coefficients from E/B: the oracle's combination equals the reference's
    _unpack_spin (healpix.py:599-611)."""
    g = np.load(GOLD + "spectra_eb.npz")
    lmax = 11
    np.testing.assert_allclose(oracle.plus_from_eb(g[f"ebin_s{spin}"], lmax), g[f"unpack_s{spin}"],
                               rtol=0, atol=1e-15)
