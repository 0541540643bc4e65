"""Checkpointed tensor-core transforms (legendre_ck.cu) against the FP64 oracle.

The checkpoint table (the FP64 recurrence's state every 128 rows, stored in single
precision with a power-of-two shift) is decoded and compared with the oracle's rows; the
transforms built on it are compared with the oracle (Nside <= 64) and with the plain FP64
GPU path (Nside 256: three superblocks, four lane groups, shifted high-order lanes), and
with the carried-state tensor-core kernels they replace.  Tolerance as for the other
tensor-core transforms: 5e-5 of the result's scale."""

import numpy as np
import pytest
import torch

import oracle
from gmaster_b200 import sht, sht_tc

pytestmark = pytest.mark.gpu

TOL = 5e-5


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300))


@pytest.fixture(params=[True, False], ids=["checkpointed", "carried"])
def ck_mode(request):
    old = sht_tc.USE_CHECKPOINTS
    sht_tc.USE_CHECKPOINTS = request.param
    yield request.param
    sht_tc.USE_CHECKPOINTS = old


@pytest.mark.parametrize("spin,sp", [(0, 0), (2, -2), (2, 2)])
def test_ck_table_rows_match_oracle(cuda, spin, sp):
    """Decoded checkpoints (v_{l_s - 1}, v_{l_s}) equal the oracle's FP64 rows at every
    segment start l_s = l0 + 128 k to 1e-6 of the row scale sqrt((2l+1)/4pi)."""
    nside, lmax = 64, 191
    tp = sht_tc.get_tc_plan(nside, lmax)
    ck = sht_tc.ck_tables(tp, spin)
    assert ck is not None
    state, shift = (t.cpu().numpy() for t in ck[sp])
    segoff = tp.ck_segoff[spin].cpu().numpy()
    nl = tp.plan.nlanes
    theta = sht.ring_geometry(nside)[0][:nl]
    checked = 0
    for m in (0, 1, 2, 3, 17, 64, 120, 190):
        l0 = max(m, abs(sp))
        rows = np.stack([oracle.lambda_row(lmax, m, sp, th) for th in theta])   # (lanes, L)
        # the kernel's +2 rows carry the (-1)^s of the E/B combination (even for s = 2) and
        # both variants the sign convention of the seed table: compare up to one sign per order
        for k in range((lmax + 1 - l0 + 127) // 128):
            ls = l0 + 128 * k
            seg = segoff[m] + k
            st = state[seg * nl:(seg + 1) * nl].astype(np.float64)
            sc = np.exp2(-64.0 * shift[seg * nl:(seg + 1) * nl].astype(np.float64))
            vpre = st[:, 0] * sc
            vs = (st[:, 0] + st[:, 1]) * sc
            want_s = rows[:, ls]
            want_pre = rows[:, ls - 1] if ls > l0 else np.zeros(nl)
            big = np.argmax(np.abs(want_s))
            sign = np.sign(vs[big] * want_s[big]) if want_s[big] != 0 else 1.0
            scale = np.sqrt((2 * ls + 1) / (4 * np.pi))
            assert np.max(np.abs(vs - sign * want_s)) <= 1e-6 * scale, (m, k)
            assert np.max(np.abs(vpre - sign * want_pre)) <= 1e-6 * scale, (m, k)
            checked += 1
    assert checked > 8


@pytest.mark.parametrize("nside,nmaps", [(16, 3), (64, 32)])
@pytest.mark.parametrize("n_iter", [0, 3])
def test_ck_map2alm_spin0(cuda, ck_mode, nside, nmaps, n_iter):
    lmax = 3 * nside - 1
    rng = np.random.default_rng(100 + nside + nmaps)
    maps = rng.normal(size=(nmaps, 12 * nside ** 2))
    got = sht_tc.map2alm_tc(torch.from_numpy(maps).cuda(), 0, nside, lmax, n_iter).cpu().numpy()
    for c in range(min(nmaps, 2)):
        want = oracle.map2alm(maps[c:c + 1], 0, nside, lmax, n_iter)[0]
        assert _rel(got[c], want) < TOL


@pytest.mark.parametrize("nside,nfields", [(16, 2), (64, 8)])
@pytest.mark.parametrize("n_iter", [0, 3])
def test_ck_map2alm_spin2(cuda, ck_mode, nside, nfields, n_iter):
    lmax = 3 * nside - 1
    rng = np.random.default_rng(200 + nside + nfields)
    maps = rng.normal(size=(2 * nfields, 12 * nside ** 2))
    got = sht_tc.map2alm_tc(torch.from_numpy(maps).cuda(), 2, nside, lmax, n_iter).cpu().numpy()
    for f in range(min(nfields, 2)):
        want = oracle.map2alm(maps[2 * f:2 * f + 2], 2, nside, lmax, n_iter)
        assert _rel(got[2 * f:2 * f + 2], want) < TOL


@pytest.mark.parametrize("spin,nside,nrows", [(0, 32, 4), (2, 32, 4), (2, 64, 16)])
def test_ck_alm2map(cuda, ck_mode, spin, nside, nrows):
    lmax = 3 * nside - 1
    L = lmax + 1
    rng = np.random.default_rng(300 + spin + nside)
    nelem = L * (L + 1) // 2
    alm = rng.normal(size=(nrows, nelem)) + 1j * rng.normal(size=(nrows, nelem))
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    order = np.repeat(np.arange(L), L - np.arange(L))
    alm[:, order == 0] = alm[:, order == 0].real
    if spin:
        alm[:, ell < 2] = 0
    got = sht_tc.alm2map_tc(torch.from_numpy(alm).cuda(), spin, nside, lmax).cpu().numpy()
    step = 1 if spin == 0 else 2
    for r in range(0, 2 * step, step):
        want = oracle.alm2map(alm[r:r + step], spin, nside, lmax)
        assert _rel(got[r:r + step], want) < TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_ck_matches_fp64_path_nside256(cuda, spin):
    """Three superblocks of rows, four lane groups, high orders whose seeds sit far below
    the single-precision range (shifted checkpoints): the checkpointed transform with one
    refinement against the plain FP64 GPU path, and against the carried-state kernels."""
    nside, lmax = 256, 767
    rng = np.random.default_rng(400 + spin)
    maps = torch.from_numpy(rng.normal(size=(4, 12 * nside ** 2))).cuda()
    ref = sht.map2alm_device(maps, spin, nside, lmax, 1, "fp64").cpu().numpy()
    old = sht_tc.USE_CHECKPOINTS
    try:
        sht_tc.USE_CHECKPOINTS = True
        got = sht_tc.map2alm_tc(maps, spin, nside, lmax, 1).cpu().numpy()
        sht_tc.USE_CHECKPOINTS = False
        carried = sht_tc.map2alm_tc(maps, spin, nside, lmax, 1).cpu().numpy()
    finally:
        sht_tc.USE_CHECKPOINTS = old
    assert _rel(got, ref) < TOL
    assert _rel(got, carried) < TOL


@pytest.mark.parametrize("spin", [0, 2])
def test_tile_skip_is_exact(cuda, spin):
    """Skipping the 64-lane groups whose checkpoint states are all zero (the rows of such a
    segment are exactly zero) leaves the batched transforms bit-identical; at Nside 512 about
    a sixth of the analysis groups are skipped."""
    nside, lmax = 512, 1535
    rng = np.random.default_rng(31 + spin)
    maps = torch.from_numpy(rng.normal(size=(8, 12 * nside ** 2))).cuda()
    old = sht_tc.USE_TILE_SKIP
    try:
        sht_tc.USE_TILE_SKIP = False
        full = sht_tc.map2alm_tc(maps, spin, nside, lmax, 3)
        syn_full = sht_tc.alm2map_tc(full, spin, nside, lmax)
        sht_tc.USE_TILE_SKIP = True
        skip = sht_tc.map2alm_tc(maps, spin, nside, lmax, 3)
        syn_skip = sht_tc.alm2map_tc(full, spin, nside, lmax)
    finally:
        sht_tc.USE_TILE_SKIP = old
    assert torch.equal(full, skip)
    assert torch.equal(syn_full, syn_skip)
    tp = sht_tc.get_tc_plan(nside, lmax)
    for sp, (seg_mask, unit_mask) in tp.ck_masks[spin].items():
        ngroups = tp.plan.nlanes // 64
        bits = (unit_mask.cpu().numpy().astype(np.uint64)[:, None] >> np.arange(ngroups, dtype=np.uint64)) & 1
        zero = 1.0 - bits.mean()
        assert 0.1 < zero < 0.3, (sp, zero)
        # a group is marked active exactly when one of its lanes has a non-zero state
        state, shift = sht_tc.ck_tables(tp, spin)[sp]
        nseg = seg_mask.shape[0]
        nz = ((state.view(nseg, -1, 2) != 0).any(dim=2) | (shift.view(nseg, -1) != 0))
        want = nz.view(nseg, ngroups, 64).any(dim=2).cpu().numpy()
        got = (seg_mask.cpu().numpy()[:, None].astype(np.uint64) >> np.arange(ngroups, dtype=np.uint64)) & 1
        assert np.array_equal(got.astype(bool), want)


@pytest.mark.parametrize("spin", [0, 2])
def test_simt_segment_skip_is_exact(cuda, spin):
    """The one-field SIMT passes skip the 128-row segments in which every lane of a CTA
    starts from a zero state.  The synthesis stays bit-identical; the analysis adds the same
    values, but its lane blocks add into each alm element with FP64 atomics in no fixed
    order, so it agrees to the rounding of those sums."""
    nside, lmax = 512, 1535
    rng = np.random.default_rng(41 + spin)
    maps = torch.from_numpy(rng.normal(size=(2, 12 * nside ** 2))).cuda()
    old = sht_tc.USE_TILE_SKIP
    try:
        sht_tc.USE_TILE_SKIP = False
        a_full = sht.map2alm_device(maps, spin, nside, lmax, 3, "mixed")
        m_full = sht.alm2map_device(a_full, spin, nside, lmax, "mixed")
        sht_tc.USE_TILE_SKIP = True
        assert sht.ck_args(sht.get_plan(nside, lmax), spin, 1)[-1] is not None
        a_skip = sht.map2alm_device(maps, spin, nside, lmax, 3, "mixed")
        m_skip = sht.alm2map_device(a_full, spin, nside, lmax, "mixed")
    finally:
        sht_tc.USE_TILE_SKIP = old
    assert float((a_full - a_skip).abs().max() / a_full.abs().max()) < 1e-13
    assert torch.equal(m_full, m_skip)
