"""The FP64 oracle, pinned against the reference's golden vectors and known-answer tests.

Golden vectors (tests/golden/*.npz) were produced by running the reference's own
numpy code (tests/golden/make_golden.py).  Known-answer tests restate the reference's
self-contained checks: explicit ring DFTs (tests/test_sht.py:463-541), the threej
closed form (tests/test_workspaces.py:122-206) and the quadrature-vs-recurrence
agreement (tests/test_workspaces.py:247-282); plus exact Wigner-3j values from the
Racah formula in rational arithmetic and explicit low-l spherical harmonics.
"""

import math
from fractions import Fraction

import numpy as np
import pytest

import oracle

GOLD = "tests/golden/"


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 16, 32, 64, 256, 2048])
def test_geometry_bit_exact_with_reference(nside):
    g = np.load(GOLD + "geometry.npz")
    theta, phi0, nphi, off = oracle.geometry(nside)
    assert np.array_equal(theta, g[f"theta_{nside}"])
    assert np.array_equal(phi0, g[f"phi0_{nside}"])
    assert np.array_equal(nphi, g[f"nphi_{nside}"])
    assert np.array_equal(off, g[f"offsets_{nside}"])
    # the C restatement agrees on every integer and to one ulp on theta
    t2, p2, n2, o2 = oracle.geometry_c(nside)
    assert np.array_equal(n2, nphi) and np.array_equal(o2, off)
    assert np.max(np.abs(t2 - theta)) <= 4 * np.finfo(float).eps
    if nside >= 2:
        assert np.array_equal(nphi, g[f"czt_nphi_{nside}"])
        assert np.array_equal(off, g[f"czt_start_{nside}"])


@pytest.mark.parametrize("key", ["191_16", "47_4", "50_7", "6143_16", "23_1", "10_16"])
def test_linear_bands_match_reference(key):
    g = np.load(GOLD + "bins.npz")
    lmax, nlb = map(int, key.split("_"))
    ells, bpws = oracle.linear_bands(lmax, nlb)
    assert np.array_equal(ells, g[f"ells_{key}"])
    assert np.array_equal(bpws, g[f"bpws_{key}"])


@pytest.mark.parametrize("lmax", [15, 16, 17, 31, 40])
def test_tt_closed_form_matches_reference(lmax):
    g = np.load(GOLD + "coupling_tt.npz")
    got = oracle.coupling_tt_closed(g[f"window_{lmax}"], lmax)
    np.testing.assert_allclose(got, g[f"tt_{lmax}"], atol=2e-14, rtol=0)


def test_tt_triangle_replica_matches_reference():
    g = np.load(GOLD + "coupling_tt.npz")
    got = oracle.coupling_tt_closed(g["window_tri"], 24)
    np.testing.assert_allclose(got, g["tri64"], atol=2e-14, rtol=0)
    # the reference's float32-product arm stays within 1e-5 of scale
    assert np.max(np.abs(g["tri32"] - got)) / np.max(np.abs(got)) < 1e-5


@pytest.mark.parametrize("lmax", [24, 47, 60])
def test_tt_quadrature_matches_closed_form(lmax):
    window = np.random.default_rng(lmax).uniform(size=2 * lmax + 1)
    even, odd = oracle.coupling_quadrature(window, lmax, 0, 0, 0, 0)
    closed = oracle.coupling_tt_closed(window, lmax)
    np.testing.assert_allclose(even + odd, closed, atol=1e-11 * np.abs(closed).max(), rtol=0)


@pytest.mark.parametrize("nside,L", [(16, 47), (32, 95), (16, 64), (16, 71), (32, 40)])
def test_ring_analysis_matches_direct_dft(nside, L):
    """test_sht.py:463-491 restated: cap, boundary and belt rings vs the explicit sum."""
    theta, phi0, nphi, start = oracle.geometry(nside)
    x = np.random.default_rng(4).normal(size=12 * nside ** 2)
    got = oracle.ring_analysis(nside, L, x.astype(np.complex128))
    for ring in {0, nside // 2, nside - 2, nside - 1, nside, 2 * nside, 3 * nside - 1,
                 3 * nside, 4 * nside - 2}:
        n = nphi[ring]
        direct = np.exp(-2j * np.pi * np.outer(np.arange(L), np.arange(n)) / n) @ x[start[ring]:start[ring] + n]
        direct = direct * np.exp(-1j * np.arange(L) * phi0[ring])
        np.testing.assert_allclose(got[ring], direct, rtol=0, atol=1e-12 * np.abs(direct).max())


@pytest.mark.parametrize("nside,L", [(8, 16), (8, 23), (8, 39), (16, 71)])
def test_spin_ring_window_both_ways(nside, L):
    """test_sht.py:494-541 restated: centred window m in (-L, L), forward and back."""
    theta, phi0, nphi, start = oracle.geometry(nside)
    rng = np.random.default_rng(7)
    sig = rng.normal(size=12 * nside ** 2) + 1j * rng.normal(size=12 * nside ** 2)
    coef = rng.normal(size=(4 * nside - 1, 2 * L - 1)) + 1j * rng.normal(size=(4 * nside - 1, 2 * L - 1))
    fwd = oracle.ring_analysis(nside, L, sig, mneg=L - 1)
    back = oracle.ring_synthesis(nside, L, coef, mneg=L - 1)
    ms = np.arange(-(L - 1), L)
    for ring in {0, nside - 1, nside, 2 * nside, 4 * nside - 2}:
        n = nphi[ring]
        phi = phi0[ring] + 2 * np.pi * np.arange(n) / n
        direct = np.exp(-1j * np.outer(ms, phi)) @ sig[start[ring]:start[ring] + n]
        np.testing.assert_allclose(fwd[ring], direct, rtol=0, atol=1e-12 * np.abs(direct).max())
        syn = np.exp(1j * np.outer(phi, ms)) @ coef[ring]
        np.testing.assert_allclose(back[start[ring]:start[ring] + n], syn, rtol=0,
                                   atol=1e-12 * np.abs(syn).max())


@pytest.mark.parametrize("sp", [0, -2, 2])
@pytest.mark.parametrize("m", [0, 1, 2, 3, 7, 40, 90])
def test_lambda_rows_match_jacobi_closed_form(sp, m):
    """The scaled recurrence equals the Jacobi closed form (long double) wherever the
    row is above the 2^-300 flush threshold."""
    for th in (1e-3, 0.1, 0.7, 1.3, np.pi / 2, 2.0, 3.1):
        a = oracle.lambda_row(150, m, sp, th)
        b = oracle.lambda_row(150, m, sp, th, jacobi=True)
        big = np.abs(b) > 1e-80
        scale = max(np.abs(b).max(), 1e-300)
        assert np.all(np.abs(a[big] - b[big]) <= 1e-11 * scale)
        assert np.all(np.abs(a[~big]) < 1e-80)


def test_lambda_explicit_low_l():
    th = 0.83
    s, c = np.sin(th), np.cos(th)
    l0 = oracle.lambda_row(4, 0, 0, th)
    np.testing.assert_allclose(l0[1], np.sqrt(3 / (4 * np.pi)) * c, rtol=1e-14)
    np.testing.assert_allclose(l0[2], np.sqrt(5 / (16 * np.pi)) * (3 * c * c - 1), rtol=1e-14)
    np.testing.assert_allclose(oracle.lambda_row(4, 1, 0, th)[1], -np.sqrt(3 / (8 * np.pi)) * s, rtol=1e-14)
    np.testing.assert_allclose(oracle.lambda_row(4, 2, 0, th)[2], 0.25 * np.sqrt(15 / (2 * np.pi)) * s * s, rtol=1e-14)
    # spin 2: _{+-2}Y_20 = (1/4) sqrt(15/2pi) sin^2 (Goldberg), _{2}Y_21 = -(1/4) sqrt(5/pi) sin (1 - cos)
    np.testing.assert_allclose(oracle.lambda_row(4, 0, -2, th)[2], 0.25 * np.sqrt(15 / (2 * np.pi)) * s * s, rtol=1e-14)
    np.testing.assert_allclose(oracle.lambda_row(4, 0, 2, th)[2], 0.25 * np.sqrt(15 / (2 * np.pi)) * s * s, rtol=1e-14)
    np.testing.assert_allclose(oracle.lambda_row(4, 1, -2, th)[2], -0.25 * np.sqrt(5 / np.pi) * s * (1 - c), rtol=1e-13)


@pytest.mark.parametrize("spin", [0, 2])
def test_roundtrip_converges(spin):
    nside, lmax = 8, 16
    rng = np.random.default_rng(3)
    nm = 1 if spin == 0 else 2
    L = lmax + 1
    nel = L * (L + 1) // 2
    alm = rng.normal(size=(nm, nel)) + 1j * rng.normal(size=(nm, nel))
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    order = np.repeat(np.arange(L), L - np.arange(L))
    alm[:, order == 0] = alm[:, order == 0].real
    if spin:
        alm[:, ell < 2] = 0
    mp = oracle.alm2map(alm, spin, nside, lmax)
    back = oracle.map2alm(mp, spin, nside, lmax, 10)
    assert np.max(np.abs(back - alm)) < 1e-8


def _racah(j1, j2, j3, m1, m2, m3):
    """Exact Wigner 3j symbol (Racah formula) as (sign, Fraction of the square)."""
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    f = math.factorial
    tri = Fraction(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3), f(j1 + j2 + j3 + 1))
    pre = f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3)
    s = Fraction(0)
    for k in range(0, j1 + j2 + j3 + 1):
        den = [k, j3 - j2 + k + m1, j3 - j1 + k - m2, j1 + j2 - j3 - k, j1 - k - m1, j2 - k + m2]
        if min(den) < 0:
            continue
        term = Fraction((-1) ** k, math.prod(f(d) for d in den))
        s += term
    val2 = tri * pre * s * s
    sign = (-1) ** (j1 - j2 - m3) * (1 if s >= 0 else -1)
    return sign * math.sqrt(float(val2))


def test_racah_reference_values():
    assert abs(_racah(1, 1, 2, 1, -1, 0) - math.sqrt(1 / 30)) < 1e-15
    assert abs(_racah(1, 1, 2, 0, 0, 0) - math.sqrt(2 / 15)) < 1e-15
    assert abs(_racah(1, 1, 0, 0, 0, 0) + 1 / math.sqrt(3)) < 1e-15


@pytest.mark.parametrize("lmax", [8, 12])
def test_coupling_blocks_match_exact_3j_sums(lmax):
    """TT, TE, M+ and M- from the oracle equal the exact 3j sums of the MASTER formulae
    (NaMaster; Alonso et al. 2019 eqs. 19-20)."""
    window = np.random.default_rng(lmax).uniform(size=2 * lmax + 1)
    n = lmax + 1
    tt = np.zeros((n, n)); te = np.zeros((n, n)); pp = np.zeros((n, n)); mm = np.zeros((n, n))
    for l1 in range(n):
        for l2 in range(n):
            for l3 in range(abs(l1 - l2), min(l1 + l2, 2 * lmax) + 1):
                w = (2 * l3 + 1) * window[l3] / (4 * np.pi) * (2 * l2 + 1)
                a = _racah(l1, l2, l3, 0, 0, 0)
                b = _racah(l1, l2, l3, 2, -2, 0)
                tt[l1, l2] += w * a * a
                te[l1, l2] += w * a * b
                if (l1 + l2 + l3) % 2 == 0:
                    pp[l1, l2] += w * b * b
                else:
                    mm[l1, l2] += w * b * b
    np.testing.assert_allclose(oracle.coupling_tt_closed(window, lmax), tt, atol=1e-14)
    np.testing.assert_allclose(oracle.coupling_blocks(window, lmax, 0, 2)["te"], te, atol=1e-13)
    pol = oracle.coupling_blocks(window, lmax, 2, 2)
    np.testing.assert_allclose(pol["pp"], pp, atol=1e-13)
    np.testing.assert_allclose(pol["mm"], mm, atol=1e-13)


def test_pcl_matches_numpy():
    lmax = 20
    L = lmax + 1
    nel = L * (L + 1) // 2
    rng = np.random.default_rng(2)
    a = rng.normal(size=(2, nel)) + 1j * rng.normal(size=(2, nel))
    ell = np.concatenate([np.arange(m, L) for m in range(L)])
    order = np.repeat(np.arange(L), L - np.arange(L))
    got = oracle.pcl(a, a, lmax)
    for i in range(2):
        for j in range(2):
            prod = np.real(a[i] * np.conj(a[j])) * np.where(order == 0, 1, 2)
            want = np.bincount(ell, weights=prod, minlength=L) / (2 * np.arange(L) + 1)
            np.testing.assert_allclose(got[i * 2 + j], want, rtol=1e-14, atol=1e-14)


def test_gauss_legendre_integrates_polynomials():
    x, w = oracle.gauss_legendre(33)
    for k in range(0, 65, 4):
        np.testing.assert_allclose(np.sum(w * x ** k), 2 / (k + 1), rtol=1e-13)


def test_toeplitz_oracle_matches_reference_golden():
    """apply_toeplitz vs the reference's _apply_toeplitz run on the same inputs
    (tests/golden/toeplitz.npz, made by tests/golden/make_golden.py)."""
    g = np.load("tests/golden/toeplitz.npz")
    k = 0
    while f"case_{k}" in g:
        lmax, lt, le, db = (int(v) for v in g[f"case_{k}"])
        got = oracle.apply_toeplitz(g[f"S_{k}"], lt, le, db)
        np.testing.assert_allclose(got, g[f"out_{k}"], rtol=1e-14, atol=1e-16)
        k += 1
    assert k >= 5
    got = oracle.apply_toeplitz(g["random_S"], 9, 2, 3)
    np.testing.assert_allclose(got, g["random_out"], rtol=1e-14, atol=1e-16)


def test_toeplitz_exact_pairs_match_reference_golden():
    """The pair set the product computes exactly equals the reference's
    _toeplitz_exact_pairs (as unordered pairs)."""
    from gmaster_b200.workspaces import toeplitz_exact_pairs

    g = np.load("tests/golden/toeplitz.npz")
    k = 0
    while f"case_{k}" in g:
        lmax, lt, le, db = (int(v) for v in g[f"case_{k}"])
        ref = {tuple(sorted(p)) for p in g[f"pairs_{k}"].tolist()}
        got = {tuple(p) for p in toeplitz_exact_pairs(lmax + 1, lt, le, db).tolist()}
        assert got == ref
        k += 1


def test_toeplitz_parameter_checks():
    from gmaster_b200.workspaces import toeplitz_sanity

    toeplitz_sanity(-1, -1, -1, 10)
    with pytest.raises(ValueError):
        toeplitz_sanity(5, 0, 2, 10)
    with pytest.raises(ValueError):
        toeplitz_sanity(5, 6, 2, 10)
    with pytest.raises(ValueError):
        toeplitz_sanity(10, 3, 2, 10)
