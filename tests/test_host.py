"""Host-side logic of gmaster_b200 (no GPU): geometry, seeds, binning, C ABI exports."""

import ctypes
import math
import re

import numpy as np
import pytest

import oracle
from gmaster_b200 import _build, sht
from gmaster_b200.bins import NmtBin


@pytest.mark.parametrize("nside", [1, 2, 4, 64, 2048])
def test_product_geometry_bit_exact(nside):
    g = np.load("tests/golden/geometry.npz")
    theta, phi0, nphi, off = sht.ring_geometry(nside)
    assert np.array_equal(theta, g[f"theta_{nside}"])
    assert np.array_equal(phi0, g[f"phi0_{nside}"])
    assert np.array_equal(nphi.astype(np.int64), g[f"nphi_{nside}"])
    assert np.array_equal(off.astype(np.int64), g[f"offsets_{nside}"])


def test_ring_offsets_formula_matches_cumsum():
    """The kernels compute ring_nphi / ring_offset in closed form (gm_common.cuh)."""
    for nside in (1, 2, 3, 8, 64):
        _, _, nphi, off = sht.ring_geometry(nside)
        npix = 12 * nside * nside
        for r in range(4 * nside - 1):
            ring = r + 1
            north = 4 * nside - ring if ring > 2 * nside else ring
            n = 4 * north if north < nside else 4 * nside
            if ring < nside:
                o = 2 * ring * (ring - 1)
            elif ring <= 3 * nside:
                o = 2 * nside * (nside - 1) + (ring - nside) * 4 * nside
            else:
                k = 4 * nside - ring
                o = npix - 2 * k * (k + 1)
            assert n == nphi[r] and o == off[r]


def test_shifted_flags():
    for nside in (1, 4, 32):
        flags = sht.shifted_flags(nside)
        _, phi0, nphi, _ = sht.ring_geometry(nside)
        assert np.array_equal(flags == 1, phi0 > 0)


@pytest.mark.parametrize("m", [0, 1, 2, 3, 10, 150])
def test_seed_table_reproduces_first_row(m):
    """sign * 2^(log2N + pc log2 cos + ps log2 sin) is lambda_{l0,m} of the oracle."""
    L = 200
    seeds = sht.seed_table(L)
    rows = [(0, 0, 1.0)]
    for spin in range(1, sht.MAX_SPIN + 1):
        v = sht.seed_variant(spin)
        # the +s variant carries (-1)^s
        rows += [(v, -spin, 1.0), (v + 1, spin, -1.0 if spin & 1 else 1.0)]
    for var, sp, extra in rows:
        l0 = max(m, abs(sp))
        for th in (0.3, 1.1, np.pi / 2):
            lg, sign, pc, ps = seeds[var, m]
            f = lg + pc * math.log2(math.cos(th / 2)) + ps * math.log2(math.sin(th / 2))
            val = sign * 2.0 ** f
            want = extra * oracle.lambda_row(L - 1, m, sp, th)[l0]
            if abs(want) > 1e-250:
                assert abs(val - want) <= 1e-12 * abs(want), (var, sp, th)


def test_nmtbin_linear_matches_reference_bands():
    g = np.load("tests/golden/bins.npz")
    b = NmtBin.from_lmax_linear(191, 16)
    keep = g["bpws_191_16"] >= 0
    assert np.array_equal(b._ells_np, g["ells_191_16"][keep])
    assert np.array_equal(b._bpws_np, g["bpws_191_16"][keep])
    assert b.get_n_bands() == int(g["bpws_191_16"].max()) + 1
    np.testing.assert_allclose(b.get_weight_list(0), np.full(16, 1 / 16))


def test_nmtbin_edges_and_dell():
    b = NmtBin.from_edges([2, 10, 30], [10, 30, 50], is_Dell=True)
    assert b.get_n_bands() == 3
    assert b.lmax == 49
    np.testing.assert_allclose(b.get_fell_list(1), np.arange(10, 30) * np.arange(11, 31) / (2 * np.pi))
    with pytest.raises(RuntimeError):
        NmtBin(bpws=[0, 0], ells=[2, 3], weights=[0, 0])


def _header_symbols():
    text = open("include/gm_b200.h").read()
    return sorted(set(re.findall(r"^(?:int|int64_t|const char \*)\s*(gm_\w+)\(", text, re.M)))


def test_cabi_library_exports_every_header_symbol():
    """The in-tree library loads on a CPU-only host and exports every declared entry point
    (no compute calls without a GPU)."""
    _build.build()
    lib = ctypes.CDLL(_build.LIB)
    syms = _header_symbols()
    assert len(syms) >= 15
    for name in syms:
        assert hasattr(lib, name), name
    lib.gm_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.gm_version()
    lib.gm_ring_twiddle_count.restype = ctypes.c_int64
    lib.gm_ring_twiddle_count.argtypes = [ctypes.c_int64]
    assert lib.gm_ring_twiddle_count(2048) == 2048 * 2049
    # coupling work units: one per l1 and 32 consecutive l2 >= l1
    lib.gm_coupling_units.restype = ctypes.c_int64
    lib.gm_coupling_units.argtypes = [ctypes.c_int64]
    for lmax in (0, 1, 31, 32, 33, 95, 767, 6143):
        want = sum((lmax - l1) // 32 + 1 for l1 in range(lmax + 1))
        assert lib.gm_coupling_units(lmax) == want, lmax
    assert lib.gm_coupling_units(-1) == 0


def test_python_binding_covers_header():
    from gmaster_b200 import _lib

    for name in _header_symbols():
        assert name in _lib.SIGNATURES, name


def test_product_never_imports_oracle():
    import pathlib

    for path in pathlib.Path("gmaster_b200").rglob("*.py"):
        text = path.read_text()
        assert "import oracle" not in text and "from oracle" not in text, path


def test_compute_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from gmaster_b200 import _lib

    with pytest.raises(RuntimeError):
        _lib.require_cuda()


def test_checkpointed_analysis_lane_limit():
    """The checkpointed analysis walks a unit's 64-lane groups as one 64-bit word: above 4096
    lanes the entry point refuses the shape (before any device work) and the transforms keep
    to the carried-recurrence kernels (no checkpoint tables)."""
    from types import SimpleNamespace

    from gmaster_b200 import _lib, sht_tc

    lib = _lib.load()
    bad_shape = [k for k, v in _lib.STATUS.items() if v == "GM_ERR_BAD_SHAPE"][0]
    null = [None] * 6
    for nside, want_shape in ((2048, False), (2049, True), (3000, True)):
        st = lib.gm_ck_analysis(nside, 3 * nside - 1, 2, -2, 4, *null, None, None, 1.0, 148, None, None)
        assert (st == bad_shape) == want_shape, (nside, st)
    tp = SimpleNamespace(plan=SimpleNamespace(nlanes=sht_tc.CK_MAX_LANES + 2), ck={})
    assert sht_tc.CK_MAX_LANES == 4096 and sht_tc.ck_tables(tp, 2) is None


def test_legendre_tile_list():
    """The autotuner's tile shapes are listed by the library without a GPU."""
    from gmaster_b200 import autotune

    t0, t2 = autotune.tiles(0), autotune.tiles(2)
    assert (1, 1) in t0 and len(t0) == len(set(t0))
    assert all(32 % (2 * nc) == 0 for nc, _ in t0)
    assert all(nc == 2 for nc, _ in t2)
    assert autotune.tiles(1) == t2 and autotune.tiles(sht.MAX_SPIN) == t2   # polarised kernels
    with pytest.raises(ValueError):
        autotune.tiles(sht.MAX_SPIN + 1)
    import os

    assert autotune.autotune_enabled() == (os.environ.get("GMASTER_B200_AUTOTUNE", "1") != "0")


def test_mask_alm_cache_follows_the_mask_tensor():
    """Mask alms are shared between fields of one mask tensor, never served after the
    mask changed in place, and dropped with the tensor."""
    import gc

    import torch

    from gmaster_b200 import field as F

    class _Info:
        lmax = 5

    class _Field:
        pass

    f = _Field()
    f.mask, f.ainfo_mask, f.n_iter_mask, f.precision = torch.zeros(12), _Info(), 3, "mixed"
    assert F._cached_mask_alms(f) is None
    F._store_mask_alms(f, torch.ones(3))
    assert F._cached_mask_alms(f) is not None
    f.precision = "fp64"
    assert F._cached_mask_alms(f) is None
    f.precision = "mixed"
    f.mask.add_(1.0)
    assert F._cached_mask_alms(f) is None
    n = len(F._MASK_ALMS)
    del f.mask
    gc.collect()
    assert len(F._MASK_ALMS) == n - 1


def test_mask_apodization_validates_before_any_device_work():
    """Argument errors of mask_apodization (gmaster/utils.py:92-101) need no GPU."""
    from gmaster_b200 import mask_apodization

    mask = np.ones(12 * 8 ** 2)
    with pytest.raises(ValueError, match="unknown"):
        mask_apodization(mask, 1.0, apotype="C3")
    with pytest.raises(ValueError, match="positive"):
        mask_apodization(mask, -1.0)
    with pytest.raises(ValueError, match="one-dimensional"):
        mask_apodization(np.ones((2, 768)), 1.0)


def test_pixel_radius_bound_matches_oracle_and_bounds_the_pixels():
    """The Smooth zeroing margin: the product's bound equals the oracle's restatement, and
    it exceeds the distance from every pixel centre to the nearest centre of a neighbouring
    ring (the vertices lie at least that far apart)."""
    import oracle
    from gmaster_b200.utils import max_pixel_radius

    for nside in (1, 2, 4, 16, 256, 2048):
        got = max_pixel_radius(nside)
        assert abs(got - oracle.pixel_radius_bound(nside)) < 1e-9 * got
        theta = oracle.geometry(nside)[0]
        assert got >= 0.5 * np.max(np.diff(theta))
        assert got < 1.25 / nside + 0.2 / nside ** 2


def test_oracle_apodization_nearest_pixel_is_exact():
    """The oracle's k-d tree distances (C1/C2) against a brute-force minimum over all
    masked pixels at Nside 8: pins the restatement of gmaster/utils.py:130-146."""
    import oracle

    nside = 8
    vec = oracle.pix2vec(nside)
    mask = (vec[:, 2] < 0.3).astype(float)
    mask[[17, 300, 555]] = 0.0
    for apotype in ("C1", "C2"):
        got = oracle.mask_apodization(mask, 25.0, apotype)
        mv = vec[mask <= 0]
        d2 = ((vec[:, None, :] - mv[None, :, :]) ** 2).sum(axis=2).min(axis=1)
        thr = 1 - np.cos(np.radians(25.0))
        x = np.sqrt(0.5 * d2 / thr)
        f = x - np.sin(2 * np.pi * x) / (2 * np.pi) if apotype == "C1" else 0.5 * (1 - np.cos(np.pi * x))
        want = np.where((mask > 0) & (0.5 * d2 < thr), mask * f, mask)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-14)


def _emulate_cov_terms(kernels, rows, signs, bptr, spec):
    """The per-element sum of gm_cov_binned / gm_cov_coupled, restated in numpy."""
    L = spec.shape[1]
    out = np.zeros((len(bptr) - 1, L, L))
    for x in range(len(bptr) - 1):
        for t in range(bptr[x], bptr[x + 1]):
            k, ra, rb = rows[t]
            A, B = spec[ra], spec[rb]
            sym = 0.5 * (A[:, None] * B[None, :] + A[None, :] * B[:, None])
            out[x] += signs[t] * sym * np.asarray(kernels[k])
    return out


@pytest.mark.parametrize("spins", [(a, b, c, d) for a in (0, 2) for b in (0, 2)
                                   for c in (0, 2) for d in (0, 2)])
def test_covariance_term_table_matches_oracle_assembly(spins):
    """The term table the CUDA covariance kernels evaluate (kernel, spectra rows, sign per
    output block) reproduces the reference's assembly loops (gmaster/covariance.py:
    407-429) restated in the oracle, for every spin combination, with random kernels."""
    import oracle
    import torch

    from gmaster_b200.covariance import NmtCovarianceWorkspace, _kernel_spins

    rng = np.random.default_rng(sum(s << i for i, s in enumerate(spins)))
    L = 5
    cw = NmtCovarianceWorkspace()
    cw.spins = spins
    cw._post_init()
    names = {(0, 0): ("00",), (0, 2): ("0s",), (2, 2): ("pp", "mm")}
    pairs = (_kernel_spins(spins[0], spins[1], spins[2], spins[3]),
             _kernel_spins(spins[0], spins[1], spins[3], spins[2]))
    cw.xiSS = []
    for pair in pairs:
        d = {n: None for n in ("00", "0s", "pp", "mm")}
        for n in names[pair]:
            d[n] = torch.from_numpy(rng.normal(size=(L, L)))
        cw.xiSS.append(d)
    na, nb, nc, nd = cw.nmaps
    cls = [rng.normal(size=(r, L)) for r in (na * nc, na * nd, nb * nc, nb * nd)]
    kernels, rows, signs, bptr = cw._terms()
    got = _emulate_cov_terms([k.numpy() for k in kernels], rows, signs, bptr, np.concatenate(cls))
    xis = [{k: (None if v is None else v.numpy()) for k, v in d.items()} for d in cw.xiSS]
    want = oracle.nka_assemble(spins, xis, *cls, L).reshape(cw.nclsa * cw.nclsb, L, L)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


def test_oracle_general_spin_form_equals_pinned_spin2():
    """The oracle's literal spin-s analysis (plus at +-m, healpix.py:800-814) reproduces its
    spin-2 form, which the golden vectors pin, so the spin-1 and spin-3 checks rest on it."""
    rng = np.random.default_rng(5)
    nside, lmax = 8, 23
    qu = rng.normal(size=(2, 12 * nside ** 2))
    for n_iter in (0, 2):
        a = oracle.map2alm(qu, 2, nside, lmax, n_iter)
        b = oracle.map2alm(qu, 2, nside, lmax, n_iter, general=True)
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(a))


def test_oracle_purification_quadrature_is_pinned():
    """The oracle's restatement of the purified quadrature (gmaster/workspaces.py:608-679,
    927-1061): its Wigner rows are the oracle's own rows transposed (d_mn = d_nm(-beta)),
    its standard blocks equal the 3j blocks, and on the full sky (no mask derivatives)
    every purified block equals its standard one."""
    import oracle

    beta = np.array([0.2, 1.3, 2.8])
    ell = np.arange(31)
    norm = np.sqrt((2 * ell + 1) / (4 * np.pi))
    for m, n in ((0, 1), (1, 2), (0, 2), (2, 2), (0, -2), (-2, -2), (1, 1)):
        got = oracle.wigner_d_table(beta, m, n, 30)
        want = np.stack([oracle.lambda_row(30, n, m, b) for b in beta]) / norm[None]
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-13)
    nside, lmax = 8, 23
    vec = oracle.pix2vec(nside)
    mask = (vec[:, 2] < 0.5) * (0.5 + 0.5 * vec[:, 0] ** 2)
    am = oracle.map2alm(mask[None], 0, nside, lmax, 3)
    window = oracle.pcl(am, am, lmax)[0]
    b = oracle.coupling_blocks_pure(window, lmax)
    te = oracle.coupling_blocks(window, lmax, 0, 2)["te"]
    pm = oracle.coupling_blocks(window, lmax, 2, 2)
    for got, want in ((b[0], te), (b[1], pm["pp"]), (b[2], pm["mm"])):
        assert np.max(np.abs(got - want)) < 1e-13 * np.max(np.abs(want))
    full = np.zeros(lmax + 1)
    full[0] = 4 * np.pi
    f = oracle.coupling_blocks_pure(full, lmax)
    for p, q in ((3, 0), (4, 1), (6, 1), (5, 2), (7, 2)):
        assert np.max(np.abs(f[p] - f[q])) < 1e-13


def test_coupling_precision_setting():
    import gmaster_b200 as nmt

    old = nmt.coupling_precision()
    try:
        for name in ("fp64", "fp32", "auto"):
            nmt.set_coupling_precision(name)
            assert nmt.coupling_precision() == name
        with pytest.raises(KeyError):
            nmt.set_coupling_precision("fp16")
    finally:
        nmt.set_coupling_precision(old)


@pytest.mark.parametrize("ncls,flags", [(2, (False, False, False, True)), (2, (False, False, True, True)),
                                        (4, (False, True, False, True)), (4, (True, True, False, False)),
                                        (4, (True, False, False, True)), (7, (False, False, False, True)),
                                        (7, (False, False, True, True))])
def test_purified_slot_levels_match_the_reference_rule(monkeypatch, ncls, flags):
    """The slot -> block choice of purified workspaces (gmaster/workspaces.py:1852-1897), on
    the CPU with random stand-in blocks: the dense matrix equals the oracle's restatement,
    and rebuilding per-slot blocks from it (what a file read does) gives it back."""
    import oracle
    import torch

    from gmaster_b200 import pure
    from gmaster_b200 import workspaces as wsm

    rng = np.random.default_rng(ncls + 10 * sum(flags))
    lmax = 6
    n = lmax + 1
    fake8 = tuple(torch.from_numpy(rng.normal(size=(n, n))) for _ in range(8))
    tt = torch.from_numpy(rng.normal(size=(n, n)))
    monkeypatch.setattr(pure, "coupling_blocks_pure", lambda window, lm: fake8)

    def fake_blocks(window, lm, which):
        out = torch.zeros((4, n, n), dtype=torch.float64)
        out[wsm._BLOCK_TT] = tt
        return out

    monkeypatch.setattr(wsm, "coupling_blocks", fake_blocks)
    w = wsm.NmtWorkspace()
    w.lmax, w.ncls = lmax, ncls
    w.window = torch.zeros(2 * lmax + 1, dtype=torch.float64)
    w.pure_e1, w.pure_b1, w.pure_e2, w.pure_b2 = flags
    w._compute_pure_blocks()
    got = w.get_coupling_matrix().numpy()
    want = oracle.assemble_pure_mcm(tuple(b.numpy() for b in fake8), tt.numpy(), lmax, ncls, flags)
    np.testing.assert_array_equal(got, want)
    slots = wsm._slot_blocks_from_dense(got, lmax, ncls, "cpu")
    w._slot_blocks = slots
    np.testing.assert_array_equal(w.get_coupling_matrix().numpy(), want)


def test_covariance_kernel_spin_rule_equals_the_reference_table():
    """The rule choosing the kernels of each Wick contraction equals the table of
    gmaster/covariance.py:266-283 (restated in the oracle) for all 16 spin combinations."""
    import oracle
    from gmaster_b200.covariance import _kernel_spins

    for (a1, a2, b1, b2), (p0, p1) in oracle._COV_PAIRS.items():
        assert _kernel_spins(a1, a2, b1, b2) == p0
        assert _kernel_spins(a1, a2, b2, b1) == p1


def test_covariance_workspace_file_layout_on_the_host(tmp_path):
    """write_to / read_from of a covariance workspace in the reference's FITS layout
    (gmaster/covariance.py:578-658), with host tensors."""
    import torch

    from gmaster_b200 import fits
    from gmaster_b200.covariance import NmtCovarianceWorkspace

    rng = np.random.default_rng(1)
    n = 9
    cw = NmtCovarianceWorkspace()
    cw.spins = (0, 2, 0, 2)
    cw.spin_a1, cw.spin_a2, cw.spin_b1, cw.spin_b2 = cw.spins
    cw.lmax, cw.lmax_mask = n - 1, n - 1
    cw.l_toeplitz, cw.l_exact, cw.dl_band = -1, -1, -1
    cw._post_init()
    xi0 = {"00": None, "0s": torch.from_numpy(rng.normal(size=(n, n))), "pp": None, "mm": None}
    xi1 = {"00": torch.from_numpy(rng.normal(size=(n, n))), "0s": None, "pp": None, "mm": None}
    cw.xiSS = [xi0, xi1]
    path = str(tmp_path / "cw.fits")
    cw.write_to(path)
    names = [h["name"] for h in fits.read(path)]
    assert names == ["CWSP_PRIMARY", "XI02_1122", "XI00_1221"]
    back = NmtCovarianceWorkspace()
    back.read_from(path, device="cpu")
    assert back.spins == (0, 2, 0, 2) and back.nclsa == 2 and back.nclsb == 2
    np.testing.assert_array_equal(back.xiSS[0]["0s"].numpy(), xi0["0s"].numpy())
    np.testing.assert_array_equal(back.xiSS[1]["00"].numpy(), xi1["00"].numpy())
    assert back.xiSS[0]["00"] is None and back.xiSS[1]["0s"] is None


def _emulate_cov_binned(cov, ops_a, ops_b):
    """The band-pair reduction of gm_cov_binned restated in numpy: for bands p, q the sum
    over l1 in p and l2 in q of w_a[l1] w_b[l2] cov[x, l1, l2], from the CSR operators."""
    pa, ea, wa = (ops_a[k].numpy() for k in ("ptr", "ells", "wfl"))
    pb, eb, wb = (ops_b[k].numpy() for k in ("ptr", "ells", "wfl"))
    out = np.zeros((cov.shape[0], len(pa) - 1, len(pb) - 1))
    for p in range(len(pa) - 1):
        l1 = ea[pa[p]:pa[p + 1]]
        for q in range(len(pb) - 1):
            l2 = eb[pb[q]:pb[q + 1]]
            blk = cov[:, l1][:, :, l2]
            out[:, p, q] = np.einsum("xij,i,j->x", blk, wa[l1], wb[l2])
    return out


def test_covariance_band_reduction_matches_the_reference_binning():
    """gm_cov_binned's reduction over the bins' CSR lists equals the reference's binning
    einsum (gmaster/covariance.py:533-538) with its output operator, for linear bands, ragged
    bands with f_ell (D_l) and two different binnings."""
    import oracle

    rng = np.random.default_rng(9)
    lmax = 30
    cov = rng.normal(size=(3, lmax + 1, lmax + 1))
    lin = NmtBin.from_lmax_linear(lmax, 4)
    rag = NmtBin.from_edges([2, 5, 13, 20], [5, 13, 20, 31], is_Dell=True)
    for ba, bb in ((lin, lin), (rag, lin), (lin, rag)):
        got = _emulate_cov_binned(cov, ba.device_operators("cpu"), bb.device_operators("cpu"))

        def output_op(b):
            op = np.zeros((b.get_n_bands(), lmax + 1))
            op[b._bpws_np, b._ells_np] = b._weights_np * b._f_ell_np
            return op

        want = np.einsum("pl,xlm,qm->xpq", output_op(ba), cov, output_op(bb))
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)
    out, _ = oracle.binning_operators(lmax, 4)
    want = np.einsum("pl,xlm,qm->xpq", out, cov, out)
    got = _emulate_cov_binned(cov, lin.device_operators("cpu"), lin.device_operators("cpu"))
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)


def test_public_names_cover_the_reference_api():
    """Every name the reference exports (gmaster/__init__.py __all__) exists here; the ones
    outside this build (flat sky, catalogs, the divide-and-conquer engine) raise
    NotImplementedError, and the engine knobs validate their arguments as the reference."""
    import gmaster_b200 as nmt

    ref = ["NmtAlmInfo", "NmtBin", "NmtBinFlat", "NmtField", "NmtFieldFlat", "NmtFieldCatalog",
           "NmtFieldCatalogClustering", "NmtFieldCatalogMomentum", "NmtCovarianceWorkspace",
           "NmtCovarianceWorkspaceFlat", "NmtMapInfo", "NmtWorkspace", "NmtWorkspaceFlat",
           "alm2map", "compute_coupled_cell", "compute_coupled_cell_flat", "compute_full_master",
           "compute_full_master_flat", "coupling_precision", "deprojection_bias",
           "deprojection_bias_flat", "gaussian_covariance", "gaussian_covariance_flat",
           "get_default_params", "get_general_coupling_matrix", "get_iNKA_cell",
           "get_master_coefficients", "latitudinal_method", "map2alm", "mask_apodization",
           "mask_apodization_flat", "moore_penrose_pinvh", "nmt_params", "ring_dtype",
           "set_coupling_precision", "set_latitudinal_method", "set_n_iter_default",
           "set_ring_precision", "set_sht_calculator", "set_table_precision",
           "set_tol_pinv_default", "synfast_flat", "synfast_spherical", "table_dtype",
           "uncorr_noise_deprojection_bias", "utils"]
    assert [n for n in ref if not hasattr(nmt, n)] == []
    for cls in (nmt.NmtFieldFlat, nmt.NmtBinFlat, nmt.NmtWorkspaceFlat, nmt.NmtFieldCatalog):
        with pytest.raises(NotImplementedError):
            cls(None)
    with pytest.raises(NotImplementedError):
        nmt.NmtCovarianceWorkspaceFlat.from_fields(None, None, None)
    for fn in (nmt.compute_coupled_cell_flat, nmt.synfast_flat, nmt.mask_apodization_flat):
        with pytest.raises(NotImplementedError):
            fn(None)
    old = (nmt.nmt_params.ring_precision, nmt.nmt_params.table_dtype, nmt.latitudinal_method())
    try:
        nmt.set_ring_precision("fp32")
        nmt.set_table_precision("fp32")
        nmt.set_latitudinal_method("march")
        assert nmt.latitudinal_method() == "march"
        with pytest.raises(KeyError):
            nmt.set_ring_precision("fp16")
        with pytest.raises(KeyError):
            nmt.set_table_precision("auto")
        with pytest.raises(KeyError):
            nmt.set_latitudinal_method("fast")
        with pytest.raises(NotImplementedError):
            nmt.set_latitudinal_method("dc")
    finally:
        nmt.set_ring_precision(old[0])
        nmt.set_table_precision(old[1])
        nmt.set_latitudinal_method(old[2])


@pytest.mark.parametrize("spins,is_teb", [((0, 1), False), ((1, 0), False), ((1, 3), False),
                                          ((3, 3), False), ((0, 3), True), ((1, 2), False),
                                          ((0, 5), False)])
def test_general_spin_slot_signs_match_the_reference_rule(monkeypatch, spins, is_teb):
    """Slots and signs of workspaces with spins other than 0/2 (gmaster/workspaces.py:
    1811-1831, 1856-1897), on the CPU with stand-in blocks for the quadrature (the
    quadrature itself is GPU-tested against the oracle): the dense matrix equals the
    oracle's restatement, and a file-style rebuild from it gives it back."""
    import oracle
    import torch

    from gmaster_b200 import workspaces as wsm

    rng = np.random.default_rng(sum(spins) + 7 * is_teb)
    lmax = 5
    n = lmax + 1
    calls = {}

    def fake_general(mask_cl, s1, s2, n1, n2, lm, lmm, table_bytes=None):
        key = (s1, s2, n1, n2)
        if key not in calls:
            calls[key] = torch.from_numpy(rng.normal(size=(2, n, n)))
        return calls[key]

    tt = torch.from_numpy(rng.normal(size=(n, n)))

    def fake_blocks(window, lm, which):
        out = torch.zeros((4, n, n), dtype=torch.float64)
        out[wsm._BLOCK_TT] = tt
        return out

    monkeypatch.setattr(wsm, "general_coupling_matrix", fake_general)
    monkeypatch.setattr(wsm, "coupling_blocks", fake_blocks)
    w = wsm.NmtWorkspace()
    w.spin1, w.spin2 = spins
    w.is_teb = is_teb
    w.ncls = 7 if is_teb else (2 if 0 in spins else 4)
    w.lmax = w.lmax_mask = lmax
    w.pcl_mask = torch.zeros(n, dtype=torch.float64)
    w.window = w.pcl_mask
    w.l_toeplitz = w.l_exact = w.dl_band = -1
    w._pure_any = False
    w._compute_blocks()
    got = w.get_coupling_matrix().numpy()
    s1, s2 = spins
    te = even = odd = None
    if s1 == 0 or s2 == 0:
        te = calls[(s1, s2, s1, s2)].sum(0).numpy()
    else:
        even, odd = (x.numpy() for x in calls[(s1, s2, s1, s2)])
    if is_teb:
        even, odd = (x.numpy() for x in calls[(s2, s2, s2, s2)])
    want = oracle.assemble_general_mcm(te, even, odd, tt.numpy(), lmax, s1, s2, is_teb)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-15)
    slots = wsm._slot_blocks_from_dense(got, lmax, w.ncls, "cpu")
    w._slot_blocks = slots
    np.testing.assert_allclose(w.get_coupling_matrix().numpy(), want, rtol=0, atol=1e-15)


def test_oracle_general_assembly_reduces_to_the_spin2_assembly():
    import oracle

    rng = np.random.default_rng(3)
    n = 5
    te, even, odd, tt = (rng.normal(size=(n, n)) for _ in range(4))
    for s1, s2 in ((0, 2), (2, 0), (2, 2), (0, 0)):
        blocks = {"tt": tt, "te": te, "pp": even, "mm": odd}
        np.testing.assert_array_equal(oracle.assemble_general_mcm(te, even, odd, tt, n - 1, s1, s2),
                                      oracle.assemble_mcm(blocks, n - 1, s1, s2))


def _split_args(text):
    """Top-level comma-separated arguments of a call's parenthesised text."""
    depth, cur, out = 0, [], []
    for ch in text.replace("->", "."):
        if ch in "(<[{":
            depth += 1
        elif ch in ")>]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    if "".join(cur).strip():
        out.append("".join(cur).strip())
    return out


def _balanced(src, start):
    """Text between the parenthesis at src[start] and its match."""
    depth = 0
    for i in range(start, len(src)):
        if src[i] == "(":
            depth += 1
        elif src[i] == ")":
            depth -= 1
            if depth == 0:
                return src[start + 1:i]
    raise ValueError("unbalanced")


def test_ffi_handlers_bind_header_entry_points():
    """gmaster_b200/csrc/ffi/gm_ffi.cc (the jax.ffi handlers, compiled where jaxlib's XLA FFI
    headers exist): every gmb_* symbol is bound to a handler defined in the file whose
    parameters follow its binding (stream, Arg buffers, Ret buffers, then attributes of the
    bound types), and every gm_* call passes as many arguments as include/gm_b200.h declares."""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = open(os.path.join(root, "gmaster_b200", "csrc", "ffi", "gm_ffi.cc")).read()
    header = open(os.path.join(root, "include", "gm_b200.h")).read()
    decl = {m.group(2): len(_split_args(m.group(3))) for m in
            re.finditer(r"\b(int|int64_t|const char \*)\s+(gm_\w+)\s*\(([^;]*?)\);", header, re.S)}
    impls = {}
    for m in re.finditer(r"ffi::Error\s+(\w+)\s*\(", src):
        params = _split_args(_balanced(src, m.end() - 1))
        impls[m.group(1)] = params
    symbols = re.findall(r"XLA_FFI_DEFINE_HANDLER_SYMBOL\((gmb_\w+),\s*(\w+),", src)
    assert len(symbols) >= 20
    for sym, impl in symbols:
        assert impl in impls, (sym, impl)
        start = src.index(f"XLA_FFI_DEFINE_HANDLER_SYMBOL({sym},")
        binding = _balanced(src, src.index("(", start))
        kinds = re.findall(r"\.(Arg|Ret|Attr)<([^>]+)>", binding)
        params = impls[impl]
        assert params[0].startswith("cudaStream_t"), sym
        assert len(params) == 1 + len(kinds), (sym, len(params), len(kinds))
        for (kind, typ), param in zip(kinds, params[1:]):
            if kind == "Arg":
                assert param.startswith("ffi::AnyBuffer"), (sym, param)
            elif kind == "Ret":
                assert param.startswith("ffi::Result<ffi::AnyBuffer>"), (sym, param)
            else:
                assert param.split()[0] == typ, (sym, param, typ)
    calls = 0
    for m in re.finditer(r"\b(gm_\w+)\(", src):
        name = m.group(1)
        if name == "gm_last_error":
            continue
        assert name in decl, name
        args = _split_args(_balanced(src, m.end() - 1))
        assert len(args) == decl[name], (name, len(args), decl[name])
        calls += 1
    assert calls >= 20
