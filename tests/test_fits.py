"""The minimal FITS writer/reader behind workspace files: layout rules of the FITS
Standard 4.0 (2880-byte blocks, 80-character cards, big-endian data) and round trips of
images, binary tables, keywords and the bandpower table."""

import numpy as np

from gmaster_b200 import fits
from gmaster_b200.bins import NmtBin


def test_card_layout():
    assert fits._card("SIMPLE", True) == "SIMPLE  =" + " " * 20 + "T" + " " * 50
    assert fits._card("NAXIS", 2) == "NAXIS   =" + " " * 20 + "2" + " " * 50
    c = fits._card("EXTNAME", "BEAMS")
    assert c.startswith("EXTNAME = 'BEAMS   '") and len(c) == 80
    assert fits._parse_value(fits._card("WAWB", 0.1)[10:]) == 0.1
    assert fits._parse_value(fits._card("X", "it's")[10:]) == "it's"
    assert fits._card("LMAX_MASK", 95).rstrip() == "HIERARCH LMAX_MASK = 95"


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    img = rng.normal(size=(5, 7))
    a = np.arange(9, dtype=np.int32) - 3
    b = rng.normal(size=9)
    c = np.arange(9, dtype=np.int64) * 10 ** 12
    header = {"LMAX": 47, "IS_TEB": False, "WAWB": 1.0 / 3.0, "NAME": "x", "NEG": -5,
              "LMAX_MASK": 95, "L_TOEPLITZ": -1}
    path = tmp_path / "t.fits"
    fits.write(path, [{"kind": "image", "name": "WSP_PRIMARY", "data": img, "header": header},
                      {"kind": "table", "name": "TAB", "columns": [("A", a), ("B", b), ("C", c)]}])
    raw = path.read_bytes()
    assert len(raw) % 2880 == 0
    assert raw[:30] == b"SIMPLE  =                    T"
    # big-endian data right after the first header block(s)
    hdus = fits.read(path)
    assert [h["name"] for h in hdus] == ["WSP_PRIMARY", "TAB"]
    assert np.array_equal(hdus[0]["data"], img)
    for k, v in header.items():
        assert hdus[0]["header"][k] == v
    t = hdus[1]["data"]
    assert np.array_equal(t["A"], a) and np.array_equal(t["B"], b) and np.array_equal(t["C"], c)
    assert t["A"].dtype == np.int32 and t["C"].dtype == np.int64
    start = raw.index(b"END" + b" " * 77) // 2880 * 2880 + 2880
    assert np.frombuffer(raw[start:start + 8], dtype=">f8")[0] == img[0, 0]


def test_bandpower_table_round_trip(tmp_path):
    b = NmtBin.from_lmax_linear(47, 4, is_Dell=True)
    path = tmp_path / "b.fits"
    fits.write(path, [{"kind": "image", "name": "P", "data": np.zeros((1, 1))}, b._fits_table()])
    b2 = NmtBin._from_fits_table(fits.read(path)[1])
    assert b2.lmax == b.lmax and b2.n_bands == b.n_bands
    assert np.array_equal(b2._ells_np, b._ells_np) and np.array_equal(b2._bpws_np, b._bpws_np)
    np.testing.assert_allclose(b2._weights_np, b._weights_np, rtol=1e-15)
    np.testing.assert_allclose(b2._f_ell_np, b._f_ell_np, rtol=1e-15)
