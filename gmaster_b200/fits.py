"""Minimal FITS reader and writer for workspace files (no external FITS library).

Workspaces are stored in the FITS layout the reference writes through fitsio
(gmaster/workspaces.py:2162-2255, gmaster/bins.py:276-302): a primary image HDU with the
dense mode-coupling matrix and the workspace keywords, and binary tables for the beams,
the mask pseudo-spectrum and the bandpower definition.  Only what those files use is
implemented, following the FITS Standard 4.0: 2880-byte blocks, 80-character header
cards, big-endian data; 2-D float64 images; binary tables of scalar int32, int64,
float32 and float64 columns.
"""

import numpy as np

BLOCK = 2880
_TFORM = {"J": ">i4", "K": ">i8", "E": ">f4", "D": ">f8", "I": ">i2", "B": "u1"}
_TFORM_OF = {np.dtype("int32"): "1J", np.dtype("int64"): "1K", np.dtype("float32"): "1E",
             np.dtype("float64"): "1D", np.dtype("int16"): "1I", np.dtype("uint8"): "1B"}


def _card(key, value=None, comment=None):
    """One 80-character header card.  Keywords longer than 8 characters (LMAX_MASK,
    L_TOEPLITZ, ...) use the HIERARCH convention, as cfitsio writes them."""
    key = key.upper()
    if len(key) > 8:
        if value is None:
            raise ValueError(f"FITS keyword too long: {key}")
        v = _card("X", value)[10:].strip()
        text = f"HIERARCH {key} = {v}"
        if len(text) > 80:
            raise ValueError(f"FITS card too long: {text}")
        return f"{text:<80}"
    if value is None:
        text = f"{key:<8}"
    else:
        if isinstance(value, (bool, np.bool_)):
            v = f"{'T' if value else 'F':>20}"
        elif isinstance(value, (int, np.integer)):
            v = f"{int(value):>20d}"
        elif isinstance(value, (float, np.floating)):
            s = repr(float(value)).upper()
            if "E" not in s and "." not in s and s not in ("NAN", "INF", "-INF"):
                s += ".0"
            v = f"{s:>20}"
        else:
            s = str(value).replace("'", "''")
            v = f"'{s:<8}'"
        text = f"{key:<8}= {v}"
        if comment:
            text += f" / {comment}"
    if len(text) > 80:
        raise ValueError(f"FITS card too long: {text}")
    return f"{text:<80}"


def _header_bytes(cards):
    text = "".join(cards) + f"{'END':<80}"
    pad = (-len(text)) % BLOCK
    return (text + " " * pad).encode("ascii")


def _pad(data):
    return data + b"\0" * ((-len(data)) % BLOCK)


def _user_cards(header):
    cards = []
    for k, v in (header or {}).items():
        cards.append(_card(k, v))
    return cards


def write(path, hdus):
    """Write HDUs to `path` (overwritten).  Each HDU is a dict: ``{"kind": "image",
    "name": ..., "data": 2-D array, "header": {...}}`` or ``{"kind": "table", "name": ...,
    "columns": [(name, 1-D array), ...], "header": {...}}``.  The first HDU must be an
    image (it becomes the primary HDU, with its EXTNAME)."""
    if not hdus or hdus[0]["kind"] != "image":
        raise ValueError("the first HDU must be an image")
    with open(path, "wb") as fh:
        for i, h in enumerate(hdus):
            if h["kind"] == "image":
                data = np.ascontiguousarray(h["data"], dtype=np.float64)
                if data.ndim != 2:
                    raise ValueError("images must be 2-D")
                cards = [_card("SIMPLE", True) if i == 0 else _card("XTENSION", "IMAGE"),
                         _card("BITPIX", -64), _card("NAXIS", 2),
                         _card("NAXIS1", data.shape[1]), _card("NAXIS2", data.shape[0])]
                cards += [_card("EXTEND", True)] if i == 0 else [_card("PCOUNT", 0), _card("GCOUNT", 1)]
                cards.append(_card("EXTNAME", h["name"]))
                cards += _user_cards(h.get("header"))
                fh.write(_header_bytes(cards))
                fh.write(_pad(data.astype(">f8").tobytes()))
            elif h["kind"] == "table":
                if i == 0:
                    raise ValueError("the first HDU must be an image")
                cols = [(n, np.asarray(a)) for n, a in h["columns"]]
                nrows = len(cols[0][1])
                if any(a.ndim != 1 or len(a) != nrows for _, a in cols):
                    raise ValueError("table columns must be 1-D and of equal length")
                forms = []
                for n, a in cols:
                    if a.dtype not in _TFORM_OF:
                        raise ValueError(f"unsupported column type {a.dtype} for {n}")
                    forms.append(_TFORM_OF[a.dtype])
                rec = np.empty(nrows, dtype=[(n, _TFORM[f[-1]]) for (n, _), f in zip(cols, forms)])
                for n, a in cols:
                    rec[n] = a
                cards = [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2),
                         _card("NAXIS1", rec.dtype.itemsize), _card("NAXIS2", nrows),
                         _card("PCOUNT", 0), _card("GCOUNT", 1), _card("TFIELDS", len(cols))]
                for k, ((n, _), f) in enumerate(zip(cols, forms), 1):
                    cards += [_card(f"TTYPE{k}", n), _card(f"TFORM{k}", f)]
                cards.append(_card("EXTNAME", h["name"]))
                cards += _user_cards(h.get("header"))
                fh.write(_header_bytes(cards))
                fh.write(_pad(rec.tobytes()))
            else:
                raise ValueError(f"unknown HDU kind {h['kind']}")


def _parse_value(s):
    s = s.strip()
    if s.startswith("'"):
        end = 1
        out = []
        while end < len(s):
            if s[end] == "'":
                if end + 1 < len(s) and s[end + 1] == "'":
                    out.append("'")
                    end += 2
                    continue
                break
            out.append(s[end])
            end += 1
        return "".join(out).rstrip()
    v = s.split("/")[0].strip()
    if v == "T":
        return True
    if v == "F":
        return False
    try:
        return int(v)
    except ValueError:
        return float(v.replace("D", "E"))


def _read_header(fh):
    header = {}
    while True:
        block = fh.read(BLOCK)
        if len(block) < BLOCK:
            if not block:
                return None
            raise ValueError("truncated FITS header")
        text = block.decode("ascii")
        for i in range(0, BLOCK, 80):
            card = text[i:i + 80]
            key = card[:8].strip()
            if key == "END":
                return header
            if key == "HIERARCH" and "=" in card:
                k, v = card[9:].split("=", 1)
                header[k.strip()] = _parse_value(v)
            elif card[8:10] == "= ":
                header[key] = _parse_value(card[10:])


def read(path):
    """All HDUs of `path` as dicts {"name", "header", "data"} (image: 2-D float64 array;
    table: dict of column name -> native-endian 1-D array)."""
    out = []
    with open(path, "rb") as fh:
        while True:
            hdr = _read_header(fh)
            if hdr is None:
                break
            naxis = int(hdr.get("NAXIS", 0))
            dims = [int(hdr[f"NAXIS{k}"]) for k in range(1, naxis + 1)]
            nbytes = int(np.prod(dims)) * abs(int(hdr["BITPIX"])) // 8 if naxis else 0
            nbytes += int(hdr.get("PCOUNT", 0))
            raw = fh.read(nbytes)
            fh.read((-nbytes) % BLOCK)
            name = hdr.get("EXTNAME", "PRIMARY")
            if hdr.get("XTENSION") == "BINTABLE":
                nf = int(hdr["TFIELDS"])
                names = [hdr[f"TTYPE{k}"] for k in range(1, nf + 1)]
                forms = [str(hdr[f"TFORM{k}"]).strip() for k in range(1, nf + 1)]
                for f in forms:
                    if f.lstrip("1") not in _TFORM:
                        raise ValueError(f"unsupported table column format {f}")
                dt = np.dtype([(n, _TFORM[f.lstrip("1")]) for n, f in zip(names, forms)])
                rec = np.frombuffer(raw[:dt.itemsize * dims[1]], dtype=dt)
                data = {n: rec[n].astype(rec[n].dtype.newbyteorder("=")) for n in names}
            elif naxis:
                bitpix = int(hdr["BITPIX"])
                code = {-64: ">f8", -32: ">f4", 64: ">i8", 32: ">i4", 16: ">i2", 8: "u1"}[bitpix]
                arr = np.frombuffer(raw, dtype=code).astype(np.float64)
                data = arr.reshape(dims[::-1])
            else:
                data = None
            out.append({"name": name, "header": hdr, "data": data})
    return out
