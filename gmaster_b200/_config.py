"""Process-wide defaults (the counterpart of gmaster/_config.py:20-53, NmtParams)."""


class NmtParams:
    """Default settings.

    Attributes
    ----------
    n_iter_default, n_iter_mask_default : int
        Jacobi iterations used by map2alm for maps and for masks (reference default 3).
    tol_pinv_default : float
        Relative eigenvalue threshold of pseudo-inverses (kept for API parity).
    precision : str
        ``"mixed"`` (default): single-precision ring stage and f16-split (tensor cores) /
        FP32 (SIMT) contraction with FP64 recurrence, accumulation and refinement.
        ``"fp64"``: every stage in double precision.
    """

    def __init__(self):
        self.n_iter_default = 3
        self.n_iter_mask_default = 3
        self.tol_pinv_default = 1e-10
        self.precision = "mixed"
        self.sht_calculator = "gmaster_b200"
        self.ring_precision = "auto"
        self.table_dtype = "fp64"
        self.latitudinal_method = "auto"


nmt_params = NmtParams()


def get_default_params():
    return NmtParams()


def set_n_iter_default(n_iter, mask=False):
    """Set the default number of Jacobi iterations (gmaster/_config.py:304-318)."""
    if n_iter < 0:
        raise ValueError("n_iter must be non-negative")
    if mask:
        nmt_params.n_iter_mask_default = int(n_iter)
    else:
        nmt_params.n_iter_default = int(n_iter)


def set_tol_pinv_default(tol_pinv):
    if tol_pinv < 0:
        raise ValueError("tol_pinv must be non-negative")
    nmt_params.tol_pinv_default = float(tol_pinv)


def set_precision(name):
    """Choose the arithmetic of the transforms: ``"mixed"`` or ``"fp64"``."""
    if name not in ("mixed", "fp64"):
        raise KeyError("precision must be 'mixed' or 'fp64'")
    nmt_params.precision = name


def get_precision():
    return nmt_params.precision


def set_sht_calculator(name):
    if name not in ("gmaster_b200", "ducc", "healpy", "jax"):
        raise KeyError(f"unknown SHT calculator {name}")


# ----------------------------------------------------------------------------- engine knobs
# The reference's transform-engine settings (gmaster/_config.py:57-268).  This build has
# one latitudinal engine (the FP64-recurrence march, on SIMT or tensor-core kernels), no
# stored transform tables (rows are generated on the fly) and a ring stage whose precision
# follows `set_precision`; the settings are validated and recorded as in the reference.

_RING_NAMES = ("auto", "follow", "fp64", "fp32")
_TABLE_NAMES = ("fp64", "fp32")
_LATITUDINAL = ("auto", "march", "dc")


def set_ring_precision(name):
    """Record the ring-FFT precision setting (gmaster/_config.py:113-133).  The ring
    stage here runs in complex64 under the "mixed" precision and complex128 under "fp64"
    (`set_precision`); `ring_dtype` reports which."""
    if name not in _RING_NAMES:
        raise KeyError("GMaster ring precision must be 'auto', 'follow', 'fp64' or 'fp32'")
    nmt_params.ring_precision = name


def ring_dtype(L=None):
    """The element type of the ring FFTs the transforms use (gmaster/_config.py:74-110)."""
    import torch

    return torch.complex64 if nmt_params.precision == "mixed" else torch.complex128


def set_table_precision(name):
    """Record the table storage precision (gmaster/_config.py:202-226).  No transform
    tables are stored here (the Legendre rows are generated in FP64 as they are used)."""
    if name not in _TABLE_NAMES:
        raise KeyError("GMaster table precision must be 'fp64' or 'fp32'")
    nmt_params.table_dtype = name


def table_dtype():
    """The recorded table precision as a torch dtype (gmaster/_config.py:63-71)."""
    import torch

    return torch.float64 if nmt_params.table_dtype == "fp64" else torch.float32


def latitudinal_method():
    """The latitudinal engine setting (gmaster/_config.py:237-245)."""
    return nmt_params.latitudinal_method


def set_latitudinal_method(name):
    """Choose the latitudinal engine (gmaster/_config.py:248-268): "auto" and "march" both
    select this build's FP64-recurrence march; the divide-and-conquer engine ("dc") is
    outside this build."""
    if name not in _LATITUDINAL:
        raise KeyError("latitudinal method must be 'auto', 'march' (fp32 v2 difference form), "
                       "or 'dc' (divide-and-conquer)")
    if name == "dc":
        raise NotImplementedError("the divide-and-conquer latitudinal engine is not part of "
                                  "this build")
    nmt_params.latitudinal_method = name
