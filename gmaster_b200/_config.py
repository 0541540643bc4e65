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
        ``"mixed"`` (default): single-precision ring stage and BF16-split / FP32
        contraction with FP64 recurrence, accumulation and refinement.
        ``"fp64"``: every stage in double precision.
    """

    def __init__(self):
        self.n_iter_default = 3
        self.n_iter_mask_default = 3
        self.tol_pinv_default = 1e-10
        self.precision = "mixed"
        self.sht_calculator = "gmaster_b200"


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
