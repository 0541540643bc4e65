"""Names of the reference's public API that lie outside this build: the flat-sky classes and
functions, catalog-based fields and their transforms.  They exist so that code written for
the reference fails with a clear `NotImplementedError` instead of an `AttributeError`."""

__all__ = [
    "NmtBinFlat", "NmtFieldFlat", "NmtWorkspaceFlat", "NmtCovarianceWorkspaceFlat",
    "NmtFieldCatalog", "NmtFieldCatalogClustering", "NmtFieldCatalogMomentum",
    "compute_coupled_cell_flat", "compute_full_master_flat", "deprojection_bias_flat",
    "gaussian_covariance_flat", "mask_apodization_flat", "synfast_flat", "catalog2alm",
    "alm2catalog",
]

_FLAT = "flat-sky (rectangular-patch) fields are not part of this build: HEALPix curved sky only"
_CATALOG = "catalog-based fields are not part of this build: HEALPix map fields only"


def _stub_class(name, reason):
    def __init__(self, *args, **kwargs):
        raise NotImplementedError(f"{name}: {reason}")

    @classmethod
    def _refuse(cls, *args, **kwargs):
        raise NotImplementedError(f"{name}: {reason}")

    return type(name, (), {"__init__": __init__, "__doc__": reason,
                           "from_fields": _refuse, "from_file": _refuse})


def _stub_function(name, reason):
    def fn(*args, **kwargs):
        raise NotImplementedError(f"{name}: {reason}")

    fn.__name__ = name
    fn.__doc__ = reason
    return fn


NmtBinFlat = _stub_class("NmtBinFlat", _FLAT)
NmtFieldFlat = _stub_class("NmtFieldFlat", _FLAT)
NmtWorkspaceFlat = _stub_class("NmtWorkspaceFlat", _FLAT)
NmtCovarianceWorkspaceFlat = _stub_class("NmtCovarianceWorkspaceFlat", _FLAT)
NmtFieldCatalog = _stub_class("NmtFieldCatalog", _CATALOG)
NmtFieldCatalogClustering = _stub_class("NmtFieldCatalogClustering", _CATALOG)
NmtFieldCatalogMomentum = _stub_class("NmtFieldCatalogMomentum", _CATALOG)
compute_coupled_cell_flat = _stub_function("compute_coupled_cell_flat", _FLAT)
compute_full_master_flat = _stub_function("compute_full_master_flat", _FLAT)
deprojection_bias_flat = _stub_function("deprojection_bias_flat", _FLAT)
gaussian_covariance_flat = _stub_function("gaussian_covariance_flat", _FLAT)
mask_apodization_flat = _stub_function("mask_apodization_flat", _FLAT)
synfast_flat = _stub_function("synfast_flat", _FLAT)
catalog2alm = _stub_function("catalog2alm", _CATALOG)
alm2catalog = _stub_function("alm2catalog", _CATALOG)
