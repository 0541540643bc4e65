"""gmaster_b200 -- B200-native pseudo-C_ell MASTER estimator on HEALPix maps.

A drop-in for the hot path of licongxu/GMaster (NaMaster-style API):
`NmtField` -> `NmtWorkspace.from_fields` -> `compute_coupled_cell` -> `decouple_cell`,
plus `map2alm` / `alm2map` for spin 0 and spin 2.  Every stage runs in hand-written
sm_100a CUDA kernels (``libgm_b200.so``, C ABI in ``include/gm_b200.h``) on one GPU;
there is no CPU fallback.  Arrays are CUDA ``torch.Tensor``s.
"""

from . import utils
from ._config import (get_default_params, get_precision, latitudinal_method, nmt_params,
                      ring_dtype, set_latitudinal_method, set_n_iter_default, set_precision,
                      set_ring_precision, set_sht_calculator, set_table_precision,
                      set_tol_pinv_default, table_dtype)
from .unsupported import (NmtBinFlat, NmtCovarianceWorkspaceFlat, NmtFieldCatalog,
                          NmtFieldCatalogClustering, NmtFieldCatalogMomentum, NmtFieldFlat,
                          NmtWorkspaceFlat, alm2catalog, catalog2alm, compute_coupled_cell_flat,
                          compute_full_master_flat, deprojection_bias_flat,
                          gaussian_covariance_flat, mask_apodization_flat, synfast_flat)
from .batch import (SimulationGraph, compute_coupled_cells, decouple_cells, fields_from_maps,
                    mc_bandpowers, workspaces_from_fields)
from .bins import NmtBin
from .covariance import NmtCovarianceWorkspace, gaussian_covariance, get_iNKA_cell
from .field import NmtField
from .utils import (NmtAlmInfo, NmtMapInfo, alm2map, map2alm, map2alm_pair, mask_apodization,
                    moore_penrose_pinvh, synfast_spherical)
from .workspaces import (NmtWorkspace, compute_coupled_cell, compute_full_master,
                         coupling_precision, deprojection_bias, get_general_coupling_matrix,
                         get_master_coefficients, set_coupling_precision,
                         uncorr_noise_deprojection_bias)

__all__ = [
    "utils", "latitudinal_method", "ring_dtype", "set_latitudinal_method", "set_ring_precision",
    "set_table_precision", "table_dtype", "NmtBinFlat", "NmtCovarianceWorkspaceFlat",
    "NmtFieldCatalog", "NmtFieldCatalogClustering", "NmtFieldCatalogMomentum", "NmtFieldFlat",
    "NmtWorkspaceFlat", "alm2catalog", "catalog2alm", "compute_coupled_cell_flat",
    "compute_full_master_flat", "deprojection_bias_flat", "gaussian_covariance_flat",
    "mask_apodization_flat", "synfast_flat",
    "NmtAlmInfo", "NmtBin", "NmtCovarianceWorkspace", "NmtField", "NmtMapInfo", "NmtWorkspace",
    "alm2map", "gaussian_covariance", "get_iNKA_cell", "compute_full_master",
    "coupling_precision", "deprojection_bias", "get_general_coupling_matrix",
    "get_master_coefficients", "set_coupling_precision", "uncorr_noise_deprojection_bias",
    "compute_coupled_cell", "compute_coupled_cells", "decouple_cells", "fields_from_maps",
    "mc_bandpowers", "workspaces_from_fields", "SimulationGraph",
    "get_default_params", "get_precision", "map2alm", "map2alm_pair",
    "mask_apodization", "moore_penrose_pinvh", "nmt_params", "set_n_iter_default", "set_precision",
    "set_sht_calculator", "set_tol_pinv_default", "synfast_spherical",
]

__version__ = "0.1.0"
