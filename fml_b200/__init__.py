"""fml_b200 — B200 (sm_100a) implementation of andersx/fml's KRR hot path.

Drop-in names (same signatures and error behaviour as the reference):

* ``Molecule`` with ``read_xyz``, ``generate_coulomb_matrix``,
  ``generate_unsorted_coulomb_matrix``,
  ``generate_local_coulomb_matrix``, ``generate_atomic_coulomb_matrix``,
  ``generate_arad_descriptor`` (fml/fml.py)
* ``gaussian_kernel``, ``laplacian_kernel``, ``get_atomic_kernels_arad``,
  ``get_atomic_symmetric_kernels_arad`` (fml/kernels/kernels.py) and the
  atom-level ``fget_atomic_kernels_arad`` / ``fget_atomic_distance_arad``
  and ``fget_alpha_arad`` (fml/kernels/farad_kernels.f90), ``get_atomic_kernels_gaussian``,
  ``get_atomic_kernels_laplacian``, ``get_alpha``, ``get_prediction``,
  ``get_alpha_from_distance``, ``get_prediction_from_distance``
  (fml/kernels/kernels.py)
* ``cho_solve``, ``cho_invert`` (fml/math/cho_solve.py), ``get_l2_distance_arad``,
  ``manhattan_distance``, ``l2_distance``, ``p_distance`` (fml/math/distance.py)

Batched forms: ``read_xyz_batch`` (many .xyz files into one packed buffer),
``generate_coulomb_matrices``, ``generate_local_coulomb_matrices``,
``generate_arad_descriptors``; the fused KRR pipeline ``krr_fit_predict`` /
``KRRPipeline`` (descriptors, kernels for every sigma, factorisations, solves
and prediction on the device).

All compute runs in libfmlb.so (hand-written CUDA for sm_100a) through its C
ABI; torch is used for device buffers and streams only. There is no CPU
fallback: without the built library or a CUDA device the calls raise.
"""

from .cho_solve import CholeskyWarning, cho_invert, cho_solve
from .data import NUCLEAR_CHARGE, PTP
from .descriptors import (generate_arad_descriptors, generate_coulomb_matrices,
                          generate_local_coulomb_matrices, generate_unsorted_coulomb_matrices)
from .distance import get_l2_distance_arad, l2_distance, manhattan_distance, p_distance
from .kernels import (fget_alpha_arad, fget_atomic_distance_arad, fget_atomic_kernels_arad,
                      fget_kernel_arad, fget_vector_kernels_gaussian,
                      gaussian_kernel, get_alpha, get_alpha_from_distance,
                      get_atomic_kernels_arad, get_atomic_kernels_gaussian,
                      get_atomic_kernels_laplacian, get_atomic_symmetric_kernels_arad,
                      get_prediction, get_prediction_from_distance, laplacian_kernel)
from .krr import KRRPipeline, krr_fit_predict
from .molecule import Molecule
from .xyz import read_xyz_batch, read_xyz_molecules

__all__ = [
    "Molecule", "gaussian_kernel", "laplacian_kernel", "get_atomic_kernels_arad",
    "get_atomic_symmetric_kernels_arad", "fget_atomic_kernels_arad", "fget_alpha_arad",
    "fget_kernel_arad", "fget_vector_kernels_gaussian",
    "fget_atomic_distance_arad", "get_atomic_kernels_gaussian", "get_atomic_kernels_laplacian",
    "get_alpha", "get_prediction", "get_alpha_from_distance", "get_prediction_from_distance",
    "get_l2_distance_arad", "manhattan_distance", "l2_distance", "p_distance", "cho_solve",
    "cho_invert",
    "CholeskyWarning",
    "generate_coulomb_matrices", "generate_unsorted_coulomb_matrices",
    "generate_local_coulomb_matrices", "generate_arad_descriptors",
    "read_xyz_batch", "read_xyz_molecules", "KRRPipeline", "krr_fit_predict", "NUCLEAR_CHARGE",
    "PTP",
]
