"""Why the KRR solve stays in FP64 (CPU, oracle and LAPACK only).

For the large-N configuration's data (sorted Coulomb matrices, up to 29
atoms) the Gaussian kernel matrix has eigenvalues spread from ~1e3 down to
the rounding level, so K + lambda*I at lambda in {1e-6, 1e-8} has a condition
number of 1e9..1e11. Rounding it to FP32 (relative error ~6e-8 per entry)
already makes it indefinite: an FP32 Cholesky factorisation breaks down,
while the FP64 one succeeds. An FP32 factor therefore cannot serve as the
solver or as the preconditioner of an FP64 refinement at these lambdas, and
the library factors in FP64 on the tensor cores (DMMA).
"""

import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from fml_b200 import synthetic


@pytest.fixture(scope="module")
def cm_kernel_inputs(oracle_mod):
    b = synthetic.generate(1024, nmax=29, seed=2)
    return oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 29)


@pytest.mark.parametrize("sigma", [100.0, 400.0, 1600.0])
@pytest.mark.parametrize("lam", [1e-6, 1e-8])
def test_fp32_cholesky_breaks_down_where_fp64_succeeds(oracle_mod, cm_kernel_inputs, sigma, lam):
    X = cm_kernel_inputs
    A = oracle_mod.gaussian_kernel(X.T, X.T, sigma) + lam * np.eye(len(X))
    _, info32 = lapack.spotrf(A.astype(np.float32), lower=1)
    _, info64 = lapack.dpotrf(A, lower=1)
    assert info64 == 0
    assert info32 > 0
