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


def _blocked_cholesky(A, W, nslices):
    """Right-looking blocked Cholesky whose trailing updates are the int8
    (Ozaki) emulation with ``nslices`` digit planes (0: exact FP64 products),
    diagonal blocks and panel solves in FP64 - the structure of
    fmlb_potrf_ozaki_f64. None on breakdown."""
    import scipy.linalg as sla
    import ozaki_emulation as emu
    L = np.tril(A).copy()
    n = len(A)
    for K0 in range(0, n, W):
        K1 = min(K0 + W, n)
        try:
            L[K0:K1, K0:K1] = np.linalg.cholesky(L[K0:K1, K0:K1])
        except np.linalg.LinAlgError:
            return None
        if K1 < n:
            L[K1:, K0:K1] = sla.solve_triangular(L[K0:K1, K0:K1], L[K1:, K0:K1].T, lower=True).T
            P = L[K1:, K0:K1]
            L[K1:, K1:] -= np.tril(P @ P.T if nslices == 0 else emu.product(P, nslices))
    return np.tril(L)


@pytest.mark.parametrize("sigma", [100.0, 1600.0])
def test_ozaki_slices_needed_for_fp64_refined_accuracy(oracle_mod, cm_kernel_inputs, sigma):
    """Why fmlb_potrf_ozaki_f64 defaults to 6 digit planes (8 bits each): on
    these kernels at lambda = 1e-8 a factor from 6 planes, refined three times
    with FP64 residuals, reaches the residual of the FP64 factor refined the
    same way, while 4 planes leave it orders of magnitude above (or break
    down)."""
    import scipy.linalg as sla
    X = cm_kernel_inputs
    A = oracle_mod.gaussian_kernel(X.T, X.T, sigma) + 1e-8 * np.eye(len(X))
    y = np.random.default_rng(0).standard_normal(len(X))

    def refined_residual(L):
        def solve(v):
            return sla.solve_triangular(L.T, sla.solve_triangular(L, v, lower=True), lower=False)
        x = solve(y)
        for _ in range(3):
            x = x + solve(y - A @ x)
        return np.linalg.norm(y - A @ x) / np.linalg.norm(y)

    r64 = refined_residual(_blocked_cholesky(A, 256, 0))
    L6 = _blocked_cholesky(A, 256, 6)
    assert L6 is not None
    assert refined_residual(L6) <= 4 * r64
    L4 = _blocked_cholesky(A, 256, 4)
    assert L4 is None or refined_residual(L4) > 100 * r64


def _pcg_iterations(A, L, y, tol=1e-10, cap=3000):
    """Preconditioned CG on A x = y with M^-1 = (L L^T)^-1, L applied in FP64;
    iterations until the recurrence residual is below tol * ||y||."""
    import scipy.linalg as sl
    x = np.zeros(len(y))
    r = y.copy()
    z = sl.cho_solve((L, True), r)
    p = z.copy()
    rz = r @ z
    ny = np.linalg.norm(y)
    it = 0
    while np.linalg.norm(r) > tol * ny and it < cap:
        Ap = A @ p
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        z = sl.cho_solve((L, True), r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
    return it


@pytest.mark.parametrize("sigma,min_between,min_iters", [(400.0, 100, 150), (1600.0, 300, 500)])
def test_shifted_fp32_factor_is_a_weak_preconditioner(oracle_mod, cm_kernel_inputs, sigma,
                                                      min_between, min_iters):
    """The route around the FP32 breakdown: factor fl32(K + delta I) in FP32
    with the smallest shift delta = 10^e lambda_max that spotrf accepts, and
    use that factor to precondition CG on K + lambda I (FP64, lambda = 1e-8).
    Every eigenvalue of K between lambda and delta is left unpreconditioned,
    and at N = 1024 there are hundreds of them; PCG then needs hundreds of
    iterations, each a full pass over K, to reach a 1e-10 residual (measured
    295 at sigma 400, 1028 at sigma 1600), where the int8-emulated FP64 factor
    needs two refinement steps."""
    X = cm_kernel_inputs
    K = oracle_mod.gaussian_kernel(X.T, X.T, sigma)
    n, lam = len(K), 1e-8
    ev = np.linalg.eigvalsh(K)
    for e in range(-10, 1):
        delta = 10.0 ** e * ev[-1]
        L32, info = lapack.spotrf((K + delta * np.eye(n)).astype(np.float32), lower=1)
        if info == 0:
            break
    assert info == 0
    between = int(np.sum((ev > lam) & (ev < delta)))
    y = synthetic.generate(1024, nmax=29, seed=2).energies
    iters = _pcg_iterations(K + lam * np.eye(n), np.tril(L32).astype(np.float64), y)
    assert between >= min_between
    assert iters >= min_iters
