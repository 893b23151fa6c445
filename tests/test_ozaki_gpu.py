"""The int8 tensor-core (Ozaki) emulation of the FP64 trailing update and the
factorisation built on it, through the C ABI.

* fmlb_syrk_lower_ozaki against a numpy statement of the same arithmetic
  (tests/ozaki_emulation.py): bit-exact; against the exact FP64 product:
  within the scheme's bound k (s + 3) 2^(e_r + e_c + 2 - 8 s) per entry.
* fmlb_potrf_ozaki_f64 + double-double refinement against LAPACK
  (fcho_solve.f90:35-42 calls dpotrf/dpotrs) at n = 16500, which crosses the
  1024-wide outer panels, kappa ~ 1e11: refined relative residual below
  1e-10, fitted values A x equal to LAPACK's to 1e-8 of |y|.
* fmlb_krr_refine_dd at condition number ~1e10 against the residual computed
  exactly in integer arithmetic.
* A wait that runs out (test hook: no copies issued) reports FMLB_ETIMEDOUT
  and leaves the context usable.
"""

from fractions import Fraction

import numpy as np
import pytest
import scipy.linalg as sla
import torch

import fml_b200
from fml_b200 import _lib

import ozaki_emulation as emu

pytestmark = pytest.mark.gpu


def _syrk_gpu(C, P, nslices, strip_cols=0):
    lib = _lib.load()
    m, k = P.shape
    Cd = torch.from_numpy(np.ascontiguousarray(C)).cuda()
    Pd = torch.from_numpy(np.ascontiguousarray(P)).cuda()
    ws = torch.empty(lib.fmlb_syrk_ozaki_workspace_bytes(m, k, nslices), dtype=torch.uint8,
                     device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("fmlb_syrk_lower_ozaki", _lib.ptr(Cd), m, m, _lib.ptr(Pd), k, k, strip_cols,
              nslices, _lib.ptr(ws), ws.numel(), _lib.ptr(info), _lib.stream_handle())
    torch.cuda.synchronize()
    return Cd.cpu().numpy(), int(info.item())


def _panel(rng, m, k):
    """Rows of very different scales, a zero row, tiny entries inside rows."""
    P = rng.standard_normal((m, k)) * np.ldexp(1.0, rng.integers(-20, 21, size=m))[:, None]
    P[m // 3] = 0.0
    P[:, ::7] *= 1e-9
    return P


@pytest.mark.parametrize("m,k,s,strip", [(700, 1024, 6, 0), (300, 256, 8, 0), (517, 96, 3, 0),
                                         (1000, 512, 7, 256), (5, 64, 1, 0), (130, 4096, 6, 0),
                                         (1, 32, 8, 0)])
def test_syrk_ozaki_bit_exact_vs_emulation(m, k, s, strip):
    rng = np.random.default_rng(m + k + s)
    P = _panel(rng, m, k)
    C = rng.standard_normal((m, m))
    out, info = _syrk_gpu(C, P, s, strip)
    assert info == 0
    ref = emu.syrk_lower(C, P, s, strip)
    np.testing.assert_array_equal(out, ref)
    exact = C - P @ P.T
    mask = np.tril(np.ones((m, m), dtype=bool))
    if strip:
        mask[:, strip:] = False
    err = np.abs(out - exact)[mask]
    # plus the FP64 rounding of the combination and of numpy's own product
    bound = (emu.error_bound(P, s) + 1e-14 * np.abs(P) @ np.abs(P).T + 1e-15 * np.abs(C))[mask]
    assert (err <= bound).all()
    np.testing.assert_array_equal(out[~mask], C[~mask])  # untouched outside the update


def test_syrk_ozaki_tiny_negative_entries():
    """Rows with one dominant entry and tiny negative ones (the shape of a
    Cholesky factor of a nearly diagonal kernel matrix): a tiny negative
    value has leading digit -1 and a remainder that rounds to 1.0, which must
    be carried instead of overflowing the next digit. Bit-exact against the
    emulation and within the scheme's bound of the exact product."""
    rng = np.random.default_rng(8)
    m, k = 400, 1024
    P = -np.abs(rng.standard_normal((m, k))) * np.ldexp(1.0, rng.integers(-80, -40, size=(m, k)))
    P[np.arange(m), rng.integers(0, k, size=m)] = rng.uniform(0.5, 0.99, size=m)
    P[:, 7] = -1e-300
    C = np.eye(m) + 1e-3 * rng.standard_normal((m, m))
    for s in (6, 7):
        out, info = _syrk_gpu(C, P, s)
        assert info == 0
        np.testing.assert_array_equal(out, emu.syrk_lower(C, P, s))
        low = np.tril(np.ones((m, m), dtype=bool))
        err = np.abs(out - (C - P @ P.T))[low]
        bound = (emu.error_bound(P, s) + 1e-14 * np.abs(P) @ np.abs(P).T + 1e-15 * np.abs(C))[low]
        assert (err <= bound).all()


def test_syrk_ozaki_nonfinite_rows_propagate():
    rng = np.random.default_rng(3)
    P = rng.standard_normal((200, 128))
    P[17, 5] = np.nan
    C = rng.standard_normal((200, 200))
    out, info = _syrk_gpu(C, P, 7)
    assert info == 0
    assert np.isnan(out[17, :18]).all() and np.isnan(out[17:, 17]).all()
    low = np.tril(np.ones((200, 200), dtype=bool))
    low[17, :] = False
    low[:, 17] = False
    assert np.isfinite(out[low]).all()


def test_syrk_ozaki_wait_timeout_reports_and_recovers():
    rng = np.random.default_rng(4)
    P = rng.standard_normal((300, 256))
    C = rng.standard_normal((300, 300))
    try:
        _lib.call("fmlb_tc_test_hooks", 20000, 1)  # ~10 us waits, no copies issued
        out, info = _syrk_gpu(C, P, 7)
    finally:
        _lib.call("fmlb_tc_test_hooks", 0, 0)
    assert info == _lib.FMLB_ETIMEDOUT
    np.testing.assert_array_equal(out, C)  # nothing was written
    out, info = _syrk_gpu(C, P, 7)
    assert info == 0
    np.testing.assert_array_equal(out, emu.syrk_lower(C, P, 7))


@pytest.fixture(scope="module")
def cm_gaussian_16500():
    """K + 1e-8 I for 16500 sorted CMs (nmax 29) at sigma 400: kappa ~ 1e11."""
    from fml_b200 import synthetic
    b = synthetic.generate(16500, nmax=29, seed=2)
    X = fml_b200.generate_coulomb_matrices(b.charges, b.coords, b.offsets, size=29)
    K = fml_b200.gaussian_kernel(X.T, X.T, 400.0)
    K[np.diag_indices_from(K)] += 1e-8
    return K, b.energies


@pytest.mark.parametrize("slices", [6, 7])
def test_potrf_ozaki_refined_solve_vs_lapack(cm_gaussian_16500, slices):
    A, y = cm_gaussian_16500
    x, res = fml_b200.cho_solve(A, y, factor="ozaki", slices=slices, refine=4,
                                return_residuals=True)
    c, info = sla.lapack.dpotrf(A, lower=0, clean=0)
    assert info == 0
    xr, _ = sla.lapack.dpotrs(c, y, lower=0)
    ny = np.linalg.norm(y)
    assert res[-1] / ny < 1e-10, res / ny
    # kappa ~ 1e11: LAPACK's own x carries ~kappa u ~ 1e-5 relative error, so
    # the solutions are compared through what they fit, A x (to 1e-8 of |y|),
    # and loosely as vectors
    assert np.linalg.norm(A @ x - A @ xr) <= 1e-8 * ny
    assert np.linalg.norm(x - xr) <= 1e-3 * np.linalg.norm(xr)


def test_potrf_ozaki_factor_close_to_fp64_factor_well_conditioned():
    rng = np.random.default_rng(9)
    n = 3000  # outer panels of 256 columns
    M = rng.standard_normal((n, n))
    A = M @ M.T / n + np.eye(n)
    Ad = torch.from_numpy(A).cuda()
    from fml_b200.cho_solve import potrf
    work, info = potrf(Ad, n, "ozaki", 8)
    assert int(info.item()) == 0
    L = torch.tril(Ad).cpu().numpy()
    Lr = np.linalg.cholesky(A)
    assert np.abs(L - Lr).max() <= 1e-12 * np.abs(Lr).max()


def _exact_residual_norm(A, x_parts, y):
    """||y - A (sum of x_parts)||_2 / ||y||_2 with the residual formed exactly."""
    n = len(y)
    xs = [sum(Fraction(float(p[j])) for p in x_parts) for j in range(n)]
    r2 = 0.0
    for i in range(n):
        s = Fraction(float(y[i]))
        row = A[i]
        for j in range(n):
            if row[j] != 0.0:
                s -= Fraction(float(row[j])) * xs[j]
        r2 += float(s) ** 2
    return np.sqrt(r2) / np.linalg.norm(y)


@pytest.mark.parametrize("factor", ["fp64", "ozaki"])
def test_refine_dd_past_fp64_floor_exact_residual(factor):
    rng = np.random.default_rng(21)
    n = 160
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.logspace(0, -10, n)
    A = (Q * lam) @ Q.T
    A = (A + A.T) / 2
    y = rng.standard_normal(n)
    # FP64 refinement stalls at its floor; double-double goes below 1e-10
    _, res64 = fml_b200.cho_solve(A, y, refine=4, return_residuals=True, factor="fp64",
                                  residual="fp64")
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Ad), n, n, _lib.stream_handle())
    diag = torch.empty(n, dtype=torch.float64, device="cuda")
    _lib.call("fmlb_get_diagonal_f64", _lib.ptr(Ad), n, n, _lib.ptr(diag), _lib.stream_handle())
    from fml_b200.cho_solve import potrf, potrs
    work, info = potrf(Ad, n, factor, 8)
    assert int(info.item()) == 0
    x = torch.from_numpy(y.copy()).cuda()
    potrs(Ad, n, work, x)
    x_lo = torch.zeros_like(x)
    yd = torch.from_numpy(y).cuda()
    lib = _lib.load()
    scratch = torch.empty(lib.fmlb_krr_refine_dd_scratch_doubles(n), dtype=torch.float64,
                          device="cuda")
    resid = torch.empty(5, dtype=torch.float64, device="cuda")
    _lib.call("fmlb_krr_refine_dd", _lib.ptr(Ad), n, n, _lib.ptr(diag), _lib.ptr(work),
              _lib.ptr(yd), _lib.ptr(x), _lib.ptr(x_lo), 4, _lib.ptr(resid), _lib.ptr(scratch),
              _lib.stream_handle())
    torch.cuda.synchronize()
    res = resid.cpu().numpy() / np.linalg.norm(y)
    exact = _exact_residual_norm(A, [x.cpu().numpy(), x_lo.cpu().numpy()], y)
    assert exact < 1e-10 and exact < res64[-1] / np.linalg.norm(y)
    # the reported residual is the double-double one rounded to FP64: it
    # matches the exact one up to the double-double evaluation error
    # (~n 2^-104 |A| |x| / |y| ~ 1e-19 here)
    assert abs(res[-1] - exact) <= 0.05 * exact + 1e-18
