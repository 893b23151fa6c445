"""``cho_solve`` / ``cho_invert``: drop-ins for fml/math/cho_solve.py:27-58.

Solves ``A x = y`` by a Cholesky factorisation on the GPU (hand-written
blocked FP64 factor + triangular solves, the replacement for the LAPACK
``dpotrf('U')`` / ``dpotrs('U')`` calls of fcho_solve.f90:35-42).

Behaviour kept from the reference: ``ValueError`` on shape mismatch
(cho_solve.py:47-51); a non-positive pivot emits a warning and the call
returns (fcho_solve.f90:36-38 prints a WARNING and continues); only the
upper triangle of ``A`` (numpy indices ``i <= j``) is read, as dpotrf('U')
reads it. Difference: ``A`` is never modified (with a Fortran-ordered float64
``A`` the reference overwrites its upper triangle with the factor as an f2py
side effect). ``strict=True`` raises ``numpy.linalg.LinAlgError`` instead of
warning.

``cho_invert`` (fcho_solve.f90:49-68, dpotrf('U') then dpotri('U')) returns
what the reference returns: a Fortran-ordered array whose upper triangle
(i <= j) holds inv(A) and whose strict lower triangle is A's, untouched by
LAPACK. The inversion runs on the GPU from the same factor (``fmlb_potri_f64``).
On a non-positive pivot the reference prints its DPOTRF warning and still runs
dpotri on the partial factor; here the warning is the same and the inverse
triangle is NaN (``strict=True`` raises).
"""

import warnings

import numpy as np
import torch

from . import _lib
from ._tensors import device, is_torch, to_device, to_output, workspace


class CholeskyWarning(RuntimeWarning):
    pass


def _upper_as_rowmajor_lower(A):
    """Device copy whose row-major lower triangle is A's upper triangle."""
    if is_torch(A):
        t = A.to(device=device(), dtype=torch.float64)
        return t.t().contiguous(), False
    a = np.asarray(A, dtype=np.float64)
    t, _ = to_device(np.ascontiguousarray(a.T), torch.float64)
    return t, True


def potrf(Ad, n, factor="fp64", slices=6):
    """In-place factorisation of a device (n, n) tensor; returns (work, info).

    factor="fp64": FP64 tensor-core trailing updates (DMMA);
    factor="ozaki": trailing updates on the int8 tensor cores with ``slices``
    8-bit digit planes per entry (the Ozaki scheme), to be followed by
    iterative refinement.
    """
    lib = _lib.load()
    info = torch.zeros(1, dtype=torch.int32, device=Ad.device)
    if factor == "fp64":
        work = workspace(lib.fmlb_potrf_workspace_bytes(n))
        _lib.call("fmlb_potrf_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(work),
                  _lib.ptr(info), _lib.stream_handle())
    elif factor == "ozaki":
        work = workspace(lib.fmlb_potrf_ozaki_workspace_bytes(n, slices))
        _lib.call("fmlb_potrf_ozaki_f64", _lib.ptr(Ad), Ad.stride(0), n, int(slices),
                  _lib.ptr(work), work.numel(), _lib.ptr(info), _lib.stream_handle())
    else:
        raise ValueError("factor must be 'fp64' or 'ozaki'")
    return work, info


def potrs(Ad, n, work, x):
    _lib.call("fmlb_potrs_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(work), _lib.ptr(x),
              _lib.stream_handle())


def _check_info(info, strict):
    code = int(info.item())
    if code == _lib.FMLB_ETIMEDOUT:
        raise _lib.FmlbError(code, "cho_solve: a device-side wait of the factorisation gave up")
    if code > 0:
        msg = "WARNING: Cholesky decomposition DPOTRF() exited with error code: %d" % code
        if strict:
            raise np.linalg.LinAlgError(msg)
        warnings.warn(msg, CholeskyWarning, stacklevel=3)


def cho_solve(A, y, strict=False, refine=None, return_residuals=False, factor="fp64",
              slices=6, residual=None):
    """Solve A x = y for symmetric positive-definite A.

    Extensions (the reference solves once with LAPACK):

    * ``factor="ozaki"`` factors on the int8 tensor cores (``slices`` digit
      planes, 1..8) and refines; ``refine`` then defaults to 2 steps and the
      residual to double-double.
    * ``refine`` > 0 adds that many iterative-refinement steps on the device
      (r = y - A x, x += solve(r)); ``residual="fp64"`` (the default for the
      FP64 factor) forms r in FP64, ``residual="dd"`` in double-double with x
      kept as a double-double pair (past the FP64 residual floor).
    * ``return_residuals`` also returns ||y - A x||_2 before each step and
      after the last (``refine`` + 1 values).
    """
    if len(A.shape) != 2 or A.shape[0] != A.shape[1]:
        raise ValueError('expected square matrix')
    if len(y.shape) != 1 or y.shape[0] != A.shape[1]:
        raise ValueError('expected matrix and vector of same stride size')
    n = A.shape[0]
    if factor not in ("fp64", "ozaki"):
        raise ValueError("factor must be 'fp64' or 'ozaki'")
    if refine is None:
        refine = 2 if factor == "ozaki" else 0
    if residual is None:
        residual = "dd" if factor == "ozaki" else "fp64"
    if refine < 0:
        raise ValueError("refine must be >= 0")
    if residual not in ("fp64", "dd"):
        raise ValueError("residual must be 'fp64' or 'dd'")
    Ad, as_np = _upper_as_rowmajor_lower(A)
    x, _ = to_device(y, torch.float64)
    x = x.clone()
    keep = refine > 0 or return_residuals
    out_np = as_np or not is_torch(y)
    if n == 0:
        return (to_output(x, out_np), np.zeros(refine + 1)) if return_residuals else \
            to_output(x, out_np)
    lib = _lib.load()
    st = _lib.stream_handle()
    if keep and residual == "fp64":  # the unfactored matrix, both triangles
        yd = x.clone()
        Kf = Ad.clone()
        _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Kf), Kf.stride(0), n, st)
    elif keep:  # K stays in the strict upper triangle the factorisation leaves alone
        yd = x.clone()
        _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Ad), Ad.stride(0), n, st)
        diag = torch.empty(n, dtype=torch.float64, device=Ad.device)
        _lib.call("fmlb_get_diagonal_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(diag), st)
    work, info = potrf(Ad, n, factor, slices)
    _check_info(info, strict)
    potrs(Ad, n, work, x)
    if not keep:
        return to_output(x, out_np)
    resid = torch.empty(refine + 1, dtype=torch.float64, device=Ad.device)
    if residual == "fp64":
        scratch = torch.empty(lib.fmlb_krr_refine_scratch_doubles(n), dtype=torch.float64,
                              device=Ad.device)
        _lib.call("fmlb_krr_refine_f64", _lib.ptr(Kf), Kf.stride(0), n, 0.0, _lib.ptr(Ad),
                  Ad.stride(0), _lib.ptr(work), _lib.ptr(yd), _lib.ptr(x), int(refine),
                  _lib.ptr(resid), _lib.ptr(scratch), st)
    else:
        scratch = torch.empty(lib.fmlb_krr_refine_dd_scratch_doubles(n), dtype=torch.float64,
                              device=Ad.device)
        x_lo = torch.zeros_like(x)
        _lib.call("fmlb_krr_refine_dd", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(diag),
                  _lib.ptr(work), _lib.ptr(yd), _lib.ptr(x), _lib.ptr(x_lo), int(refine),
                  _lib.ptr(resid), _lib.ptr(scratch), st)
    out = to_output(x, out_np)
    if return_residuals:
        return out, resid.cpu().numpy()
    return out


def cho_invert(A, strict=False):
    """inv(A) of a symmetric positive-definite A, in the reference's layout."""
    if len(A.shape) != 2 or A.shape[0] != A.shape[1]:
        raise ValueError('expected square matrix')
    n = A.shape[0]
    Ad, as_np = _upper_as_rowmajor_lower(A)
    if n == 0:
        return to_output(Ad, as_np)
    work, info = potrf(Ad, n)
    ldv = n + (n & 1)  # even stride: 16-byte aligned rows for the tensor-core tiles
    V = torch.empty((n, ldv), dtype=torch.float64, device=Ad.device)
    _lib.call("fmlb_potri_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(work), _lib.ptr(V), ldv,
              _lib.ptr(info), _lib.stream_handle())
    del V
    code = int(info.item())
    if code > 0:
        msg = "WARNING: Cholesky decomposition DPOTRF() exited with error code: %d" % code
        if strict:
            raise np.linalg.LinAlgError(msg)
        warnings.warn(msg, CholeskyWarning, stacklevel=2)
        Ad.masked_fill_(torch.ones_like(Ad, dtype=torch.bool).tril(), float("nan"))
    # Ad's lower triangle is inv(A), its strict upper triangle A's strict lower
    # one transposed: Ad is the row-major image of the result's Fortran layout.
    if as_np:
        return Ad.cpu().numpy().T
    return Ad.t()
