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


def potrf(Ad, n):
    """In-place FP64 factorisation of a device (n, n) tensor; returns (work, info)."""
    work = workspace(_lib.load().fmlb_potrf_workspace_bytes(n))
    info = torch.zeros(1, dtype=torch.int32, device=Ad.device)
    _lib.call("fmlb_potrf_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(work), _lib.ptr(info),
              _lib.stream_handle())
    return work, info


def potrs(Ad, n, work, x):
    _lib.call("fmlb_potrs_f64", _lib.ptr(Ad), Ad.stride(0), n, _lib.ptr(work), _lib.ptr(x),
              _lib.stream_handle())


def cho_solve(A, y, strict=False, refine=0, return_residuals=False):
    """Solve A x = y for symmetric positive-definite A.

    ``refine`` > 0 adds that many FP64 iterative-refinement steps on the
    device (r = y - A x with A kept unfactored, x += solve(r));
    ``return_residuals`` also returns ||y - A x||_2 before each step and
    after the last (``refine`` + 1 values; the plain solve's residual for
    ``refine=0``). Both are extensions: the reference solves once.
    """
    if len(A.shape) != 2 or A.shape[0] != A.shape[1]:
        raise ValueError('expected square matrix')
    if len(y.shape) != 1 or y.shape[0] != A.shape[1]:
        raise ValueError('expected matrix and vector of same stride size')
    n = A.shape[0]
    if refine < 0:
        raise ValueError("refine must be >= 0")
    Ad, as_np = _upper_as_rowmajor_lower(A)
    x, _ = to_device(y, torch.float64)
    x = x.clone()
    keep = refine > 0 or return_residuals
    if keep:  # the unfactored matrix, both triangles, for the FP64 residual
        yd = x.clone()
        Kf = Ad.clone()
        _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Kf), Kf.stride(0), n,
                  _lib.stream_handle())
    work, info = potrf(Ad, n)
    code = int(info.item())
    if code > 0:
        msg = "WARNING: Cholesky decomposition DPOTRF() exited with error code: %d" % code
        if strict:
            raise np.linalg.LinAlgError(msg)
        warnings.warn(msg, CholeskyWarning, stacklevel=2)
    potrs(Ad, n, work, x)
    if not keep:
        return to_output(x, as_np or not is_torch(y))
    lib = _lib.load()
    scratch = torch.empty(lib.fmlb_krr_refine_scratch_doubles(n), dtype=torch.float64,
                          device=Ad.device)
    resid = torch.empty(refine + 1, dtype=torch.float64, device=Ad.device)
    _lib.call("fmlb_krr_refine_f64", _lib.ptr(Kf), Kf.stride(0), n, 0.0, _lib.ptr(Ad),
              Ad.stride(0), _lib.ptr(work), _lib.ptr(yd), _lib.ptr(x), int(refine),
              _lib.ptr(resid), _lib.ptr(scratch), _lib.stream_handle())
    out = to_output(x, as_np or not is_torch(y))
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
