"""Distance matrices: drop-ins for fml/math/distance.py.

* ``manhattan_distance``, ``l2_distance``, ``p_distance`` (distance.py:58-117
  -> fdistance.f90): ``A`` (d, na), ``B`` (d, nb) with descriptors as
  columns; D (na, nb), Fortran-ordered like the reference's ``empty(...,
  order='F')`` (``fmlb_distance_matrix_f64``).
* ``get_l2_distance_arad`` (distance.py:120-189 -> atomic_arad_l2_distance_all,
  farad.f90:452-600): the l2 distance of every atom pair of two molecule
  sets, computed by the same FP64 atom-pair core as the ARAD kernels
  (``fmlb_arad_distances``).
"""

import numpy as np
import torch

from . import _lib
from ._tensors import device, is_torch, to_device, to_output, workspace
from .kernels import _descriptor_rows, _ptp_arrays


def _check_pair(A, B):
    if len(A.shape) != 2 or len(B.shape) != 2:
        raise ValueError('expected matrices of dimension=2')
    if B.shape[0] != A.shape[0]:
        raise ValueError('expected matrices containing vectors of same size')


def _distance(kind, A, B, p_int=0, p_real=0.0):
    a, as_np = _descriptor_rows(A)
    b = a if B is A else _descriptor_rows(B)[0]
    na, d = a.shape
    nb = b.shape[0]
    D = torch.empty((na, nb), dtype=torch.float64, device=a.device)
    _lib.call("fmlb_distance_matrix_f64", kind, _lib.ptr(a), na, d, _lib.ptr(b), nb, d, d,
              int(p_int), float(p_real), _lib.ptr(D), nb, _lib.stream_handle())
    if as_np and not is_torch(B):
        return np.asfortranarray(D.cpu().numpy())
    return D


def manhattan_distance(A, B):
    """fmanhattan_distance, fdistance.f90:23-46: D[j, i] = sum |A[:, j] - B[:, i]|."""
    _check_pair(A, B)
    return _distance(0, A, B)


def l2_distance(A, B):
    """fl2_distance, fdistance.f90:49-80: D[j, i] = ||A[:, j] - B[:, i]||_2."""
    _check_pair(A, B)
    return _distance(1, A, B)


def p_distance(A, B, p=2):
    """fdistance.f90:83-155: (sum (A[:, j] - B[:, i])**p)**(1/p); an int p of 2
    is l2_distance, another int p the integer form, a float p the real form,
    anything else ValueError (distance.py:92-117)."""
    _check_pair(A, B)
    if type(p) == type(1):
        if p == 2:
            return _distance(1, A, B)
        return _distance(2, A, B, p_int=p)
    elif type(p) == type(1.0):
        return _distance(3, A, B, p_real=p)
    raise ValueError('expected exponent of integer or float type')


def get_l2_distance_arad(X1, X2, Z1, Z2, width=0.2, cut_distance=6.0, r_width=1.0,
                         c_width=0.5):
    """D (nm1, nm2, amax, amax) float64; zero past each molecule's atoms."""
    amax = X1.shape[1]
    # the reference's argument checks, distance.py:145-156
    assert X1.shape[3] == amax, "ERROR: Check ARAD decriptor sizes! code = 1"
    assert X2.shape[1] == amax, "ERROR: Check ARAD decriptor sizes! code = 2"
    assert X2.shape[3] == amax, "ERROR: Check ARAD decriptor sizes! code = 3"
    nm1, nm2 = len(Z1), len(Z2)
    assert X1.shape[0] == nm1, "ERROR: Check ARAD decriptor sizes! code = 4"
    assert X2.shape[0] == nm2, "ERROR: Check ARAD decriptor sizes! code = 5"
    x1, as_np = to_device(X1, torch.float64)
    x2, _ = to_device(X2, torch.float64)
    z1p, n1 = _ptp_arrays(Z1, amax)
    z2p, n2 = _ptp_arrays(Z2, amax)
    z1, _ = to_device(z1p, torch.float64)
    z2, _ = to_device(z2p, torch.float64)
    n1d, _ = to_device(n1, torch.int32)
    n2d, _ = to_device(n2, torch.int32)
    D = torch.empty((nm1, nm2, amax, amax), dtype=torch.float64, device=device())
    ws = workspace(_lib.load().fmlb_arad_workspace_bytes(nm1, nm2, amax, 0))
    _lib.call("fmlb_arad_distances", _lib.ptr(x1), _lib.ptr(z1), _lib.ptr(n1d), nm1,
              _lib.ptr(x2), _lib.ptr(z2), _lib.ptr(n2d), nm2, amax, float(width),
              float(cut_distance), float(r_width), float(c_width), _lib.ptr(D), _lib.ptr(ws),
              ws.numel(), _lib.stream_handle())
    return to_output(D, as_np)
