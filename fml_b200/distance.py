"""ARAD distance matrices: drop-in for ``get_l2_distance_arad``
(fml/math/distance.py:120-189 -> atomic_arad_l2_distance_all,
fml/math/farad.f90:452-600).

The l2 distance of every atom pair of two molecule sets, computed by the
same FP64 atom-pair core as the ARAD kernels (``fmlb_arad_distances``).
"""

import torch

from . import _lib
from ._tensors import device, to_device, to_output, workspace
from .kernels import _ptp_arrays


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
