"""Batched descriptor generation on the GPU (one launch per batch).

* ``generate_coulomb_matrices`` — sorted Coulomb matrices, the batched form
  of ``fgenerate_coulomb_matrix`` (fml/representations/frepresentations.f90:23-110).
* ``generate_unsorted_coulomb_matrices`` — the same matrix in the input atom
  order (``fgenerate_unsorted_coulomb_matrix``, frepresentations.f90:112-202).
* ``generate_local_coulomb_matrices`` — one Coulomb matrix per atom, the
  batched form of ``fgenerate_local_coulomb_matrix`` (kind "local",
  frepresentations.f90:204-294) and ``fgenerate_atomic_coulomb_matrix``
  (kind "atomic", frepresentations.f90:297-390).
* ``generate_arad_descriptors`` — ARAD descriptors, the batched form of
  ``ARAD.describe`` (fml/arad.py:70-145).

Molecules are passed packed and ragged: ``charges`` (total_atoms,),
``coords`` (total_atoms, 3), ``offsets`` (nmol + 1,).
"""

import numpy as np
import torch

from . import _lib
from ._tensors import device, is_torch, to_device, to_output
from .data import PTP_ROW


def _numel(x):
    return int(x.numel()) if is_torch(x) else int(np.size(x))


def _check_offsets(offsets, size, what, charges=None, coords=None):
    off = offsets.cpu().numpy() if is_torch(offsets) else np.asarray(offsets)
    if off.ndim != 1 or len(off) < 1:
        raise ValueError("%s: offsets must be a 1-D array of nmol + 1 entries" % what)
    if off[0] < 0:
        raise ValueError("%s: offsets must start at 0 or above" % what)
    if charges is not None and (off[-1] > len(charges) or off[-1] * 3 > _numel(coords)):
        raise ValueError("%s: offsets reach atom %d, past the %d charges / %d coordinates"
                         % (what, int(off[-1]), len(charges), _numel(coords) // 3))
    counts = np.diff(off)
    if (counts < 0).any():
        raise ValueError("%s: offsets must be non-decreasing" % what)
    if len(counts) and counts.max() > size:
        # frepresentations.f90:45-49 stops the process on a size mismatch;
        # here it is an exception
        raise ValueError("%s: a molecule has %d atoms, more than size=%d"
                         % (what, int(counts.max()), size))
    return len(counts)


def generate_coulomb_matrices(charges, coords, offsets, size=23, return_order=False,
                              float32_ld=None):
    """Sorted Coulomb matrices, (nmol, size*(size+1)/2) float64.

    ``return_order`` also returns the (nmol, size) sorted atom order (-1 padded).
    ``float32_ld`` additionally returns a float32 copy with that row stride
    (zero-padded), for the mixed-precision kernels.
    """
    nmol = _check_offsets(offsets, size, "generate_coulomb_matrices", charges, coords)
    L = size * (size + 1) // 2
    z, as_np = to_device(charges, torch.float64)
    r, _ = to_device(coords, torch.float64)
    off, _ = to_device(offsets, torch.int32)
    dev = device()
    cm = torch.empty((nmol, L), dtype=torch.float64, device=dev)
    order = torch.empty((nmol, size), dtype=torch.int32, device=dev) if return_order else None
    cm32 = None
    if float32_ld is not None:
        if float32_ld < L:
            raise ValueError("float32_ld must be >= %d" % L)
        cm32 = torch.empty((nmol, float32_ld), dtype=torch.float32, device=dev)
    _lib.call("fmlb_coulomb_matrices", _lib.ptr(z), _lib.ptr(r), _lib.ptr(off), nmol, size,
              _lib.ptr(cm), L, _lib.ptr(cm32), float32_ld or 0, _lib.ptr(order), None,
              _lib.stream_handle())
    out = [to_output(cm, as_np)]
    if return_order:
        out.append(to_output(order, as_np))
    if cm32 is not None:
        out.append(cm32)
    return out[0] if len(out) == 1 else tuple(out)


def generate_unsorted_coulomb_matrices(charges, coords, offsets, size=23):
    """Unsorted Coulomb matrices, (nmol, size*(size+1)/2) float64: the packed
    lower triangle in the input atom order (fgenerate_unsorted_coulomb_matrix,
    frepresentations.f90:112-202)."""
    nmol = _check_offsets(offsets, size, "generate_unsorted_coulomb_matrices", charges, coords)
    if size > 255:
        raise ValueError("generate_unsorted_coulomb_matrices: size > 255 is not supported")
    L = size * (size + 1) // 2
    z, as_np = to_device(charges, torch.float64)
    r, _ = to_device(coords, torch.float64)
    off, _ = to_device(offsets, torch.int32)
    cm = torch.empty((nmol, L), dtype=torch.float64, device=device())
    _lib.call("fmlb_unsorted_coulomb_matrices", _lib.ptr(z), _lib.ptr(r), _lib.ptr(off), nmol,
              size, _lib.ptr(cm), L, None, _lib.stream_handle())
    return to_output(cm, as_np)


LOCAL_CM_KINDS = {"local": 0, "atomic": 1}


def generate_local_coulomb_matrices(charges, coords, offsets, size=23, kind="local"):
    """Per-atom Coulomb matrices, (total_atoms, size*(size+1)/2) float64.

    Row ``offsets[m] + k`` is the packed lower triangle for central atom k of
    molecule m: k first and the rest by descending row norm ("local"), or
    every atom by ascending distance to k ("atomic").
    """
    if kind not in LOCAL_CM_KINDS:
        raise ValueError("kind must be 'local' or 'atomic'")
    nmol = _check_offsets(offsets, size, "generate_local_coulomb_matrices", charges, coords)
    if size > 255:
        raise ValueError("generate_local_coulomb_matrices: size > 255 is not supported")
    L = size * (size + 1) // 2
    z, as_np = to_device(charges, torch.float64)
    r, _ = to_device(coords, torch.float64)
    off, _ = to_device(offsets, torch.int32)
    natoms = int((offsets.cpu().numpy() if is_torch(offsets) else np.asarray(offsets))[-1])
    cm = torch.empty((natoms, L), dtype=torch.float64, device=device())
    _lib.call("fmlb_local_coulomb_matrices", _lib.ptr(z), _lib.ptr(r), _lib.ptr(off), nmol, size,
              LOCAL_CM_KINDS[kind], _lib.ptr(cm), L, None, _lib.stream_handle())
    return to_output(cm, as_np)


def generate_arad_descriptors(charges, coords, offsets, size=23, cut=5.0):
    """ARAD descriptors, (nmol, size, 5, size) float64."""
    nmol = _check_offsets(offsets, size, "generate_arad_descriptors", charges, coords)
    if size > 128:
        raise ValueError("generate_arad_descriptors: size > 128 is not supported")
    zc = charges.cpu().numpy() if is_torch(charges) else np.asarray(charges)
    zi = np.asarray(zc, dtype=np.int64)
    if len(zi):
        bad = (zi < 0) | (zi > 127) | (zi != np.asarray(zc))
        bad |= PTP_ROW[np.clip(zi, 0, 127)] < 0
        if bad.any():  # the reference's PTP dict lookup (fml/arad.py:98) raises KeyError
            raise KeyError(zc[np.nonzero(bad)[0][0]])
    z, as_np = to_device(charges, torch.float64)
    r, _ = to_device(coords, torch.float64)
    off, _ = to_device(offsets, torch.int32)
    out = torch.empty((nmol, size, 5, size), dtype=torch.float64, device=device())
    _lib.call("fmlb_arad_descriptors", _lib.ptr(z), _lib.ptr(r), _lib.ptr(off), nmol, size,
              float(cut), _lib.ptr(out), None, _lib.stream_handle())
    return to_output(out, as_np)
