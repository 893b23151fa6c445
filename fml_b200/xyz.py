"""Batched XYZ ingestion: many files -> one packed ragged molecule buffer.

``read_xyz_batch(paths)`` parses every file with the rules of
``Molecule.read_xyz`` (fml/fml.py:109-132) on host threads in libfmlb
(``fmlb_xyz_scan`` / ``fmlb_xyz_parse``) and returns the layout the batched
descriptor calls take: charges (A,), coords (A, 3), offsets (M + 1,). On a
CUDA machine the host arrays are page-locked, and ``to_device=True`` issues
one asynchronous copy per array on the current stream, so ingestion of the
next batch can overlap the descriptors of this one.
"""

import ctypes
import os
from typing import NamedTuple, Optional

import numpy as np
import torch

from . import _lib
from .data import NUCLEAR_CHARGE

_TABLE_SYMBOLS = list(NUCLEAR_CHARGE.keys())
_TABLE_CHARGES = np.array([float(NUCLEAR_CHARGE[s]) for s in _TABLE_SYMBOLS], dtype=np.float64)


class XyzBatch(NamedTuple):
    charges: torch.Tensor          # (A,) float64, host (page-locked on a CUDA machine)
    coords: torch.Tensor           # (A, 3) float64
    offsets: np.ndarray            # (M + 1,) int32
    natoms_declared: np.ndarray    # (M,) int32, line 1 of each file
    symbol_index: torch.Tensor     # (A,) int32 into ``symbols``
    symbols: list                  # element table (NUCLEAR_CHARGE order)
    device_charges: Optional[torch.Tensor] = None
    device_coords: Optional[torch.Tensor] = None
    device_offsets: Optional[torch.Tensor] = None

    def atomtypes(self, m):
        """Element symbols of molecule m (Molecule.atomtypes)."""
        idx = self.symbol_index[self.offsets[m]:self.offsets[m + 1]].tolist()
        return [self.symbols[i] for i in idx]


def _c_strings(items):
    arr = (ctypes.c_char_p * max(len(items), 1))(*items)
    return arr, ctypes.cast(arr, ctypes.c_void_p)


def _np_ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def read_xyz_batch(paths, nthreads=0, to_device=False):
    """Parse ``paths`` into one packed batch (see the module docstring).

    Raises KeyError for an element missing from NUCLEAR_CHARGE (the
    reference's dict lookup) and ValueError for an unreadable file, a bad
    atom count or a coordinate that is not a decimal number. The count and
    the coordinates are read as Python's int() and float() read ASCII text
    (signs, fractions, exponents, inf / infinity / nan in any case, digit-group
    underscores such as "1_0.5"); non-ASCII digits and declared counts outside
    the int32 range raise ValueError.
    """
    enc = [os.fsencode(os.fspath(p)) for p in paths]
    n = len(enc)
    keep_p, parr = _c_strings(enc)
    declared = np.zeros(max(n, 1), dtype=np.int32)
    parsed = np.zeros(max(n, 1), dtype=np.int32)
    _call("fmlb_xyz_scan", parr, n, _np_ptr(declared), _np_ptr(parsed), int(nthreads))
    offsets = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(parsed[:n], out=offsets[1:])
    total = int(offsets[-1])
    pin = torch.cuda.is_available()
    charges = torch.empty(total, dtype=torch.float64, pin_memory=pin)
    coords = torch.empty((total, 3), dtype=torch.float64, pin_memory=pin)
    sym = torch.empty(total, dtype=torch.int32, pin_memory=pin)
    keep_t, tarr = _c_strings([s.encode() for s in _TABLE_SYMBOLS])
    _call("fmlb_xyz_parse", parr, n, _np_ptr(offsets), tarr, _np_ptr(_TABLE_CHARGES),
          len(_TABLE_SYMBOLS), ctypes.c_void_p(charges.data_ptr() if total else 0),
          ctypes.c_void_p(coords.data_ptr() if total else 0),
          ctypes.c_void_p(sym.data_ptr() if total else 0), int(nthreads))
    del keep_p, keep_t
    batch = XyzBatch(charges, coords, offsets, declared[:n].copy(), sym, _TABLE_SYMBOLS)
    if to_device:
        dev = torch.device("cuda", torch.cuda.current_device())
        batch = batch._replace(device_charges=charges.to(dev, non_blocking=True),
                               device_coords=coords.to(dev, non_blocking=True),
                               device_offsets=torch.from_numpy(offsets).to(dev))
    return batch


def _call(name, *args):
    try:
        _lib.call(name, *args)
    except ValueError as e:
        msg = str(e)
        if "unknown element " in msg:  # the reference's NUCLEAR_CHARGE[...] KeyError
            raise KeyError(msg.rsplit("unknown element ", 1)[1]) from None
        raise


def read_xyz_molecules(paths, nthreads=0):
    """``Molecule`` objects for many files in one native pass, each as
    ``Molecule.read_xyz`` (fml/fml.py:109-132) would fill it: ``natoms`` (the
    declared count), ``atomtypes``, ``nuclear_charges`` and ``coordinates``."""
    from .molecule import Molecule
    batch = read_xyz_batch(paths, nthreads=nthreads)
    coords = batch.coords.numpy()
    mols = []
    for m in range(len(batch.offsets) - 1):
        a, b = int(batch.offsets[m]), int(batch.offsets[m + 1])
        mol = Molecule()
        mol.natoms = int(batch.natoms_declared[m])
        mol.atomtypes = batch.atomtypes(m)
        mol.nuclear_charges = [NUCLEAR_CHARGE[t] for t in mol.atomtypes]  # the table's values
        mol.coordinates = coords[a:b].copy()
        mols.append(mol)
    return mols
