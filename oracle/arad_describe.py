"""CPU ORACLE — test infrastructure, not product code.

numpy restatement of the reference's ARAD descriptor, ``ARAD.describe`` in
fml/arad.py:70-145 (molecular, non-periodic path ``cell is None``,
fml/arad.py:89-91). It is pinned against the reference's own ``arad.py``
through the fixtures in tests/golden/ (tests/golden/make_golden.py).

Output layout (fml/arad.py:74): ``(maxMolSize, 5, maxAts)`` float64 with
channel 0 = sorted neighbour distances padded with 1e100 (:93, :138),
channels 1/2 = PTP row / column of each neighbour (:139-140),
channels 3/4 = damped mean cosine / sine of the neighbour angles (:141-142).
"""

import numpy as np

from .ptp import PTP

EPSILON = 100.0 * np.finfo(float).eps  # fml/arad.py:42


def _angles(sp, norms):
    """fml/arad.py:29-33 (getAngle): arccos(sp/norms) where the mask holds."""
    angles = np.zeros(sp.shape)
    mask = np.logical_and(np.abs(sp - norms) > EPSILON, np.abs(norms) > EPSILON)
    with np.errstate(invalid="ignore"):
        angles[mask] = np.arccos(sp[mask] / norms[mask])
    return angles


def describe(coords, charges, size=30, cut=5.0):
    coords = np.asarray(coords, dtype=np.float64)
    charges = np.asarray(charges)
    L = len(coords)
    M = np.zeros((size, 5, size))
    M[:, 0, :] = 1e100
    oc = np.asarray([PTP[int(o)] for o in charges]).reshape(-1, 2)
    for i in range(L):
        cd = -coords[i] + coords  # :97
        sp = np.sum(cd[:, None] * cd[None, :], axis=2)  # :101
        d1 = np.sqrt(np.sum(cd ** 2, axis=1))  # :102
        d2 = d1[:, None] * d1[None, :]  # :103
        ang = _angles(sp, d2)
        damp = 1.0 - np.sin(np.pi * d1[None, :] / (2.0 * cut))  # :107-108
        cos_a = np.cos(ang) * damp
        sin_a = np.sin(ang) * damp
        # :110 with numpy's default sort, as the reference calls it: its order
        # of exactly equidistant neighbours (not stable above 16 entries) is
        # part of the descriptor (channels 1-4)
        order = np.argsort(d1)
        d1s = d1[order]
        keep = np.nonzero(d1s < cut)[0]  # :121
        sel = order[keep]
        d1k = d1s[keep]
        cos_k = cos_a[np.ix_(sel, sel)]
        sin_k = sin_a[np.ix_(sel, sel)]
        norm = np.sum(1.0 - np.sin(np.pi * d1k[None, :] / (2.0 * cut)))  # :137
        n = len(d1k)
        M[i, 0, :n] = d1k
        M[i, 1, :n] = oc[sel, 0]
        M[i, 2, :n] = oc[sel, 1]
        M[i, 3, :n] = np.sum(cos_k, axis=1) / norm
        M[i, 4, :n] = np.sum(sin_k, axis=1) / norm
    return M
