"""Element tables used by the host side of the hot path.

``NUCLEAR_CHARGE`` maps element symbols to nuclear charges for the XYZ reader
(reference: fml/data.py:23-137 — the same symbol set, including the two
placeholder symbols ``Uuq``/``Uuh`` and without Z = 113, 115, 117, 118).

``PTP`` gives the periodic-table position (period row, group column) used by
the ARAD descriptor channels 1-2 and by the ARAD kernel's stoichiometric factor
(reference: fml/arad.py:43-68 and fml/kernels/kernels.py:41-66; both hold the
same table). The table is rebuilt here from its layout rules; two entries of
the reference table are irregular and are kept as the reference has them:
Z = 101 appears twice in the reference dict literal, so its last value
(7, 32) is the one in force, and Z = 102 maps to (7, 14).
"""

import numpy as np

_SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn "
    "Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce "
    "Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn "
    "Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf Db Sg Bh Hs Mt Ds Rg Cn"
).split()

NUCLEAR_CHARGE = {sym: z for z, sym in enumerate(_SYMBOLS, start=1)}
NUCLEAR_CHARGE["Uuq"] = 114
NUCLEAR_CHARGE["Uuh"] = 116


def _build_ptp():
    """Return {Z: [row, col]} following the reference's periodic layout.

    s-block -> columns 1-2, p-block -> 3-8, d-block -> 9-18 (periods 4-5) or
    10-18 (periods 6-7, whose column 9 is taken by the f-block start), and the
    f-block (57-71, 89-103) -> 19-33. He sits in column 8.
    """
    t = {1: [1, 1], 2: [1, 8]}
    for row, first in ((2, 3), (3, 11)):
        t[first] = [row, 1]
        t[first + 1] = [row, 2]
        for k in range(6):
            t[first + 2 + k] = [row, 3 + k]
    for row, s0, d0, p0 in ((4, 19, 21, 31), (5, 37, 39, 49)):
        t[s0] = [row, 1]
        t[s0 + 1] = [row, 2]
        for k in range(10):
            t[d0 + k] = [row, 9 + k]
        for k in range(6):
            t[p0 + k] = [row, 3 + k]
    for row, s0, f0, d0, p0 in ((6, 55, 57, 72, 81), (7, 87, 89, 104, 113)):
        t[s0] = [row, 1]
        t[s0 + 1] = [row, 2]
        for k in range(15):
            t[f0 + k] = [row, 19 + k]
        for k in range(9):
            t[d0 + k] = [row, 10 + k]
        for k in range(6):
            t[p0 + k] = [row, 3 + k]
    # irregular entries of the reference table (see module docstring)
    t[101] = [7, 32]
    t[102] = [7, 14]
    return t


PTP = _build_ptp()

#: dense lookup tables indexed by Z (0 and unknown Z hold -1)
PTP_ROW = np.full(128, -1, dtype=np.int32)
PTP_COL = np.full(128, -1, dtype=np.int32)
for _z, (_r, _c) in PTP.items():
    PTP_ROW[_z] = _r
    PTP_COL[_z] = _c


def ptp_of(charges):
    """Map an array of nuclear charges to an (n, 2) float64 array of PTP.

    Raises KeyError for a charge the table does not hold, as the reference's
    dict lookup does (fml/kernels/kernels.py:276).
    """
    z = np.asarray(charges)
    zi = z.astype(np.int64)
    bad = (zi < 0) | (zi >= 128)
    if bad.any() or (PTP_ROW[np.clip(zi, 0, 127)] < 0).any():
        missing = [int(v) for v in np.unique(zi) if v < 0 or v >= 128 or PTP_ROW[v] < 0]
        raise KeyError(missing[0] if missing else None)
    return np.stack([PTP_ROW[zi], PTP_COL[zi]], axis=-1).astype(np.float64)
