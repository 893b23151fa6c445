"""numpy statement of the int8 (Ozaki) trailing update, for tests only.

It follows the arithmetic of fml_b200/csrc/ozaki_f64.cu step by step: the
per-row exponent from frexp of the row maximum, base-256 digits by repeated
flooring (a signed leading digit, unsigned lower ones), the exact integer
products summed per diagonal (float64 holds them exactly), the Horner
combination in 256 with one rounding per step (what the kernel's FMA does),
and the power-of-two scaling. The kernel must match it bit for bit.
"""

import numpy as np


def split(P, nslices):
    """(digits list of (m, k) integer-valued float64, exponents (m,))."""
    P = np.asarray(P, dtype=np.float64)
    mx = np.abs(P).max(axis=1) if P.shape[1] else np.zeros(P.shape[0])
    e = np.where(mx > 0, np.frexp(mx)[1], 0).astype(np.int64)
    x = np.ldexp(P, -(e[:, None] + 1))
    digits = []
    for _ in range(nslices):
        x = x * 256.0
        d = np.floor(x)
        x = x - d
        digits.append(d)
    return digits, e


def product(P, nslices):
    """The emulated P P^T (m, m)."""
    d, e = split(P, nslices)
    m = P.shape[0]
    acc = np.zeros((m, m))
    for q in range(nslices):
        Dq = np.zeros((m, m))
        for a in range(q + 1):
            Dq += d[a] @ d[q - a].T
        acc = acc * 256.0 + Dq
    return np.ldexp(acc, e[:, None] + e[None, :] + 2 - 8 * (nslices + 1))


def syrk_lower(C, P, nslices, strip_cols=0):
    """C - P P^T on the lower triangle (first strip_cols columns if > 0)."""
    C = np.array(C, dtype=np.float64, copy=True)
    m = C.shape[0]
    V = product(P, nslices)
    mask = np.tril(np.ones((m, m), dtype=bool))
    if strip_cols > 0:
        mask[:, strip_cols:] = False
    C[mask] -= V[mask]
    return C


def error_bound(P, nslices):
    """Entry-wise bound on |emulated - exact| P P^T: k (s + 3) 2^(e_r + e_c + 2 - 8 s)."""
    _, e = split(P, nslices)
    k = P.shape[1]
    return k * (nslices + 3) * np.ldexp(1.0, e[:, None] + e[None, :] + 2 - 8 * nslices)
