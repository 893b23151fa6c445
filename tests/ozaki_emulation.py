"""numpy statement of the int8 (Ozaki) trailing update, for tests only.

It follows the arithmetic of fml_b200/csrc/ozaki_f64.cu step by step: the
per-row exponent from frexp of the row maximum, base-256 digits by repeated
flooring (a signed leading digit; lower digits stored with the zero point
128), the per-row sums of those digits, the exact integer products summed
per diagonal (float64 holds them exactly), the Horner combination in 256
with one rounding per step (what the kernel's FMA does), the zero-point
terms added in the kernel's order, and the power-of-two scaling. The kernel
must match it bit for bit.
"""

import numpy as np


def split(P, nslices, kp=None):
    """(digit planes as integer-valued float64, exponents, zero point c', row sums S)."""
    P = np.asarray(P, dtype=np.float64)
    m, k = P.shape
    kp = k if kp is None else kp
    Pp = np.zeros((m, kp))
    Pp[:, :k] = P
    mx = np.abs(P).max(axis=1) if k else np.zeros(m)
    e = np.where(mx > 0, np.frexp(mx)[1], 0).astype(np.int64)
    x = np.ldexp(Pp, -(e[:, None] + 1))
    digits = []
    for t in range(nslices):
        x = x * 256.0
        d = np.floor(x)
        x = x - d
        up = x >= 1.0  # 1 - |tiny| rounded to 1.0 after a leading -1: carry
        x = np.where(up, x - 1.0, x)
        d = np.where(up, d + 1.0, d)
        digits.append(d - (128.0 if t else 0.0))
    zc = np.ldexp(1.0, -8 * nslices - 1)
    for t in range(2, nslices + 1):
        zc += np.ldexp(128.0, -8 * t)
    S = np.zeros(m)
    for t in range(nslices):
        S = S + np.ldexp(digits[t].sum(axis=1), -8 * (t + 1))
    return digits, e, zc, S


def product(P, nslices, kp=None):
    """The emulated P P^T (m, m)."""
    d, e, zc, S = split(P, nslices, kp)
    m, kk = d[0].shape
    acc = np.zeros((m, m))
    for q in range(nslices):
        Dq = np.zeros((m, m))
        for a in range(q + 1):
            Dq += d[a] @ d[q - a].T
        acc = acc * 256.0 + Dq
    core = (np.ldexp(acc, -8 * (nslices + 1)) + zc * (S[:, None] + S[None, :])) + kk * zc * zc
    return np.ldexp(core, e[:, None] + e[None, :] + 2)


def syrk_lower(C, P, nslices, strip_cols=0):
    """C - P P^T on the lower triangle (first strip_cols columns if > 0); the
    kernel pads k to a multiple of 32 with zeros."""
    C = np.array(C, dtype=np.float64, copy=True)
    m = C.shape[0]
    kp = -(-P.shape[1] // 32) * 32
    V = product(P, nslices, kp)
    mask = np.tril(np.ones((m, m), dtype=bool))
    if strip_cols > 0:
        mask[:, strip_cols:] = False
    C[mask] -= V[mask]
    return C


def error_bound(P, nslices):
    """Entry-wise bound on |emulated - exact| P P^T: k (s + 3) 2^(e_r + e_c + 2 - 8 s)."""
    _, e, _, _ = split(P, nslices)
    k = P.shape[1]
    return k * (nslices + 3) * np.ldexp(1.0, e[:, None] + e[None, :] + 2 - 8 * nslices)
