"""numpy statement of the int8 (Ozaki) trailing update, for tests only.

It follows the arithmetic of fml_b200/csrc/ozaki_f64.cu step by step: the
per-row exponent from frexp of the row maximum, base-256 digits by repeated
flooring (a signed leading digit; lower digits stored with the zero point
128), the per-row sums of those digits, the exact integer products summed
per diagonal (float64 holds them exactly), the Horner combination in 256
with one rounding per step (what the kernel's FMA does) over each pass of
at most four diagonals, the zero-point terms added in the kernel's order,
the power-of-two scaling, and one subtraction from C per pass. The kernel
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


PASS_Q = 4  # diagonals per pass of the kernel (accumulators of 128 TMEM columns)


def product_parts(P, nslices, kp=None):
    """The emulated P P^T as the kernel subtracts it: one (m, m) part per pass.

    Diagonals [0, 4) form the first part and [4, s) the second (s > 4 only);
    each part is a Horner sum in 256 scaled by 256^-(q1 + 1) for its last
    diagonal q1 - 1, and the last part carries the zero-point terms."""
    d, e, zc, S = split(P, nslices, kp)
    m, kk = d[0].shape
    scale = e[:, None] + e[None, :] + 2
    parts = []
    for q0 in range(0, nslices, PASS_Q):
        q1 = min(nslices, q0 + PASS_Q)
        acc = np.zeros((m, m))
        for q in range(q0, q1):
            Dq = np.zeros((m, m))
            for a in range(q + 1):
                Dq += d[a] @ d[q - a].T
            acc = acc * 256.0 + Dq
        core = np.ldexp(acc, -8 * (q1 + 1))
        if q1 == nslices:
            core = (core + zc * (S[:, None] + S[None, :])) + kk * zc * zc
        parts.append(np.ldexp(core, scale))
    return parts


def product(P, nslices, kp=None):
    """The emulated P P^T (m, m), the passes' parts summed."""
    parts = product_parts(P, nslices, kp)
    V = parts[0]
    for part in parts[1:]:
        V = V + part
    return V


def syrk_lower(C, P, nslices, strip_cols=0):
    """C - P P^T on the lower triangle (first strip_cols columns if > 0), one
    subtraction per pass in the kernel's order; the kernel pads k to a
    multiple of 32 with zeros."""
    C = np.array(C, dtype=np.float64, copy=True)
    m = C.shape[0]
    kp = -(-P.shape[1] // 32) * 32
    mask = np.tril(np.ones((m, m), dtype=bool))
    if strip_cols > 0:
        mask[:, strip_cols:] = False
    for V in product_parts(P, nslices, kp):
        C[mask] -= V[mask]
    return C


def error_bound(P, nslices):
    """Entry-wise bound on |emulated - exact| P P^T: k (s + 3) 2^(e_r + e_c + 2 - 8 s)."""
    _, e, _, _ = split(P, nslices)
    k = P.shape[1]
    return k * (nslices + 3) * np.ldexp(1.0, e[:, None] + e[None, :] + 2 - 8 * nslices)
