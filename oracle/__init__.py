"""CPU ORACLE — test infrastructure, not product code.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference arm use this package, as the checker; the product package
``fml_b200`` never imports it.

* ``oracle.c`` (built into ``liboracle.so`` by ``oracle/Makefile``) restates the
  reference's Fortran routines on the hot path in plain C, FP64, with the
  reference's OpenMP outer loops.
* ``arad_describe.py`` restates ``ARAD.describe`` (fml/arad.py:70-145).
* ``cho_solve`` calls LAPACK ``dpotrf``/``dpotrs`` through scipy (OpenBLAS),
  the same LAPACK routines fml/math/fcho_solve.f90:35-42 calls; the reference
  pins no LAPACK version (Makefile:14 links the system ``-llapack``).

The functions below keep the reference's Python signatures
(fml/kernels/kernels.py, fml/math/cho_solve.py) so parity tests read like
the reference's own usage.
"""

import ctypes
import os
import subprocess

import numpy as np

from .arad_describe import describe as arad_describe  # noqa: F401
from .ptp import ptp_of

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.orc_cm_sorted.restype = ctypes.c_int
        lib.orc_cm_sorted_batch.restype = ctypes.c_int
        lib.orc_cm_local_batch.restype = ctypes.c_int
        lib.orc_cm_unsorted_batch.restype = ctypes.c_int
        lib.orc_potrf_upper.restype = ctypes.c_int
        lib.orc_num_threads.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def num_threads():
    return _lib().orc_num_threads()


# --------------------------------------------------------------------------
# descriptors
# --------------------------------------------------------------------------
def generate_coulomb_matrix(charges, coords, size=23, return_order=False):
    """frepresentations.f90:23-110 for one molecule."""
    z = np.ascontiguousarray(charges, dtype=np.float64)
    r = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    if len(z) != len(r):
        raise ValueError("coordinates / nuclear_charges size mismatch")
    if len(z) > size:
        raise ValueError("molecule has more atoms than size")
    cm = np.zeros(size * (size + 1) // 2)
    order = np.zeros(max(len(z), 1), dtype=np.int32)
    _lib().orc_cm_sorted(len(z), _p(z), _p(r), size, _p(cm), _p(order, _ip))
    return (cm, order[: len(z)]) if return_order else cm


def coulomb_matrices(charges, coords, offsets, size=23, return_order=False):
    """Batch of sorted CMs over a packed ragged molecule buffer."""
    z = np.ascontiguousarray(charges, dtype=np.float64)
    r = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    nmol = len(off) - 1
    cm = np.zeros((nmol, size * (size + 1) // 2))
    order = np.full((nmol, size), -1, dtype=np.int32)
    rc = _lib().orc_cm_sorted_batch(nmol, _p(off, _ip), _p(z), _p(r), size, _p(cm),
                                    _p(order, _ip))
    if rc:
        raise ValueError("molecule has more atoms than size")
    return (cm, order) if return_order else cm


def unsorted_coulomb_matrices(charges, coords, offsets, size=23):
    """frepresentations.f90:112-202 restated in oracle.c: (nmol, size*(size+1)/2)."""
    z = np.ascontiguousarray(charges, dtype=np.float64)
    r = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    cm = np.zeros((len(off) - 1, size * (size + 1) // 2))
    if _lib().orc_cm_unsorted_batch(len(off) - 1, _p(off, _ip), _p(z), _p(r), size, _p(cm)):
        raise ValueError("molecule has more atoms than size")
    return cm


def local_coulomb_matrices(charges, coords, offsets, size=23, kind="local"):
    """Per-atom CMs (total_atoms, size*(size+1)/2): frepresentations.f90:204-294
    (kind "local") and :297-390 (kind "atomic"), restated in oracle.c."""
    z = np.ascontiguousarray(charges, dtype=np.float64)
    r = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    nmol = len(off) - 1
    cm = np.zeros((int(off[-1]) if nmol else 0, size * (size + 1) // 2))
    rc = _lib().orc_cm_local_batch(nmol, _p(off, _ip), _p(z), _p(r), size,
                                   {"local": 0, "atomic": 1}[kind], _p(cm))
    if rc:
        raise ValueError("molecule has more atoms than size")
    return cm


def vector_kernels(kind, x1, x2, n1, n2, sigmas):
    """fkernels.f90:23-162 restated in oracle.c; x (nm, amax, d) rows,
    kind "gaussian" or "laplacian" -> (nsig, nm1, nm2)."""
    x1 = np.ascontiguousarray(x1, dtype=np.float64)
    x2 = np.ascontiguousarray(x2, dtype=np.float64)
    n1 = np.ascontiguousarray(n1, dtype=np.int32)
    n2 = np.ascontiguousarray(n2, dtype=np.int32)
    sig = np.ascontiguousarray(np.atleast_1d(sigmas), dtype=np.float64)
    K = np.zeros((len(sig), x1.shape[0], x2.shape[0]))
    _lib().orc_vector_kernels({"gaussian": 0, "laplacian": 1}[kind], _p(x1), _p(n1, _ip),
                              x1.shape[0], x1.shape[1], _p(x2), _p(n2, _ip), x2.shape[0],
                              x2.shape[1], x1.shape[2], _p(sig), len(sig), _p(K))
    return K


def arad_descriptors(charges, coords, offsets, size=23, cut=5.0):
    off = np.asarray(offsets)
    out = np.zeros((len(off) - 1, size, 5, size))
    for m in range(len(off) - 1):
        out[m] = arad_describe(coords[off[m]:off[m + 1]], charges[off[m]:off[m + 1]], size, cut)
    return out


# --------------------------------------------------------------------------
# kernels (reference signatures: A is (d, na), B is (d, nb))
# --------------------------------------------------------------------------
def _rows(A):
    # the reference's A(:, j) is descriptor j; store descriptors as C rows
    return np.ascontiguousarray(np.asarray(A, dtype=np.float64).T)


def gaussian_kernel(A, B, sigma):
    """fkernels.f90:317-349 via kernels.py:167-196."""
    a, b = _rows(A), _rows(B)
    na, nb, d = a.shape[0], b.shape[0], a.shape[1]
    K = np.empty((na, nb))
    _lib().orc_gaussian_kernel(_p(a), na, _p(b), nb, d, ctypes.c_double(sigma), _p(K))
    return K


def laplacian_kernel(A, B, sigma):
    """fkernels.f90:351-377 via kernels.py:136-164."""
    a, b = _rows(A), _rows(B)
    na, nb, d = a.shape[0], b.shape[0], a.shape[1]
    K = np.empty((na, nb))
    _lib().orc_laplacian_kernel(_p(a), na, _p(b), nb, d, ctypes.c_double(sigma), _p(K))
    return K


def kernels_multi(kind, A, B, sigmas):
    """Gaussian (kind "gaussian") or Laplacian ("laplacian") kernels for every
    sigma from one pass over the pairs (fkernels.f90:317-377); each plane is
    bit-identical to gaussian_kernel / laplacian_kernel at that sigma.
    Returns (nsigma, na, nb)."""
    a, b = _rows(A), _rows(B)
    na, nb, d = a.shape[0], b.shape[0], a.shape[1]
    sig = np.ascontiguousarray(np.atleast_1d(np.asarray(sigmas, dtype=np.float64)))
    if not 1 <= len(sig) <= 16:
        raise ValueError("1..16 sigmas")
    K = np.empty((len(sig), na, nb))
    _lib().orc_kernels_multi({"gaussian": 0, "laplacian": 1}[kind], _p(a), na, _p(b), nb, d,
                             _p(sig), len(sig), _p(K))
    return K


def _ptp_pad(Z, amax):
    out = np.zeros((len(Z), amax, 2))
    for i, z in enumerate(Z):
        if len(z):
            out[i, : len(z)] = ptp_of(z)
    return out


def get_atomic_kernels_arad(X1, X2, Z1, Z2, sigmas, width=0.2, cut_distance=6.0,
                            r_width=1.0, c_width=0.5):
    """farad_kernels.f90:439-616 via kernels.py:229-297."""
    X1 = np.ascontiguousarray(X1, dtype=np.float64)
    X2 = np.ascontiguousarray(X2, dtype=np.float64)
    amax = X1.shape[1]
    n1 = np.array([len(z) for z in Z1], dtype=np.int32)
    n2 = np.array([len(z) for z in Z2], dtype=np.int32)
    z1, z2 = _ptp_pad(Z1, amax), _ptp_pad(Z2, amax)
    s = np.ascontiguousarray(sigmas, dtype=np.float64)
    K = np.zeros((len(s), len(Z1), len(Z2)))
    _lib().orc_arad_kernels(_p(X1), _p(X2), _p(z1), _p(z2), _p(n1, _ip), _p(n2, _ip), _p(s),
                            len(Z1), len(Z2), len(s), amax, ctypes.c_double(width),
                            ctypes.c_double(cut_distance), ctypes.c_double(r_width),
                            ctypes.c_double(c_width), _p(K))
    return K


def get_atomic_symmetric_kernels_arad(X1, Z1, sigmas, width=0.2, cut_distance=6.0,
                                      r_width=1.0, c_width=0.5):
    """farad_kernels.f90:619-755 via kernels.py:300-349."""
    X1 = np.ascontiguousarray(X1, dtype=np.float64)
    amax = X1.shape[1]
    n1 = np.array([len(z) for z in Z1], dtype=np.int32)
    z1 = _ptp_pad(Z1, amax)
    s = np.ascontiguousarray(sigmas, dtype=np.float64)
    K = np.zeros((len(s), len(Z1), len(Z1)))
    _lib().orc_arad_symmetric_kernels(_p(X1), _p(z1), _p(n1, _ip), _p(s), len(Z1), len(s), amax,
                                      ctypes.c_double(width), ctypes.c_double(cut_distance),
                                      ctypes.c_double(r_width), ctypes.c_double(c_width), _p(K))
    return K


def distance_matrix(kind, A, B, p=None):
    """fdistance.f90:23-155 restated in oracle.c; A (d, na), B (d, nb) in the
    reference layout, kind "manhattan" | "l2" | "p_int" | "p_real"."""
    a = np.ascontiguousarray(np.asarray(A, dtype=np.float64).T)
    b = np.ascontiguousarray(np.asarray(B, dtype=np.float64).T)
    D = np.zeros((a.shape[0], b.shape[0]))
    k = {"manhattan": 0, "l2": 1, "p_int": 2, "p_real": 3}[kind]
    _lib().orc_distance_matrix(k, _p(a), a.shape[0], _p(b), b.shape[0], a.shape[1],
                               int(p) if k == 2 else 0,
                               ctypes.c_double(float(p) if k == 3 else 0.0), _p(D))
    return D


def get_l2_distance_arad(X1, X2, Z1, Z2, width=0.2, cut_distance=6.0, r_width=1.0,
                         c_width=0.5):
    """fml/math/distance.py:120-189 -> atomic_arad_l2_distance_all (farad.f90:452-600),
    restated in oracle.c: D (nm1, nm2, amax, amax)."""
    X1 = np.ascontiguousarray(X1, dtype=np.float64)
    X2 = np.ascontiguousarray(X2, dtype=np.float64)
    amax = X1.shape[1]
    n1 = np.array([len(z) for z in Z1], dtype=np.int32)
    n2 = np.array([len(z) for z in Z2], dtype=np.int32)
    z1, z2 = _ptp_pad(Z1, amax), _ptp_pad(Z2, amax)
    D = np.zeros((len(Z1), len(Z2), amax, amax))
    _lib().orc_arad_l2_distance_all(_p(X1), _p(X2), _p(z1), _p(z2), _p(n1, _ip), _p(n2, _ip),
                                    len(Z1), len(Z2), amax, ctypes.c_double(width),
                                    ctypes.c_double(cut_distance), ctypes.c_double(r_width),
                                    ctypes.c_double(c_width), _p(D))
    return D


def _explicit_inverse(K, y, n):
    """dpotrf('U'), dpotri('U'), dsymv('U') on K (numpy, upper triangle read),
    then each molecule's value spread over its atoms: the common tail of the
    reference's explicit-inverse routines. Returns (alpha, info, info2)."""
    from scipy.linalg import blas, lapack
    c, info = lapack.dpotrf(np.asfortranarray(K), lower=0, clean=0)
    inv, info2 = lapack.dpotri(c, lower=0)
    ltcly = blas.dsymv(1.0, inv, np.asarray(y, dtype=np.float64), lower=0)
    return np.repeat(ltcly, n), int(info), int(info2)


def _offsets(N):
    n = np.asarray(N, dtype=np.int32)
    off = np.zeros(len(n) + 1, dtype=np.int32)
    np.cumsum(n, out=off[1:])
    return n, off


def get_alpha(Q, N, Y, sigma, llambda):
    """kernels.py:119-126 -> fget_alpha (fkernels.f90:380-478); Q (d, na)."""
    q = np.ascontiguousarray(np.asarray(Q, dtype=np.float64).T)
    n, off = _offsets(N)
    K = np.zeros((len(n), len(n)))
    _lib().orc_atomic_laplacian_kernel(_p(q), q.shape[0], q.shape[1], _p(off, _ip), len(n),
                                       ctypes.c_double(sigma), _p(K))
    K[np.diag_indices(len(n))] += llambda
    return _explicit_inverse(K, Y, n)


def get_prediction(Q, Q2, N2, alpha, sigma):
    """kernels.py:101-108 -> fget_prediction (fkernels.f90:480-539)."""
    q = np.ascontiguousarray(np.asarray(Q, dtype=np.float64).T)
    q2 = np.ascontiguousarray(np.asarray(Q2, dtype=np.float64).T)
    n2, off2 = _offsets(N2)
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    Y = np.zeros(len(n2))
    _lib().orc_atomic_laplacian_predict(_p(q), q.shape[0], _p(q2), q2.shape[0], q.shape[1],
                                        _p(off2, _ip), len(n2), _p(a), ctypes.c_double(sigma),
                                        _p(Y))
    return Y


def get_alpha_from_distance(D, N, Y, sigma, llambda):
    """kernels.py:127-134 -> fget_alpha_from_distance (fkernels.f90:541-641)."""
    d = np.ascontiguousarray(D, dtype=np.float64)
    n, off = _offsets(N)
    K = np.zeros((len(n), len(n)))
    _lib().orc_distance_mol_kernel(_p(d), d.shape[0], _p(off, _ip), len(n),
                                   ctypes.c_double(sigma), _p(K))
    K[np.diag_indices(len(n))] += llambda
    return _explicit_inverse(K, Y, n)


def get_prediction_from_distance(D2, N2, alpha, sigma):
    """kernels.py:110-117 -> fget_prediction_from_distance (fkernels.f90:645-702)."""
    d2 = np.ascontiguousarray(D2, dtype=np.float64)
    n2, off2 = _offsets(N2)
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    Y = np.zeros(len(n2))
    _lib().orc_distance_predict(_p(d2), d2.shape[0], d2.shape[1], _p(off2, _ip), len(n2), _p(a),
                                ctypes.c_double(sigma), _p(Y))
    return Y


def fget_kernel_arad(q, z, n, sigma, nm):
    """farad_kernels.f90:95-227: the fixed-parameter symmetric ARAD kernel of
    the first nm molecules (eps 1e-11), from oracle.c."""
    q = np.ascontiguousarray(np.asarray(q, dtype=np.float64)[:nm])
    z = np.ascontiguousarray(np.asarray(z, dtype=np.float64)[:nm])
    n = np.ascontiguousarray(np.asarray(n)[:nm], dtype=np.int32)
    K = np.zeros((nm, nm))
    _lib().orc_arad_alpha_kernel(_p(q), _p(z), _p(n, _ip), nm, q.shape[1],
                                 ctypes.c_double(sigma), ctypes.c_double(0.0), _p(K))
    return K


def fget_alpha_arad(q, z, n, y, sigma, lambda_):
    """farad_kernels.f90:231-436: K + lambda I from oracle.c, then LAPACK
    dpotrf('U'), dpotri('U') and BLAS dsymv('U') as the routine calls them
    (:391-403), and the per-molecule value spread over its atoms (:407-432).
    Returns (alpha (sum(n),), potrf info, potri info)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    z = np.ascontiguousarray(z, dtype=np.float64)
    n = np.ascontiguousarray(n, dtype=np.int32)
    nm, amax = q.shape[0], q.shape[1]
    K = np.zeros((nm, nm))
    _lib().orc_arad_alpha_kernel(_p(q), _p(z), _p(n, _ip), nm, amax, ctypes.c_double(sigma),
                                 ctypes.c_double(lambda_), _p(K))
    return _explicit_inverse(K, y, n)


def fget_atomic_kernels_arad(q1, q2, z1, z2, n1, n2, sigmas, na1, na2, nsigmas, width,
                             cut_distance, r_width, c_width):
    """farad_kernels.f90:757-899 (the f2py routine fml.kernels exports).
    q (na, 5, m) per-atom descriptors, z (na, 2), n (na,) neighbour counts."""
    amax = max(np.shape(q1)[2], np.shape(q2)[2])
    Q1, Q2 = (np.zeros((q.shape[0], 5, amax)) for q in (np.asarray(q1), np.asarray(q2)))
    Q1[:, :, :np.shape(q1)[2]] = q1
    Q2[:, :, :np.shape(q2)[2]] = q2
    K = np.zeros((nsigmas, na1, na2))
    _lib().orc_arad_atomic_kernels(
        _p(Q1), _p(Q2), _p(np.ascontiguousarray(z1, np.float64)),
        _p(np.ascontiguousarray(z2, np.float64)), _p(np.ascontiguousarray(n1, np.int32), _ip),
        _p(np.ascontiguousarray(n2, np.int32), _ip), _p(np.ascontiguousarray(sigmas, np.float64)),
        na1, na2, nsigmas, amax, ctypes.c_double(width), ctypes.c_double(cut_distance),
        ctypes.c_double(r_width), ctypes.c_double(c_width), _p(K))
    return K


def atomic_distances_arad(q1, q2, z1, z2, n1, n2, width, cut_distance, r_width, c_width):
    """The l2 distances of fget_atomic_distance_arad (farad_kernels.f90:902-1030),
    D[i, j] = l2(i, j), shape (na1, na2)."""
    amax = max(np.shape(q1)[2], np.shape(q2)[2])
    Q1, Q2 = (np.zeros((q.shape[0], 5, amax)) for q in (np.asarray(q1), np.asarray(q2)))
    Q1[:, :, :np.shape(q1)[2]] = q1
    Q2[:, :, :np.shape(q2)[2]] = q2
    D = np.zeros((len(Q1), len(Q2)))
    _lib().orc_arad_atomic_distances(
        _p(Q1), _p(Q2), _p(np.ascontiguousarray(z1, np.float64)),
        _p(np.ascontiguousarray(z2, np.float64)), _p(np.ascontiguousarray(n1, np.int32), _ip),
        _p(np.ascontiguousarray(n2, np.int32), _ip), len(Q1), len(Q2), amax,
        ctypes.c_double(width), ctypes.c_double(cut_distance), ctypes.c_double(r_width),
        ctypes.c_double(c_width), _p(D))
    return D


# --------------------------------------------------------------------------
# solve
# --------------------------------------------------------------------------
def cho_solve(A, y):
    """fcho_solve.f90:23-47: LAPACK dpotrf('U') then dpotrs('U') (scipy/OpenBLAS).

    Returns (x, info_potrf)."""
    from scipy.linalg import lapack

    A = np.asarray(A, dtype=np.float64)
    c, info = lapack.dpotrf(np.asfortranarray(A), lower=0, clean=0, overwrite_a=0)
    x, info2 = lapack.dpotrs(c, np.asarray(y, dtype=np.float64), lower=0)
    return x, int(info)


def cho_invert(A):
    """fml/math/cho_solve.py:27-30 -> fcho_solve.f90:49-68: LAPACK dpotrf('U')
    then dpotri('U') on a Fortran copy; the strict lower triangle keeps A's
    values (LAPACK does not touch it)."""
    from scipy.linalg import lapack
    a = np.asfortranarray(np.array(A, dtype=np.float64))
    c, info = lapack.dpotrf(a, lower=0, clean=0, overwrite_a=0)
    inv, info2 = lapack.dpotri(c, lower=0, overwrite_c=0)
    out = np.asfortranarray(inv)
    il = np.tril_indices(len(a), -1)
    out[il] = a[il]
    return out, int(info), int(info2)


def cho_solve_restated(A, y):
    """Plain-C unblocked restatement of dpotrf('U') + dpotrs('U'). (x, info)."""
    U = np.array(A, dtype=np.float64, order="C", copy=True)
    n = U.shape[0]
    info = _lib().orc_potrf_upper(n, _p(U))
    x = np.array(y, dtype=np.float64, copy=True)
    if info == 0:
        _lib().orc_potrs_upper(n, _p(U), _p(x))
    return x, int(info)
