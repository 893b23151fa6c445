"""Kernel matrices: drop-ins for fml/kernels/kernels.py.

* ``gaussian_kernel(A, B, sigma)``  -> fgaussian_kernel (fkernels.f90:317-349)
* ``laplacian_kernel(A, B, sigma)`` -> flaplacian_kernel (fkernels.f90:351-377)
* ``get_atomic_kernels_arad`` / ``get_atomic_symmetric_kernels_arad``
  -> fget_kernels_arad / fget_symmetric_kernels_arad (farad_kernels.f90:439-755)
* ``get_atomic_kernels_gaussian`` / ``get_atomic_kernels_laplacian`` and
  the directly exported ``fget_vector_kernels_gaussian`` ->
  fget_vector_kernels_gaussian / fget_vector_kernels_laplacian
  (fkernels.f90:23-162), sums over atom pairs of per-atom descriptors
* ``fget_alpha_arad`` / ``fget_kernel_arad`` -> the routines of those names
  (farad_kernels.f90:95-436): explicit-inverse ARAD KRR weights and the
  fixed-parameter symmetric ARAD kernel
* ``get_alpha`` / ``get_prediction`` / ``get_alpha_from_distance`` /
  ``get_prediction_from_distance`` -> fget_alpha, fget_prediction and their
  from-distance forms (fkernels.f90:380-702): atomic Laplacian KRR
* ``fget_atomic_kernels_arad`` / ``fget_atomic_distance_arad`` -> the
  atom-level routines of the same names (farad_kernels.f90:757-1030), which
  fml.kernels exports directly

Signatures follow the reference: ``A`` is (d, na) and ``B`` is (d, nb) with
descriptors as columns; the result is (na, nb). Extension: ``sigma`` may be a
sequence, giving (nsigma, na, nb) from one pass. ``A is B`` selects the
symmetric build (lower tiles computed, mirrored; bit-identical to the full
build).

Differences from the reference, by design: results are C-ordered (the
reference returns Fortran order; values are the same), and
``get_atomic_symmetric_kernels_arad`` works (the reference wrapper calls
``fget_symmetric_kernels_arad`` without importing it, kernels.py:36-39 vs
:348, and raises NameError).
"""

import warnings

import numpy as np
import torch

from . import _lib
from .cho_solve import CholeskyWarning, potrf
from ._tensors import device, is_torch, to_device, to_output, workspace
from .data import PTP_COL, PTP_ROW

PRECISIONS = {"fp64": 0, "fp32": 1}


def _sigma_list(sigma):
    if np.ndim(sigma) == 0:
        return [float(sigma)], True
    s = [float(v) for v in np.asarray(sigma).ravel()]
    if not s:
        raise ValueError("need at least one sigma")
    return s, False


def _descriptor_rows(A):
    """(d, n) reference layout -> (n, d) rows on the device (float64)."""
    if is_torch(A):
        t = A.to(device=device(), dtype=torch.float64)
        return t.t().contiguous(), False
    a = np.asarray(A, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("expected a 2-D descriptor matrix (d, n)")
    rows, _ = to_device(np.ascontiguousarray(a.T), torch.float64)
    return rows, True


def _pairwise(A, B, sigma, fn, out_dtype=torch.float64):
    sig, scalar = _sigma_list(sigma)
    symmetric = A is B
    a, as_np = _descriptor_rows(A)
    b = a if symmetric else _descriptor_rows(B)[0]
    if a.shape[1] != b.shape[1]:
        raise ValueError("A and B must hold descriptors of the same length")
    na, d = a.shape
    nb = b.shape[0]
    K = torch.empty((len(sig), na, nb), dtype=out_dtype, device=device())
    sp, keep = _lib.host_doubles(sig)
    if na and nb:
        _lib.call(fn, _lib.ptr(a), na, d, _lib.ptr(b), nb, d, d, sp, len(sig), _lib.ptr(K), nb,
                  na * nb, 1 if symmetric else 0, _lib.stream_handle())
    del keep
    out = K[0] if scalar else K
    return to_output(out, as_np)


def _gaussian_tc(A, B, sigma):
    """Tensor-core (tcgen05, BF16 hi/lo x3) Gaussian kernel, FP32 result."""
    sig, scalar = _sigma_list(sigma)
    if len(sig) > 8:
        raise ValueError("the tensor-core path takes at most 8 sigmas per call")
    symmetric = A is B
    a, as_np = _descriptor_rows(A)
    b = a if symmetric else _descriptor_rows(B)[0]
    if a.shape[1] != b.shape[1]:
        raise ValueError("A and B must hold descriptors of the same length")
    na, d = a.shape
    nb = b.shape[0]
    dev = device()
    lib = _lib.load()
    K = torch.empty((len(sig), na, nb), dtype=torch.float32, device=dev)
    if na and nb:
        mu = torch.empty(d, dtype=torch.float64, device=dev)
        st = _lib.stream_handle()
        _lib.call("fmlb_column_mean_f64", _lib.ptr(b), nb, d, d, _lib.ptr(mu), st)
        nbytes = lib.fmlb_tc_operand_bytes(na, d) + (0 if symmetric else
                                                      lib.fmlb_tc_operand_bytes(nb, d))
        ws = workspace(nbytes)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        sp, keep = _lib.host_doubles(sig)
        _lib.call("fmlb_gaussian_kernel_tc", _lib.ptr(a), na, d, _lib.ptr(b), nb, d, d,
                  _lib.ptr(mu), sp, len(sig), _lib.ptr(K), nb, na * nb, 1 if symmetric else 0,
                  _lib.ptr(ws), ws.numel(), _lib.ptr(status), st)
        del keep
        code = int(status.item())
        if code:
            raise _lib.FmlbError(_lib.FMLB_ETIMEDOUT,
                                 "fmlb_gaussian_kernel_tc: a device-side wait gave up (%d)" % code)
    out = K[0] if scalar else K
    return to_output(out, as_np)


def gaussian_kernel(A, B, sigma, precision="fp64"):
    """K_ij = exp(-0.5 / sigma**2 * ||A_i - B_j||_2**2).

    precision="fp64": FP64 direct differences (the reference's arithmetic);
    precision="bf16x3": tcgen05 tensor cores, BF16 hi/lo splits of the
    mean-centred descriptors, FP32 result.
    """
    if precision == "bf16x3":
        return _gaussian_tc(A, B, sigma)
    if precision != "fp64":
        raise ValueError("precision must be 'fp64' or 'bf16x3'")
    return _pairwise(A, B, sigma, "fmlb_gaussian_kernel_f64")


def laplacian_kernel(A, B, sigma, precision="fp64"):
    """K_ij = exp(-1 / sigma * ||A_i - B_j||_1).

    precision="fp64": FP64 direct differences (the reference's arithmetic);
    precision="fp32": FP32 CUDA-core kernel, FP32 result.
    """
    if precision == "fp32":
        return _pairwise(A, B, sigma, "fmlb_laplacian_kernel_f32", torch.float32)
    if precision != "fp64":
        raise ValueError("precision must be 'fp64' or 'fp32'")
    return _pairwise(A, B, sigma, "fmlb_laplacian_kernel_f64")


# ---------------------------------------------------------------------------
# ARAD
# ---------------------------------------------------------------------------
def _ptp_arrays(Z, amax):
    """kernels.py:261-292: PTP (nm, amax, 2) float64 and atom counts N (nm,) int32.

    One table lookup over the concatenated charges and one scatter into the
    padded rows, with the reference's errors in its order: charges are
    truncated toward zero as int(q) does (a non-finite charge raises
    ValueError or OverflowError as int() does); a charge the table does not
    hold raises KeyError with the first such charge in molecule and atom order
    (the dict lookup of kernels.py:276, done for every molecule before any
    row is filled); then a molecule with more atoms than the descriptor size
    raises IndexError (the row fill of kernels.py:281)."""
    nm = len(Z)
    zs = [np.asarray(z, dtype=np.float64).reshape(-1) for z in Z]
    N = np.array([len(z) for z in zs], dtype=np.int32)
    Zp = np.zeros((nm, amax, 2))
    if not (nm and N.sum()):
        return Zp, N
    zf = np.concatenate(zs)
    fin = np.isfinite(zf)
    zi = np.trunc(np.clip(np.where(fin, zf, 0.0), -1.0, 128.0)).astype(np.int64)
    bad = ~fin | (zi < 0) | (zi > 127)
    bad |= PTP_ROW[np.clip(zi, 0, 127)] < 0
    if bad.any():
        # int() of the first offending charge raises for NaN / inf as the
        # reference's int(q) does; otherwise the dict lookup's KeyError
        raise KeyError(int(zf[int(np.argmax(bad))]))
    if N.max() > amax:
        raise IndexError("index %d is out of bounds for axis 1 with size %d" % (amax, amax))
    mol = np.repeat(np.arange(nm), N)
    slot = np.arange(len(zi)) - np.repeat(np.cumsum(N) - N, N)
    Zp[mol, slot, 0] = PTP_ROW[zi]
    Zp[mol, slot, 1] = PTP_COL[zi]
    return Zp, N


def _arad(X1, X2, Z1, Z2, sigmas, width, cut_distance, r_width, c_width, symmetric, precision):
    prec = PRECISIONS[precision]
    sig, _ = _sigma_list(sigmas)
    amax = X1.shape[1]
    nm1 = len(Z1)
    nm2 = nm1 if symmetric else len(Z2)
    x1, as_np = to_device(X1, torch.float64)
    z1p, n1 = _ptp_arrays(Z1, amax)
    z1, _ = to_device(z1p, torch.float64)
    n1d, _ = to_device(n1, torch.int32)
    if symmetric:
        x2 = z2 = n2d = None
    else:
        x2, _ = to_device(X2, torch.float64)
        z2p, n2 = _ptp_arrays(Z2, amax)
        z2, _ = to_device(z2p, torch.float64)
        n2d, _ = to_device(n2, torch.int32)
    K = torch.empty((len(sig), nm1, nm2), dtype=torch.float64, device=device())
    nbytes = _lib.load().fmlb_arad_workspace_bytes(nm1, nm2, amax, 1 if symmetric else 0)
    ws = workspace(nbytes)
    sp, keep = _lib.host_doubles(sig)
    _lib.call("fmlb_arad_kernels", _lib.ptr(x1), _lib.ptr(z1), _lib.ptr(n1d), nm1,
              _lib.ptr(x2), _lib.ptr(z2), _lib.ptr(n2d), nm2, amax, sp, len(sig),
              float(width), float(cut_distance), float(r_width), float(c_width),
              1 if symmetric else 0, prec, _lib.ptr(K), _lib.ptr(ws), ws.numel(),
              _lib.stream_handle())
    del keep
    return to_output(K, as_np)


def arad_launches(symmetric, precision, amax, nsigma):
    """Kernel launches of one ``fmlb_arad_kernels`` call (mirrors its host code)."""
    fast = precision == "fp32" and amax <= 32
    sets = 1 if symmetric else 2
    if fast:  # prep, class scan, assign, record sort, self per set; class build; fast + gated
        return 5 * sets + 1 + 2 * -(-nsigma // 8)  # generic pair per sigma chunk
    return sets + -(-nsigma // 16)


def _atomic_inputs(q1a, q2a, z1, z2, n1, n2):
    """Per-atom descriptors on the device, padded to one width, with PTP and counts."""
    amax = max(q1a.shape[2], q2a.shape[2])
    dev = device()

    def padded(q):
        t, _ = to_device(q, torch.float64)
        if t.shape[2] == amax:
            return t.contiguous()
        out = torch.zeros((t.shape[0], 5, amax), dtype=torch.float64, device=dev)
        out[:, :, :t.shape[2]] = t
        return out

    def rows(z):
        return to_device(z if is_torch(z) else np.asarray(z, np.float64).reshape(-1, 2),
                         torch.float64)[0]

    def counts(n):
        return to_device(n if is_torch(n) else np.asarray(n, np.int32), torch.int32)[0]

    return padded(q1a), padded(q2a), rows(z1), rows(z2), counts(n1), counts(n2), amax


def fget_atomic_kernels_arad(q1, q2, z1, z2, n1, n2, sigmas, na1, na2, nsigmas, width,
                             cut_distance, r_width, c_width):
    """Atom-level ARAD kernel, the routine fml.kernels exports from its Fortran
    (farad_kernels.f90:757-899; the f2py argument order is kept).

    q1 (na1, 5, m1) / q2 (na2, 5, m2): per-atom ARAD descriptors; z1 (na1, 2) /
    z2 (na2, 2): period row and group column of each atom; n1 / n2: neighbour
    counts. Returns (nsigmas, na1, na2), FP64 in the reference's order.
    Difference: the reference prints its inv_cut value to stdout; this does not.
    """
    q1a = q1 if is_torch(q1) else np.asarray(q1, dtype=np.float64)
    q2a = q2 if is_torch(q2) else np.asarray(q2, dtype=np.float64)
    if q1a.shape[0] != na1 or q2a.shape[0] != na2 or len(n1) != na1 or len(n2) != na2:
        raise ValueError("na1 / na2 do not match the descriptor and count arrays")
    sig, _ = _sigma_list(sigmas)
    if len(sig) != nsigmas:
        raise ValueError("nsigmas does not match sigmas")
    Q1, Q2, Z1d, Z2d, N1d, N2d, amax = _atomic_inputs(q1a, q2a, z1, z2, n1, n2)
    dev = device()
    K = torch.empty((nsigmas, na1, na2), dtype=torch.float64, device=dev)
    ws = workspace(_lib.load().fmlb_arad_atomic_workspace_bytes(na1, na2, amax))
    sp, keep = _lib.host_doubles(sig)
    _lib.call("fmlb_arad_atomic_kernels", _lib.ptr(Q1), _lib.ptr(Z1d), _lib.ptr(N1d), na1,
              _lib.ptr(Q2), _lib.ptr(Z2d), _lib.ptr(N2d), na2, amax, sp, nsigmas, float(width),
              float(cut_distance), float(r_width), float(c_width), _lib.ptr(K), _lib.ptr(ws),
              ws.numel(), _lib.stream_handle())
    del keep
    return to_output(K, not is_torch(q1))


def fget_atomic_distance_arad(q1, q2, z1, z2, n1, n2, na1, na2, width, cut_distance, r_width,
                              c_width):
    """Atom-pair l2 distances, the routine fml.kernels exports from its Fortran
    (farad_kernels.f90:902-1030; the f2py argument order is kept).

    The reference stores l2(i, j) at kernel(j, i) of an (na1, na2) array
    (:1019): the result is the transpose of the distance matrix, and only
    na1 == na2 stays inside the array. That result is reproduced for
    na1 == na2; other shapes raise ValueError.
    """
    if na1 != na2:
        raise ValueError("fget_atomic_distance_arad writes kernel(j, i) into an (na1, na2) "
                         "array: only na1 == na2 is defined")
    q1a = q1 if is_torch(q1) else np.asarray(q1, dtype=np.float64)
    q2a = q2 if is_torch(q2) else np.asarray(q2, dtype=np.float64)
    if q1a.shape[0] != na1 or q2a.shape[0] != na2 or len(n1) != na1 or len(n2) != na2:
        raise ValueError("na1 / na2 do not match the descriptor and count arrays")
    Q1, Q2, Z1d, Z2d, N1d, N2d, amax = _atomic_inputs(q1a, q2a, z1, z2, n1, n2)
    D = torch.empty((na1, na2), dtype=torch.float64, device=device())
    ws = workspace(_lib.load().fmlb_arad_atomic_workspace_bytes(na1, na2, amax))
    _lib.call("fmlb_arad_atomic_distances", _lib.ptr(Q1), _lib.ptr(Z1d), _lib.ptr(N1d), na1,
              _lib.ptr(Q2), _lib.ptr(Z2d), _lib.ptr(N2d), na2, amax, float(width),
              float(cut_distance), float(r_width), float(c_width), _lib.ptr(D), _lib.ptr(ws),
              ws.numel(), _lib.stream_handle())
    return to_output(D.t().contiguous(), not is_torch(q1))


def _explicit_inverse_weights(Kt, yd, counts):
    """The common tail of the reference's explicit-inverse KRR routines
    (fget_alpha, fget_alpha_from_distance, fget_alpha_arad): dpotrf('U'),
    dpotri('U'), dsymv('U') with y, and each molecule's value spread over its
    atoms. ``Kt`` (nm, nm) device holds K + lambda I with K's upper triangle
    in its row-major lower triangle (it is overwritten). Returns numpy
    (sum(counts),); NaN after a non-positive pivot, with the reference's
    DPOTRF warning."""
    nm = Kt.shape[0]
    dev = Kt.device
    work, info = potrf(Kt, nm)
    ldv = nm + (nm & 1)
    V = torch.empty((nm, ldv), dtype=torch.float64, device=dev)
    _lib.call("fmlb_potri_f64", _lib.ptr(Kt), nm, nm, _lib.ptr(work), _lib.ptr(V), ldv,
              _lib.ptr(info), _lib.stream_handle())
    del V
    _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Kt), nm, nm, _lib.stream_handle())
    ltcly = torch.empty(nm, dtype=torch.float64, device=dev)
    _lib.call("fmlb_gemv_f64", _lib.ptr(Kt), nm, nm, nm, _lib.ptr(yd), _lib.ptr(ltcly),
              _lib.stream_handle())
    code = int(info.item())
    vals = np.repeat(ltcly.cpu().numpy(), counts)
    if code > 0:
        warnings.warn("WARNING: Cholesky decomposition DPOTRF() exited with error code: %d"
                      % code, CholeskyWarning, stacklevel=3)
        vals[:] = np.nan
    return vals


def _counts(N, what):
    n = np.asarray(N.cpu() if is_torch(N) else N, dtype=np.int64).reshape(-1)
    if len(n) and n.min() < 0:
        raise ValueError("%s: atom counts must be >= 0" % what)
    off = np.zeros(len(n) + 1, dtype=np.int64)
    np.cumsum(n, out=off[1:])
    return n.astype(np.int32), off


def _segment_sums(v, off):
    """Y[j] = sum(v[off[j]:off[j+1]]) (the reference's per-molecule sums)."""
    counts = np.diff(off)
    out = np.zeros(len(counts))
    nz = counts > 0
    if nz.any():
        out[nz] = np.add.reduceat(v[:off[-1]], off[:-1][nz])
    return out


def get_alpha(Q, N, Y, sigma, llambda):
    """kernels.py:119-126 -> fget_alpha (fkernels.f90:380-478): atomic
    Laplacian KRR weights. Q (d, na) per-atom descriptors as columns, N atoms
    per molecule, Y (nm,). K[i, j] = sum over atom pairs of molecules i, j of
    exp(-|q_a - q_b|_1 / sigma), plus llambda on the diagonal, inverted from
    its Cholesky factor on the GPU; returns alpha (sum(N),), each atom holding
    its molecule's weight."""
    n, off = _counts(N, "get_alpha")
    nm = len(n)
    q, _ = _descriptor_rows(Q)  # (na, d)
    if off[-1] > q.shape[0]:
        raise ValueError("get_alpha: sum(N) = %d exceeds the %d atoms of Q"
                         % (off[-1], q.shape[0]))
    if len(Y) != nm:
        raise ValueError("get_alpha: Y must hold one value per molecule")
    if nm == 0:
        return np.zeros(0)
    dev = q.device
    amax = max(int(n.max()), 1)
    if amax > 128:
        raise ValueError("get_alpha: at most 128 atoms per molecule")
    od = torch.from_numpy(off.astype(np.int32)).to(dev)
    K = torch.empty((nm, nm), dtype=torch.float64, device=dev)
    sp, keep = _lib.host_doubles([float(sigma)])
    _lib.call("fmlb_vector_kernels_packed_f64", 1, _lib.ptr(q), _lib.ptr(od), nm, amax,
              _lib.ptr(q), _lib.ptr(od), nm, amax, q.shape[1], sp, 1, _lib.ptr(K), None,
              _lib.stream_handle())
    del keep
    _lib.call("fmlb_add_diagonal_f64", _lib.ptr(K), nm, nm, float(llambda), _lib.stream_handle())
    yd, _ = to_device(Y if is_torch(Y) else np.asarray(Y, dtype=np.float64), torch.float64)
    return _explicit_inverse_weights(K, yd, n)


def get_prediction(Q, Q2, N2, alpha, sigma):
    """kernels.py:101-108 -> fget_prediction (fkernels.f90:480-539):
    Y[j] = sum over the atoms a2 of test molecule j of sum over all training
    atoms a of exp(-|q_a - q2_a2|_1 / sigma) alpha[a]. The atom sums run in
    the fused kernel-times-weights launch (the kernel matrix is not stored)."""
    n2, off2 = _counts(N2, "get_prediction")
    q, _ = _descriptor_rows(Q)
    q2, _ = _descriptor_rows(Q2)
    if q.shape[1] != q2.shape[1]:
        raise ValueError("get_prediction: descriptor sizes differ")
    if off2[-1] > q2.shape[0]:
        raise ValueError("get_prediction: sum(N2) exceeds the atoms of Q2")
    na, na2 = q.shape[0], q2.shape[0]
    if len(alpha) < na:
        raise ValueError("get_prediction: alpha must hold one weight per atom of Q")
    if na2 == 0 or na == 0:
        return np.zeros(len(n2))
    ad, _ = to_device(alpha if is_torch(alpha) else np.asarray(alpha, dtype=np.float64),
                      torch.float64)
    csa = torch.empty(na2, dtype=torch.float64, device=q.device)
    lib = _lib.load()
    ws = workspace(lib.fmlb_kernel_predict_workspace_bytes(na2, na, 1))
    sp, keep = _lib.host_doubles([float(sigma)])
    _lib.call("fmlb_kernel_predict_f64", 1, _lib.ptr(q2), na2, q2.shape[1], _lib.ptr(q), na,
              q.shape[1], q.shape[1], sp, 1, _lib.ptr(ad), na, _lib.ptr(csa), na2,
              _lib.ptr(ws), ws.numel(), _lib.stream_handle())
    del keep
    return _segment_sums(csa.cpu().numpy(), off2)


def get_alpha_from_distance(D, N, Y, sigma, llambda):
    """kernels.py:127-134 -> fget_alpha_from_distance (fkernels.f90:541-641):
    the molecule kernel sum over atom pairs of exp(-D[b, a] / sigma) from a
    precomputed (na, na) atom distance matrix, plus llambda, inverted from its
    Cholesky factor; returns alpha (sum(N),)."""
    n, off = _counts(N, "get_alpha_from_distance")
    nm = len(n)
    d, _ = to_device(D if is_torch(D) else np.asarray(D, dtype=np.float64), torch.float64)
    if d.dim() != 2 or off[-1] > min(d.shape):
        raise ValueError("get_alpha_from_distance: D must be (na, na) with na >= sum(N)")
    if len(Y) != nm:
        raise ValueError("get_alpha_from_distance: Y must hold one value per molecule")
    if nm == 0:
        return np.zeros(0)
    od = torch.from_numpy(off.astype(np.int32)).to(d.device)
    S = torch.empty((nm, nm), dtype=torch.float64, device=d.device)
    _lib.call("fmlb_segment_exp_sum_f64", _lib.ptr(d), d.stride(0), d.shape[0], d.shape[1],
              _lib.ptr(od), nm, _lib.ptr(od), nm, -1.0 / float(sigma), _lib.ptr(S), nm,
              _lib.stream_handle())
    # S[j, i] = K(i, j): its row-major lower triangle is K's upper one
    _lib.call("fmlb_add_diagonal_f64", _lib.ptr(S), nm, nm, float(llambda), _lib.stream_handle())
    yd, _ = to_device(Y if is_torch(Y) else np.asarray(Y, dtype=np.float64), torch.float64)
    return _explicit_inverse_weights(S, yd, n)


def get_prediction_from_distance(D2, N2, alpha, sigma):
    """kernels.py:110-117 -> fget_prediction_from_distance (fkernels.f90:645-702):
    D2 (na, na2) distances between training and test atoms; Y[j] = sum over
    the atoms i of test molecule j of sum_a exp(-D2[a, i] / sigma) alpha[a].
    Difference: the reference leaves its per-atom accumulator uninitialised
    (no csa = 0 before :688); here it starts at zero."""
    n2, off2 = _counts(N2, "get_prediction_from_distance")
    d2, _ = to_device(D2 if is_torch(D2) else np.asarray(D2, dtype=np.float64), torch.float64)
    if d2.dim() != 2 or off2[-1] > d2.shape[1]:
        raise ValueError("get_prediction_from_distance: D2 must be (na, na2), na2 >= sum(N2)")
    na, na2 = d2.shape
    if len(alpha) < na:
        raise ValueError("get_prediction_from_distance: alpha must hold na weights")
    if na2 == 0:
        return np.zeros(len(n2))
    ad, _ = to_device(alpha if is_torch(alpha) else np.asarray(alpha, dtype=np.float64),
                      torch.float64)
    csa = torch.empty(na2, dtype=torch.float64, device=d2.device)
    lib = _lib.load()
    scratch = torch.empty(lib.fmlb_exp_colsum_scratch_doubles(na2), dtype=torch.float64,
                          device=d2.device)
    _lib.call("fmlb_exp_weighted_colsum_f64", _lib.ptr(d2), d2.stride(0), na, na2,
              -1.0 / float(sigma), _lib.ptr(ad), _lib.ptr(csa), _lib.ptr(scratch),
              _lib.stream_handle())
    return _segment_sums(csa.cpu().numpy(), off2)


def _alpha_inputs(q, z, n, nm=None):
    qa = q if is_torch(q) else np.asarray(q, dtype=np.float64)
    if qa.ndim != 4 or qa.shape[2] != 5 or qa.shape[3] != qa.shape[1]:
        raise ValueError("q must be (nm, amax, 5, amax)")
    nm = qa.shape[0] if nm is None else int(nm)
    amax = qa.shape[1]
    if nm < 0 or nm > qa.shape[0]:
        raise ValueError("nm must lie in 0..%d" % qa.shape[0])
    nn = np.asarray(n.cpu() if is_torch(n) else n, dtype=np.int32).reshape(-1)[:nm]
    if len(nn) != nm or (nm and (nn.min() < 0 or nn.max() > amax)):
        raise ValueError("n must hold nm atom counts in 0..amax")
    x, _ = to_device(qa[:nm], torch.float64)
    zd, _ = to_device(z[:nm] if is_torch(z) else np.asarray(z, dtype=np.float64)[:nm],
                      torch.float64)
    nd, _ = to_device(nn, torch.int32)
    return x, zd, nd, nn, nm, amax


def _arad_fixed_kernel(x, zd, nd, nm, amax, sigma, lam):
    K = torch.empty((nm, nm), dtype=torch.float64, device=device())
    ws = workspace(_lib.load().fmlb_arad_workspace_bytes(nm, nm, amax, 1))
    _lib.call("fmlb_arad_alpha_kernel_f64", _lib.ptr(x), _lib.ptr(zd), _lib.ptr(nd), nm, amax,
              float(sigma), float(lam), _lib.ptr(K), _lib.ptr(ws), ws.numel(),
              _lib.stream_handle())
    return K


def fget_kernel_arad(q, z, n, sigma, nm):
    """The routine fml.kernels exports from its Fortran (farad_kernels.f90:95-227;
    f2py argument order): the symmetric ARAD kernel (nm, nm) of the first nm
    molecules for one sigma, with the routine's fixed width 0.2, cut 6,
    r_width 1, c_width 0.5 and eps 1e-11 (the matrix fget_alpha_arad factors,
    without lambda)."""
    x, zd, nd, nn, nm, amax = _alpha_inputs(q, z, n, nm)
    if nm == 0:
        return np.zeros((0, 0))
    if sigma <= 0:
        raise ValueError("sigma must be positive")
    return to_output(_arad_fixed_kernel(x, zd, nd, nm, amax, sigma, 0.0), not is_torch(q))


def fget_alpha_arad(q, z, n, y, sigma, lambda_, alpha=None):
    """Explicit-inverse ARAD KRR weights, the routine fml.kernels exports from
    its Fortran (farad_kernels.f90:231-436; the f2py argument order is kept).

    q (nm, amax, 5, amax) ARAD descriptors, z (nm, amax, 2) PTP rows/columns,
    n (nm,) atom counts, y (nm,) properties. Builds K + lambda I (the routine's
    fixed ARAD parameters), inverts it from its Cholesky factor (dpotrf +
    dpotri) and multiplies by y (dsymv), all on the GPU; every atom of
    molecule j gets inv(K + lambda I)[j] . y. ``alpha`` (sum(n),) is filled in
    place as f2py's intent(inout) does; without it a new array is returned.
    A non-positive pivot prints the reference's DPOTRF warning as a
    CholeskyWarning, and the weights are NaN.
    """
    x, zd, nd, nn, nm, amax = _alpha_inputs(q, z, n)
    if len(y) != nm:
        raise ValueError("y must hold one value per molecule")
    yd, _ = to_device(y if is_torch(y) else np.asarray(y, dtype=np.float64), torch.float64)
    K = _arad_fixed_kernel(x, zd, nd, nm, amax, sigma, lambda_)
    vals = _explicit_inverse_weights(K, yd, nn)  # :391-432
    if alpha is None:
        return vals
    if len(alpha) < len(vals):
        raise ValueError("alpha must hold sum(n) = %d entries" % len(vals))
    alpha[:] = 0.0
    alpha[:len(vals)] = vals
    return None


def get_atomic_kernels_arad(X1, X2, Z1, Z2, sigmas, width=0.2, cut_distance=6.0, r_width=1.0,
                            c_width=0.5, precision="fp64"):
    """Kernels (nsigma, nm1, nm2) between two sets of ARAD descriptors."""
    amax = X1.shape[1]
    # the reference's argument checks, kernels.py:251-259
    assert X1.shape[3] == amax, "ERROR: Check ARAD decriptor sizes! code = 1"
    assert X2.shape[1] == amax, "ERROR: Check ARAD decriptor sizes! code = 2"
    assert X2.shape[3] == amax, "ERROR: Check ARAD decriptor sizes! code = 3"
    assert X1.shape[0] == len(Z1), "ERROR: Check ARAD decriptor sizes! code = 4"
    assert X2.shape[0] == len(Z2), "ERROR: Check ARAD decriptor sizes! code = 5"
    return _arad(X1, X2, Z1, Z2, sigmas, width, cut_distance, r_width, c_width, False, precision)


def get_atomic_symmetric_kernels_arad(X1, Z1, sigmas, width=0.2, cut_distance=6.0, r_width=1.0,
                                      c_width=0.5, precision="fp64"):
    """Kernels (nsigma, nm1, nm1) of one set with itself (i <= j computed, mirrored)."""
    amax = X1.shape[1]
    assert X1.shape[3] == amax, "ERROR: Check ARAD decriptor sizes! code = 1"
    assert X1.shape[0] == len(Z1), "ERROR: Check ARAD decriptor sizes! code = 4"
    return _arad(X1, None, Z1, None, sigmas, width, cut_distance, r_width, c_width, True,
                 precision)


def _vector_kernels(kind, x1, x2, n1, n2, sigmas):
    """x1 (nm1, amax1, d), x2 (nm2, amax2, d) float64 rows -> (nsig, nm1, nm2)."""
    sig, _ = _sigma_list(sigmas)
    if len(sig) > 32:
        raise ValueError("at most 32 sigmas per call")
    if any(v <= 0.0 for v in sig):
        raise ValueError("sigmas must be positive")
    nm1, amax1, d = x1.shape
    nm2, amax2, d2 = x2.shape
    if d != d2:
        raise ValueError("descriptor sizes differ: %d vs %d" % (d, d2))
    n1 = np.asarray(n1, dtype=np.int32).reshape(-1)
    n2 = np.asarray(n2, dtype=np.int32).reshape(-1)
    if len(n1) != nm1 or len(n2) != nm2:
        raise ValueError("atom-count lists do not match the number of molecules")
    for n, amax in ((n1, amax1), (n2, amax2)):
        if len(n) and (n.min() < 0 or n.max() > amax):
            raise ValueError("atom counts must lie in 0..%d" % amax)
    if max(amax1, amax2) > 128:
        raise ValueError("at most 128 atoms per molecule")
    dev = device()
    K = torch.empty((len(sig), nm1, nm2), dtype=torch.float64, device=dev)
    if nm1 == 0 or nm2 == 0:
        return K
    n1d = torch.from_numpy(n1).to(dev)
    n2d = torch.from_numpy(n2).to(dev)
    sig_p, _keep = _lib.host_doubles(sig)
    _lib.call("fmlb_vector_kernels_f64", kind, _lib.ptr(x1), _lib.ptr(n1d), nm1, max(amax1, 1),
              _lib.ptr(x2), _lib.ptr(n2d), nm2, max(amax2, 1), d, sig_p, len(sig),
              _lib.ptr(K), None, _lib.stream_handle())
    return K


def _atom_rows(x):
    """(d, amax, nm) reference layout, x[f, ia, i] -> (nm, amax, d) on the device."""
    if is_torch(x):
        t = x.to(device=device(), dtype=torch.float64)
        return t.permute(2, 1, 0).contiguous(), False
    a = np.asarray(x, dtype=np.float64)
    if a.ndim != 3:
        raise ValueError("expected a 3-D descriptor array (d, amax, nm)")
    rows, _ = to_device(np.ascontiguousarray(a.transpose(2, 1, 0)), torch.float64)
    return rows, True


def get_atomic_kernels_laplacian(x1, x2, N1, N2, sigmas):
    """kernels.py:351-363 -> (nsigmas, nm1, nm2) float64.

    ``x1``/``x2`` are (d, amax, nm) (x[f, ia, i], the reference's Fortran
    argument layout); ``N1``/``N2`` the atoms per molecule.
    K[k, i, j] = sum over atom pairs of exp(-|x1_ia - x2_ja|_1 / sigma_k).
    """
    a, as_np = _atom_rows(x1)
    b = a if x2 is x1 else _atom_rows(x2)[0]
    return to_output(_vector_kernels(1, a, b, N1, N2, sigmas), as_np)


def fget_vector_kernels_gaussian(q1, q2, n1, n2, sigmas, nm1, nm2, nsigmas):
    """The routine fml.kernels exports from its Fortran (fkernels.f90:93-162;
    f2py argument order): q1 / q2 (d, amax, nm) per-atom descriptors, n1 / n2
    atoms per molecule -> (nsigmas, nm1, nm2), K[k, i, j] = sum over atom pairs
    of exp(-|q1_ia - q2_ja|^2 / (2 sigma_k^2))."""
    if len(n1) != nm1 or len(n2) != nm2 or len(np.atleast_1d(sigmas)) != nsigmas:
        raise ValueError("nm1 / nm2 / nsigmas do not match n1 / n2 / sigmas")
    a, as_np = _atom_rows(q1)
    b = a if q2 is q1 else _atom_rows(q2)[0]
    return to_output(_vector_kernels(0, a, b, n1, n2, sigmas), as_np)


def _local_cm_rows(mols):
    n = np.array([m.natoms for m in mols], dtype=np.int32)
    amax = int(n.max()) if len(n) else 1
    size = mols[0].local_coulomb_matrix.shape[1]
    x = np.zeros((len(mols), amax, size), dtype=np.float64)
    for i, m in enumerate(mols):
        x[i, :n[i], :size] = np.asarray(m.local_coulomb_matrix)
    return to_device(x, torch.float64)[0], n


def get_atomic_kernels_gaussian(mols1, mols2, sigmas):
    """kernels.py:379-411 -> (nsigmas, nm1, nm2) float64 numpy.

    Uses each molecule's ``local_coulomb_matrix`` (``Molecule.
    generate_local_coulomb_matrix``). K[k, i, j] = sum over atom pairs of
    exp(-|x1_ia - x2_ja|^2 / (2 sigma_k^2)).
    """
    a, n1 = _local_cm_rows(mols1)
    b, n2 = (a, n1) if mols2 is mols1 else _local_cm_rows(mols2)
    return to_output(_vector_kernels(0, a, b, n1, n2, sigmas), True)
