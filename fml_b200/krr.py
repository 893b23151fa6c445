"""Kernel-ridge regression on the GPU, FP64-accurate path.

The user-side KRR the reference's README composes (fml/fml.py descriptors,
fml/kernels/kernels.py kernel, fml/math/cho_solve.py solve, ``K_test @
alpha`` prediction) as one device pipeline:

    sorted Coulomb matrices (one launch for all molecules)
    -> K_train for every sigma (symmetric FP64 build, one pass)
    -> K + lambda I -> Cholesky factor -> solve, per sigma
    -> fused prediction sum_t k(x_q, x_t) alpha_t for every sigma

``KRRPipeline`` owns every device buffer, so ``run`` allocates nothing and can
be timed or captured; ``krr_fit_predict`` is the public one-call form that
takes host (numpy) or device (torch) molecules and returns predictions.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._tensors import device, to_device, to_output

KINDS = {"gaussian": 0, "laplacian": 1}
PANEL = 128  # inner panel width of the FP64 factorisation (NB in cholesky_f64.cu)


def outer_panel(n):
    """Outer panel width of the FP64 factorisation (outer_width in cholesky_f64.cu)."""
    return 8 * PANEL if n >= 16384 else 4 * PANEL if n >= 8192 else 2 * PANEL


def potrf_launches(n, ozaki=False):
    """Kernel launches of fmlb_potrf_f64 / fmlb_potrf_ozaki_f64 for an n x n
    matrix (mirrors their loops)."""
    W = outer_panel(n)
    count = 0
    for K0 in range(0, n, W):
        end = min(K0 + W, n)
        for k0 in range(K0, end, PANEL):
            count += 1 + (1 if n - k0 - PANEL > 0 else 0)  # diagonal block + panel solve
            count += 1 if end - (k0 + PANEL) > 0 else 0     # rest of the outer panel
        if K0 > 0:
            count += 1 + (1 if ozaki else 0)                 # strip (+ digit split)
    for K0 in range(0, n - W, W):
        count += 1 if n - (K0 + 2 * W) > 0 else 0           # bulk update
    return count


class KRRPipeline:
    """Preallocated FP64 KRR: ``n_train`` training and ``n_mol - n_train`` test molecules.

    The first ``n_train`` molecules of the batch are the training set.

    ``factor="fp64"`` factors on the FP64 tensor cores; ``factor="ozaki"``
    runs the trailing updates on the int8 tensor cores (``slices`` digit
    planes) and is followed by ``refine`` double-double refinement steps
    (default 2 for it, 0 for the FP64 factor). With ``refine`` > 0 the
    relative residual ||y - (K + lambda I) alpha|| / ||y|| before each step
    and after the last is kept per sigma in ``resid`` (device, divided by
    ||y|| by ``relative_residuals``).
    """

    def __init__(self, n_mol, n_train, size, sigmas, lam, kind="gaussian", factor="fp64",
                 slices=6, refine=None):
        lib = _lib.load()
        self.dev = device()
        self.n_mol, self.n_train, self.n_test = n_mol, n_train, n_mol - n_train
        self.size = size
        self.d = size * (size + 1) // 2
        self.sigmas = [float(s) for s in sigmas]
        self.nsig = len(self.sigmas)
        if not 1 <= self.nsig <= 8:
            raise ValueError("1..8 sigmas per pipeline")
        self.lam = float(lam)
        self.kind = KINDS[kind]
        f64 = dict(dtype=torch.float64, device=self.dev)
        n = n_train
        self.X = torch.empty((n_mol, self.d), **f64)
        self.K = torch.empty((self.nsig, n, n), **f64)
        if factor not in ("fp64", "ozaki"):
            raise ValueError("factor must be 'fp64' or 'ozaki'")
        self.factor, self.slices = factor, int(slices)
        self.refine = (2 if factor == "ozaki" else 0) if refine is None else int(refine)
        if factor == "ozaki":
            wb = lib.fmlb_potrf_ozaki_workspace_bytes(n, self.slices)
        else:
            wb = lib.fmlb_potrf_workspace_bytes(n)
        self.work = torch.empty((self.nsig, wb), dtype=torch.uint8, device=self.dev)
        # the diagonal of K + lambda I is kept for the residual: the factor
        # overwrites it, K's strict upper triangle stays in place
        self.diag = torch.empty((self.nsig, n), **f64)
        self.ytr = torch.empty(n, **f64)
        self.scratch = None
        if self.refine > 0:
            self.alpha_lo = torch.empty((self.nsig, n), **f64)
            self._alloc_scratch()
            self.resid = torch.zeros((self.nsig, self.refine + 1), **f64)
        self.info = torch.zeros(self.nsig, dtype=torch.int32, device=self.dev)
        self.alpha = torch.empty((self.nsig, n), **f64)
        self.pred = torch.empty((self.nsig, max(self.n_test, 1)), **f64)
        pb = lib.fmlb_kernel_predict_workspace_bytes(max(self.n_test, 1), n, self.nsig)
        self.pwork = torch.empty(pb, dtype=torch.uint8, device=self.dev)
        self._sig_arr = (ctypes.c_double * self.nsig)(*self.sigmas)
        self._sig_ptr = ctypes.cast(self._sig_arr, ctypes.POINTER(ctypes.c_double))
        # one stream per sigma: the factorisations overlap, so one's narrow
        # final outer steps run under another's bulk updates
        self._sig_streams = [torch.cuda.Stream(device=self.dev) for _ in range(self.nsig)]
        self._fork = torch.cuda.Event()
        self._joins = [torch.cuda.Event() for _ in range(self.nsig)]

    def launches_per_run(self):
        """Kernel launches of one ``run`` (mirrors the loops in the C library)."""
        nblk = -(-self.n_train // PANEL)
        potrf = potrf_launches(self.n_train, self.factor == "ozaki")
        potrs = 2 * nblk
        per_sigma = 1 + potrf + potrs
        per_sigma += 1  # the kept diagonal
        if self.refine > 0:  # per step 3 residual + 2 norm + potrs + update, final residual
            per_sigma += self.refine * (5 + potrs + 1) + 5
        return 1 + 1 + self.nsig * per_sigma + (2 if self.n_test else 0)

    def _alloc_scratch(self):
        sd = _lib.load().fmlb_krr_refine_dd_scratch_doubles(self.n_train)
        self.scratch = torch.empty((self.nsig, sd), dtype=torch.float64, device=self.dev)

    def relative_residuals(self):
        """(nsigma, refine + 1) host array of ||r|| / ||y|| before each
        refinement step and after the last (refine > 0 only)."""
        if self.refine == 0:
            raise ValueError("the pipeline keeps residuals only with refine > 0")
        ny = float(torch.linalg.vector_norm(self.ytr))
        return self.resid.cpu().numpy() / ny

    def residual_now(self):
        """(nsigma,) host array: ||y - (K + lambda I) alpha|| / ||y|| of the
        current weights, formed in double-double from the factored buffers
        (K's strict upper triangle and the kept diagonal)."""
        if self.scratch is None:
            self._alloc_scratch()
        n = self.n_train
        out = torch.empty((self.nsig, 1), dtype=torch.float64, device=self.dev)
        st = _lib.stream_handle()
        for k in range(self.nsig):
            lo = self.alpha_lo[k] if self.refine > 0 else torch.zeros(n, dtype=torch.float64,
                                                                      device=self.dev)
            _lib.call("fmlb_krr_refine_dd", _lib.ptr(self.K[k]), n, n, _lib.ptr(self.diag[k]),
                      _lib.ptr(self.work[k]), _lib.ptr(self.ytr), _lib.ptr(self.alpha[k]),
                      _lib.ptr(lo), 0, _lib.ptr(out[k]), _lib.ptr(self.scratch[k]), st)
        ny = float(torch.linalg.vector_norm(self.ytr))
        return out[:, 0].cpu().numpy() / ny

    def run_descriptors(self, X, y_train, stream=None):
        """Like ``run`` with the descriptor rows (n_mol, d) given instead of molecules."""
        self.X.copy_(X)
        return self._solve_predict(y_train, stream)

    def run(self, charges, coords, offsets, y_train, stream=None):
        """Device tensors in; predictions (nsigma, n_test) on the device out."""
        s = _lib.stream_handle(stream)
        n, d = self.n_train, self.d
        _lib.call("fmlb_coulomb_matrices", _lib.ptr(charges), _lib.ptr(coords), _lib.ptr(offsets),
                  self.n_mol, self.size, _lib.ptr(self.X), d, None, 0, None, None, s)
        return self._solve_predict(y_train, stream)

    def _solve_predict(self, y_train, stream=None):
        s = _lib.stream_handle(stream)
        n, d = self.n_train, self.d
        fn = "fmlb_gaussian_kernel_f64" if self.kind == 0 else "fmlb_laplacian_kernel_f64"
        _lib.call(fn, _lib.ptr(self.X), n, d, _lib.ptr(self.X), n, d, d, self._sig_ptr, self.nsig,
                  _lib.ptr(self.K), n, n * n, 1, s)
        main = stream if stream is not None else torch.cuda.current_stream(self.dev)
        with torch.cuda.stream(main):
            self.ytr.copy_(y_train)
        self._fork.record(main)
        for k in range(self.nsig):
            Kk = self.K[k]
            sk = self._sig_streams[k]
            sk.wait_event(self._fork)
            h = _lib.stream_handle(sk)
            _lib.call("fmlb_add_diagonal_f64", _lib.ptr(Kk), n, n, self.lam, h)
            _lib.call("fmlb_get_diagonal_f64", _lib.ptr(Kk), n, n, _lib.ptr(self.diag[k]), h)
            if self.factor == "ozaki":
                _lib.call("fmlb_potrf_ozaki_f64", _lib.ptr(Kk), n, n, self.slices,
                          _lib.ptr(self.work[k]), self.work.shape[1],
                          _lib.ptr(self.info[k:k + 1]), h)
            else:
                _lib.call("fmlb_potrf_f64", _lib.ptr(Kk), n, n, _lib.ptr(self.work[k]),
                          _lib.ptr(self.info[k:k + 1]), h)
            with torch.cuda.stream(sk):
                self.alpha[k].copy_(y_train)
            _lib.call("fmlb_potrs_f64", _lib.ptr(Kk), n, n, _lib.ptr(self.work[k]),
                      _lib.ptr(self.alpha[k]), h)
            if self.refine > 0:
                with torch.cuda.stream(sk):
                    self.alpha_lo[k].zero_()
                _lib.call("fmlb_krr_refine_dd", _lib.ptr(Kk), n, n, _lib.ptr(self.diag[k]),
                          _lib.ptr(self.work[k]), _lib.ptr(self.ytr), _lib.ptr(self.alpha[k]),
                          _lib.ptr(self.alpha_lo[k]), self.refine, _lib.ptr(self.resid[k]),
                          _lib.ptr(self.scratch[k]), h)
            self._joins[k].record(sk)
        for ev in self._joins:
            main.wait_event(ev)
        if self.n_test:
            Xq = self.X[n:]
            _lib.call("fmlb_kernel_predict_f64", self.kind, _lib.ptr(Xq), self.n_test, d,
                      _lib.ptr(self.X), n, d, d, self._sig_ptr, self.nsig, _lib.ptr(self.alpha), n,
                      _lib.ptr(self.pred), self.pred.shape[1], _lib.ptr(self.pwork),
                      self.pwork.numel(), s)
        return self.pred[:, :self.n_test]


def krr_fit_predict(charges, coords, offsets, y_train, n_train, sigmas, lam, size=23,
                    kind="gaussian", return_info=False, factor="fp64", slices=6, refine=None):
    """Train on the first ``n_train`` molecules, predict the rest, for every sigma.

    Molecules are packed (charges, coords, offsets). Returns (nsigma, n_test)
    predictions (numpy for numpy input, a device tensor for torch input).
    ``factor``, ``slices`` and ``refine`` as for ``KRRPipeline``.
    """
    off = offsets.cpu().numpy() if isinstance(offsets, torch.Tensor) else np.asarray(offsets)
    n_mol = len(off) - 1
    z, as_np = to_device(charges, torch.float64)
    r, _ = to_device(coords, torch.float64)
    o, _ = to_device(offsets, torch.int32)
    y, _ = to_device(y_train, torch.float64)
    pipe = KRRPipeline(n_mol, n_train, size, np.atleast_1d(sigmas), lam, kind, factor, slices,
                       refine)
    pred = pipe.run(z, r, o, y)
    out = to_output(pred, as_np)
    if return_info:
        return out, pipe.info.cpu().numpy()
    return out
