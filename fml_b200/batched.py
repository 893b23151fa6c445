"""Batched uneven KRR: many independent problems trained and evaluated at once.

Each problem is the reference's user-side KRR — kernel matrix
(fml/kernels/kernels.py), ``cho_solve`` (fml/math/cho_solve.py), prediction —
with its own training size, sigma and lambda. Problems up to
``split_threshold`` training points run together in ONE persistent launch
(``fmlb_krr_batched_f64``: one CTA per SM pulling whole problems from a device
queue, largest first); larger problems run the multi-CTA pipeline
(``KRRPipeline``'s kernels) on a second stream meanwhile. ``run`` can be
captured into a CUDA graph and replayed. ``split_threshold`` and the grid come
from ``fml_b200.autotune`` unless given.

Problem kinds:
* ``GaussianProblem`` — descriptor rows (n, d) / (nt, d), Gaussian kernel
  built on the device;
* ``PrecomputedProblem`` — kernel matrices given (for example the ARAD kernel
  from ``get_atomic_symmetric_kernels_arad`` / ``get_atomic_kernels_arad``).
"""

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import device

PROBLEM_DTYPE = np.dtype([
    ("x_train", "<i8"), ("x_test", "<i8"), ("y", "<i8"), ("pred", "<i8"), ("kbuf", "<i8"),
    ("work", "<i8"), ("ktest", "<i8"), ("n", "<i4"), ("nt", "<i4"), ("kind", "<i4"),
    ("pad", "<i4"), ("sigma", "<f8"), ("lambda", "<f8")])


@dataclass
class GaussianProblem:
    X_train: np.ndarray  # (n, d) descriptor rows
    y: np.ndarray        # (n,)
    X_test: np.ndarray   # (nt, d)
    sigma: float
    lam: float


@dataclass
class PrecomputedProblem:
    K: np.ndarray        # (n, n) training kernel (lower triangle used)
    K_test: np.ndarray   # (nt, n)
    y: np.ndarray
    lam: float


class BatchedKRR:
    def __init__(self, problems, split_threshold=None, grid=None):
        lib = _lib.load()
        assert lib.fmlb_batch_problem_bytes() == PROBLEM_DTYPE.itemsize
        self.dev = device()
        self.problems = list(problems)
        gauss = [p for p in self.problems if isinstance(p, GaussianProblem)]
        self.d = gauss[0].X_train.shape[1] if gauss else 1
        if split_threshold is None or grid is None:
            from .autotune import batched_config
            cfg = batched_config(self.problems)
            split_threshold = cfg["split_threshold"] if split_threshold is None else split_threshold
            grid = cfg["grid"] if grid is None else grid
        self.split_threshold = int(split_threshold)
        self.grid = int(grid)
        self._pack()

    # ------------------------------------------------------------------ layout
    def _pack(self):
        lib = _lib.load()
        d = self.d
        xrows, yparts, recs = [], [], []
        xoff = yoff = poff = boff = 0
        self.small, self.big = [], []
        for i, p in enumerate(self.problems):
            rec = np.zeros(1, dtype=PROBLEM_DTYPE)[0]
            if isinstance(p, GaussianProblem):
                n, nt = p.X_train.shape[0], p.X_test.shape[0]
                rec["kind"] = 0
                rec["x_train"], rec["x_test"] = xoff, xoff + n
                xrows += [np.asarray(p.X_train, np.float64), np.asarray(p.X_test, np.float64)]
                xoff += n + nt
                rec["sigma"] = p.sigma
            else:
                n, nt = p.K.shape[0], p.K_test.shape[0]
                rec["kind"] = 1
            rec["n"], rec["nt"], rec["lambda"] = n, nt, p.lam
            rec["y"], rec["pred"] = yoff, poff
            yparts.append(np.asarray(p.y, np.float64))
            yoff += n
            poff += nt
            rec["kbuf"] = boff
            rec["work"] = boff + n * n
            boff += lib.fmlb_batch_buffer_doubles(n)
            if rec["kind"] == 1:
                rec["ktest"] = boff
                boff += nt * n
            recs.append(rec)
            (self.big if (rec["kind"] == 0 and n > self.split_threshold) else self.small).append(i)
        self.recs = np.array(recs, dtype=PROBLEM_DTYPE)
        f64 = dict(dtype=torch.float64, device=self.dev)
        X = np.concatenate(xrows) if xrows else np.zeros((1, d))
        self.X = torch.from_numpy(np.ascontiguousarray(X)).to(self.dev)
        self.Y = torch.from_numpy(np.concatenate(yparts)).to(self.dev)
        self.pred = torch.zeros(max(poff, 1), **f64)
        self.buf = torch.zeros(max(boff, 1), **f64)
        self.info = torch.zeros(len(self.problems), dtype=torch.int32, device=self.dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=self.dev)
        # precomputed kernels: the pristine copies (the factorisation overwrites buf)
        self._pre = []
        for i, p in enumerate(self.problems):
            if isinstance(p, PrecomputedProblem):
                r = self.recs[i]
                n, nt = int(r["n"]), int(r["nt"])
                src = torch.from_numpy(np.ascontiguousarray(p.K, np.float64)).to(self.dev)
                srct = torch.from_numpy(np.ascontiguousarray(p.K_test, np.float64)).to(self.dev)
                self.buf[int(r["ktest"]):int(r["ktest"]) + nt * n].copy_(srct.reshape(-1))
                self._pre.append((int(r["kbuf"]), n, src))
        small = sorted(self.small, key=lambda i: -int(self.recs[i]["n"]))
        self.order = torch.tensor(small if small else [0], dtype=torch.int32, device=self.dev)
        self.nsmall = len(small)
        self.recs_dev = torch.from_numpy(self.recs.view(np.uint8).copy()).to(self.dev)
        # multi-CTA path for the large problems
        self._big = []
        for i in self.big:
            r = self.recs[i]
            n = int(r["n"])
            work = torch.empty(lib.fmlb_potrf_workspace_bytes(n), dtype=torch.uint8,
                               device=self.dev)
            pw = torch.empty(lib.fmlb_kernel_predict_workspace_bytes(max(int(r["nt"]), 1), n, 1),
                             dtype=torch.uint8, device=self.dev)
            sig = (ctypes.c_double * 1)(float(r["sigma"]))
            self._big.append((i, work, pw, sig))
        self.stream2 = torch.cuda.Stream(device=self.dev)

    # ------------------------------------------------------------------ running
    def _launch(self):
        P = _lib.ptr
        cur = torch.cuda.current_stream()
        st = _lib.stream_handle(cur)
        for off, n, src in self._pre:  # restore precomputed kernels
            self.buf[off:off + n * n].copy_(src.reshape(-1))
        if self._big:
            self.stream2.wait_stream(cur)
        _lib.call("fmlb_krr_batched_f64", P(self.recs_dev), P(self.order), self.nsmall,
                  P(self.counter), P(self.X), self.d, self.d, P(self.Y), P(self.pred),
                  P(self.buf), P(self.info), self.grid, st)
        if self._big:
            s2 = _lib.stream_handle(self.stream2)
            d = self.d
            with torch.cuda.stream(self.stream2):
                for i, work, pw, sig in self._big:
                    r = self.recs[i]
                    n, nt = int(r["n"]), int(r["nt"])
                    K = self.buf[int(r["kbuf"]):int(r["kbuf"]) + n * n]
                    alpha = self.buf[int(r["work"]):int(r["work"]) + n]
                    xtr = self.X[int(r["x_train"]):int(r["x_train"]) + n]
                    xte = self.X[int(r["x_test"]):int(r["x_test"]) + nt]
                    sp = ctypes.cast(sig, ctypes.POINTER(ctypes.c_double))
                    _lib.call("fmlb_gaussian_kernel_f64", P(xtr), n, d, P(xtr), n, d, d, sp, 1,
                              P(K), n, n * n, 1, s2)
                    _lib.call("fmlb_add_diagonal_f64", P(K), n, n, float(r["lambda"]), s2)
                    _lib.call("fmlb_potrf_f64", P(K), n, n, P(work), P(self.info[i:i + 1]), s2)
                    alpha.copy_(self.Y[int(r["y"]):int(r["y"]) + n])
                    _lib.call("fmlb_potrs_f64", P(K), n, n, P(work), P(alpha), s2)
                    if nt:
                        _lib.call("fmlb_kernel_predict_f64", 0, P(xte), nt, d, P(xtr), n, d, d,
                                  sp, 1, P(alpha), n, P(self.pred[int(r["pred"]):]), nt, P(pw),
                                  pw.numel(), s2)
            cur.wait_stream(self.stream2)

    def run(self):
        """One batched pass on the current stream (capturable)."""
        self._launch()

    def capture(self):
        """Capture one pass into a CUDA graph; returns the graph (replay())."""
        self._launch()  # warm-up: sets kernel attributes and lookahead streams
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        return g

    def predictions(self):
        pred = self.pred.cpu().numpy()
        return [pred[int(r["pred"]):int(r["pred"]) + int(r["nt"])] for r in self.recs]

    def infos(self):
        return self.info.cpu().numpy()

    def launches_per_run(self):
        """Kernel launches of one pass: the persistent kernel + the multi-CTA path."""
        from .krr import potrf_launches
        count = 1
        for i, *_ in self._big:
            r = self.recs[i]
            n = int(r["n"])
            count += 1 + 1 + potrf_launches(n) + 2 * -(-n // 128) + (2 if int(r["nt"]) else 0)
        return count
