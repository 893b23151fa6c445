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
  built inside the persistent launch;
* ``AradProblem`` — ARAD descriptors (n, amax, 5, amax) and charges; the ARAD
  kernels (training, symmetric, and test x training) are built by
  ``fmlb_arad_kernels`` launches inside the same pass (and graph), spread over
  a few side streams, before the solve;
* ``PrecomputedProblem`` — kernel matrices given.
"""

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import device
from .kernels import PRECISIONS, _ptp_arrays, arad_launches

PROBLEM_DTYPE = np.dtype([
    ("x_train", "<i8"), ("x_test", "<i8"), ("y", "<i8"), ("pred", "<i8"), ("kbuf", "<i8"),
    ("work", "<i8"), ("ktest", "<i8"), ("n", "<i4"), ("nt", "<i4"), ("kind", "<i4"),
    ("pad", "<i4"), ("sigma", "<f8"), ("lambda", "<f8")])

ARAD_STREAMS = 4


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


@dataclass
class AradProblem:
    X_train: object      # (n, amax, 5, amax) ARAD descriptors (numpy or device tensor)
    Z_train: list        # n arrays of nuclear charges
    y: np.ndarray        # (n,)
    X_test: object       # (nt, amax, 5, amax)
    Z_test: list
    sigma: float
    lam: float
    width: float = 0.2
    cut_distance: float = 6.0
    r_width: float = 1.0
    c_width: float = 0.5
    precision: str = "fp32"


def n_train_of(p):
    if isinstance(p, GaussianProblem):
        return p.X_train.shape[0]
    if isinstance(p, AradProblem):
        return len(p.Z_train)
    return p.K.shape[0]


class BatchedKRR:
    def __init__(self, problems, split_threshold=None, grid=None):
        lib = _lib.load()
        assert lib.fmlb_batch_problem_bytes() == PROBLEM_DTYPE.itemsize
        self.dev = device()
        self.problems = list(problems)
        gauss = [p for p in self.problems if isinstance(p, GaussianProblem)]
        self.d = gauss[0].X_train.shape[1] if gauss else 1
        self._pack()
        self.stream2 = torch.cuda.Stream(device=self.dev)
        self.side = [torch.cuda.Stream(device=self.dev) for _ in range(ARAD_STREAMS)]
        self._big_ws = {}
        self._pristine = None
        if split_threshold is None or grid is None:
            from .autotune import DEFAULT, batched_config
            self.configure(DEFAULT["split_threshold"], DEFAULT["grid"])
            cfg = batched_config(self.problems, batch=self)
            split_threshold = cfg["split_threshold"] if split_threshold is None else split_threshold
            grid = cfg["grid"] if grid is None else grid
        self.configure(split_threshold, grid)

    # ------------------------------------------------------------------ layout
    def _pack(self):
        lib = _lib.load()
        d = self.d
        xrows, yparts, recs = [], [], []
        xoff = yoff = poff = boff = 0
        for p in self.problems:
            rec = np.zeros(1, dtype=PROBLEM_DTYPE)[0]
            if isinstance(p, GaussianProblem):
                n, nt = p.X_train.shape[0], p.X_test.shape[0]
                if p.X_train.shape[1] != d or (nt and p.X_test.shape[1] != d):
                    raise ValueError("all Gaussian problems must share the descriptor length")
                rec["kind"] = 0
                rec["x_train"], rec["x_test"] = xoff, xoff + n
                xrows += [np.asarray(p.X_train, np.float64), np.asarray(p.X_test, np.float64)]
                xoff += n + nt
                rec["sigma"] = p.sigma
            elif isinstance(p, AradProblem):
                n, nt = len(p.Z_train), len(p.Z_test)
                rec["kind"] = 1
                rec["sigma"] = p.sigma
            else:
                n, nt = p.K.shape[0], p.K_test.shape[0]
                rec["kind"] = 1
            if n < 1:
                raise ValueError("every problem needs at least one training point")
            if len(p.y) != n:
                raise ValueError("y has %d entries for %d training points" % (len(p.y), n))
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
        self.recs = np.array(recs, dtype=PROBLEM_DTYPE)
        f64 = dict(dtype=torch.float64, device=self.dev)
        X = np.concatenate(xrows) if xrows else np.zeros((1, d))
        self.X = torch.from_numpy(np.ascontiguousarray(X)).to(self.dev)
        self.Y = torch.from_numpy(np.concatenate(yparts)).to(self.dev)
        self.pred = torch.zeros(max(poff, 1), **f64)
        self.buf = torch.zeros(max(boff, 1), **f64)
        self.info = torch.zeros(len(self.problems), dtype=torch.int32, device=self.dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.recs_dev = torch.from_numpy(self.recs.view(np.uint8).copy()).to(self.dev)
        # precomputed kernels: the pristine copies (the factorisation overwrites buf)
        self._pre = []
        self._arad = []
        ws_need = [0] * ARAD_STREAMS
        for i, p in enumerate(self.problems):
            r = self.recs[i]
            n, nt = int(r["n"]), int(r["nt"])
            if isinstance(p, PrecomputedProblem):
                src = torch.from_numpy(np.ascontiguousarray(p.K, np.float64)).to(self.dev)
                srct = torch.from_numpy(np.ascontiguousarray(p.K_test, np.float64)).to(self.dev)
                self.buf[int(r["ktest"]):int(r["ktest"]) + nt * n].copy_(srct.reshape(-1))
                self._pre.append((int(r["kbuf"]), n, src))
            elif isinstance(p, AradProblem):
                self._arad.append(self._stage_arad(i, p, ws_need))
        self.arad_ws = [torch.empty(max(b, 256), dtype=torch.uint8, device=self.dev)
                        for b in ws_need]

    def _stage_arad(self, i, p, ws_need):
        lib = _lib.load()
        if p.precision not in PRECISIONS:
            raise ValueError("precision must be 'fp64' or 'fp32'")
        X1 = torch.as_tensor(p.X_train).to(device=self.dev, dtype=torch.float64).contiguous()
        X2 = torch.as_tensor(p.X_test).to(device=self.dev, dtype=torch.float64).contiguous()
        amax = X1.shape[1]
        if X1.dim() != 4 or X1.shape[3] != amax or X1.shape[2] != 5 or \
                (len(p.Z_test) and tuple(X2.shape[1:]) != tuple(X1.shape[1:])):
            raise ValueError("ARAD descriptors must be (n, amax, 5, amax)")
        z1, n1 = _ptp_arrays(p.Z_train, amax)
        z2, n2 = _ptp_arrays(p.Z_test, amax)
        n, nt = len(p.Z_train), len(p.Z_test)
        j = len(self._arad) % ARAD_STREAMS
        ws_need[j] = max(ws_need[j], lib.fmlb_arad_workspace_bytes(n, n, amax, 1),
                         lib.fmlb_arad_workspace_bytes(nt, n, amax, 0))
        t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(self.dev, dt)  # noqa: E731
        sig = (ctypes.c_double * 1)(float(p.sigma))
        return dict(i=i, j=j, n=n, nt=nt, amax=amax, X1=X1, X2=X2,
                    Z1=t(z1, torch.float64), N1=t(n1, torch.int32),
                    Z2=t(z2, torch.float64), N2=t(n2, torch.int32), sig=sig,
                    prec=PRECISIONS[p.precision], precision=p.precision,
                    params=(float(p.width), float(p.cut_distance), float(p.r_width),
                            float(p.c_width)))

    def configure(self, split_threshold, grid):
        """Choose which problems take the multi-CTA path and the persistent grid."""
        lib = _lib.load()
        self.split_threshold = int(split_threshold)
        self.grid = int(grid)
        self.small, self.big = [], []
        for i, r in enumerate(self.recs):
            (self.big if int(r["n"]) > self.split_threshold else self.small).append(i)
        small = sorted(self.small, key=lambda i: -int(self.recs[i]["n"]))
        self.order = torch.tensor(small if small else [0], dtype=torch.int32, device=self.dev)
        self.nsmall = len(small)
        self._big = []
        for i in self.big:
            r = self.recs[i]
            n, nt = int(r["n"]), int(r["nt"])
            if i not in self._big_ws:
                work = torch.empty(lib.fmlb_potrf_workspace_bytes(n), dtype=torch.uint8,
                                   device=self.dev)
                pw = torch.empty(lib.fmlb_kernel_predict_workspace_bytes(max(nt, 1), n, 1),
                                 dtype=torch.uint8, device=self.dev)
                self._big_ws[i] = (work, pw, (ctypes.c_double * 1)(float(r["sigma"])))
            self._big.append((i,) + self._big_ws[i])

    # ------------------------------------------------------------------ running
    def _arad_builds(self, cur):
        P = _lib.ptr
        for s in self.side:
            s.wait_stream(cur)
        for a in self._arad:
            r = self.recs[a["i"]]
            n, nt = a["n"], a["nt"]
            st = _lib.stream_handle(self.side[a["j"]])
            ws = self.arad_ws[a["j"]]
            sp = ctypes.cast(a["sig"], ctypes.POINTER(ctypes.c_double))
            _lib.call("fmlb_arad_kernels", P(a["X1"]), P(a["Z1"]), P(a["N1"]), n, None, None,
                      None, n, a["amax"], sp, 1, *a["params"], 1, a["prec"],
                      P(self.buf[int(r["kbuf"]):]), P(ws), ws.numel(), st)
            if nt:
                _lib.call("fmlb_arad_kernels", P(a["X2"]), P(a["Z2"]), P(a["N2"]), nt,
                          P(a["X1"]), P(a["Z1"]), P(a["N1"]), n, a["amax"], sp, 1, *a["params"],
                          0, a["prec"], P(self.buf[int(r["ktest"]):]), P(ws), ws.numel(), st)
        for s in self.side:
            cur.wait_stream(s)

    def keep_kernels(self):
        """Build the ARAD kernels once and keep copies, so that ``run(builds=False)``
        restores them instead of rebuilding (used to time the solve alone)."""
        cur = torch.cuda.current_stream()
        self._arad_builds(cur)
        self._pristine = []
        for a in self._arad:
            r = self.recs[a["i"]]
            off, n = int(r["kbuf"]), a["n"]
            self._pristine.append((off, n, self.buf[off:off + n * n].clone()))
        torch.cuda.synchronize()

    def _launch(self, builds=True):
        P = _lib.ptr
        cur = torch.cuda.current_stream()
        st = _lib.stream_handle(cur)
        if self._arad:
            if builds or self._pristine is None:
                self._arad_builds(cur)
            else:
                for off, n, src in self._pristine:
                    self.buf[off:off + n * n].copy_(src)
        for off, n, src in self._pre:  # restore precomputed kernels
            self.buf[off:off + n * n].copy_(src.reshape(-1))
        if self._big:
            self.stream2.wait_stream(cur)
        if self.nsmall:
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
                    pred = self.pred[int(r["pred"]):]
                    sp = ctypes.cast(sig, ctypes.POINTER(ctypes.c_double))
                    if int(r["kind"]) == 0:
                        xtr = self.X[int(r["x_train"]):int(r["x_train"]) + n]
                        _lib.call("fmlb_gaussian_kernel_f64", P(xtr), n, d, P(xtr), n, d, d, sp,
                                  1, P(K), n, n * n, 1, s2)
                    _lib.call("fmlb_add_diagonal_f64", P(K), n, n, float(r["lambda"]), s2)
                    _lib.call("fmlb_potrf_f64", P(K), n, n, P(work), P(self.info[i:i + 1]), s2)
                    alpha.copy_(self.Y[int(r["y"]):int(r["y"]) + n])
                    _lib.call("fmlb_potrs_f64", P(K), n, n, P(work), P(alpha), s2)
                    if not nt:
                        continue
                    if int(r["kind"]) == 0:
                        xte = self.X[int(r["x_test"]):int(r["x_test"]) + nt]
                        _lib.call("fmlb_kernel_predict_f64", 0, P(xte), nt, d, P(xtr), n, d, d,
                                  sp, 1, P(alpha), n, P(pred), nt, P(pw), pw.numel(), s2)
                    else:
                        _lib.call("fmlb_gemv_f64", P(self.buf[int(r["ktest"]):]), n, nt, n,
                                  P(alpha), P(pred), s2)
            cur.wait_stream(self.stream2)

    def run(self, builds=True):
        """One batched pass on the current stream (capturable)."""
        self._launch(builds)

    def capture(self, builds=True):
        """Capture one pass into a CUDA graph; returns the graph (replay())."""
        self._launch(builds)  # warm-up: sets kernel attributes and lookahead streams
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch(builds)
        return g

    def predictions(self):
        pred = self.pred.cpu().numpy()
        return [pred[int(r["pred"]):int(r["pred"]) + int(r["nt"])] for r in self.recs]

    def infos(self):
        return self.info.cpu().numpy()

    def launches_per_run(self):
        """Kernel launches of one pass: ARAD builds, the persistent kernel and the
        multi-CTA path."""
        from .krr import potrf_launches
        count = 1 if self.nsmall else 0
        for a in self._arad:
            count += arad_launches(True, a["precision"], a["amax"], 1)
            if a["nt"]:
                count += arad_launches(False, a["precision"], a["amax"], 1)
        for i, *_ in self._big:
            r = self.recs[i]
            n = int(r["n"])
            count += (1 if int(r["kind"]) == 0 else 0) + 1 + potrf_launches(n) + \
                2 * -(-n // 128) + (1 if int(r["nt"]) else 0)
            if int(r["kind"]) == 0 and int(r["nt"]):
                count += 1  # the prediction's chunk reduction
        return count
