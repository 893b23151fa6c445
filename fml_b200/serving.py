"""KRR serving loop: trained models resident on the device, continuous
batching of prediction requests, admission by an HBM budget, retraining with
appended data, p50/p99 latency.

The reference has no server; a served prediction is its user-side KRR
prediction (descriptor: fml/fml.py:64-86; kernel: fml/kernels/kernels.py;
``K_test @ alpha``) for a model trained by ``cho_solve``
(fml/math/cho_solve.py), kept on the device between requests.

Design:
* a model keeps its training descriptors, its Cholesky factor, alpha and (for
  ARAD, where rebuilding is expensive) the training kernel matrix on the
  device; CM-Gaussian models rebuild K on retrain (a fast FP64 build);
* prediction requests wait in per-model FIFO queues; whenever a slot (a
  stream with its own pinned staging buffers) is free, the model with the
  oldest waiting request is chosen and as many of its waiting requests as fit
  ``max_batch_molecules`` are merged into ONE batch: one host->device copy,
  one descriptor launch, one kernel/prediction pass, one device->host copy.
  Batches of different models run on different streams and overlap on the
  device; cheap batches (CM) run only on the high-priority streams;
* a batch, or a retrain, is admitted only when the resident models, the slot
  arenas, the retrains in flight and the memory it adds fit the HBM budget;
* retrains (``+m`` molecules appended to a model's training set) run on a
  stream between the CM and ARAD priorities and are launched from a worker
  thread (a retrain
  enqueues thousands of kernels, and a launch into a full queue blocks); the
  model switches to the new version when the retrain completes, batches
  already launched keep the old one;
* each prediction is computed row by row with the same kernels whatever the
  batch it is in, so a request's result is the same alone and in the mix.

The slots only overlap if the CUDA driver gives their streams separate
hardware work queues: set ``CUDA_DEVICE_MAX_CONNECTIONS`` (default 8) to at
least ``max_inflight + 4`` before the process creates its CUDA context, or a
short CM batch can wait behind a long ARAD batch that shares its queue.
"""

import collections
import concurrent.futures
import ctypes
import os
import threading
import time
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import device
from .data import PTP_COL, PTP_ROW
from .kernels import PRECISIONS, arad_launches
from .krr import potrf_launches

ARAD_PARAMS = (0.2, 6.0, 1.0, 0.5)  # width, cut_distance, r_width, c_width (kernels.py defaults)
ARAD_CUT = 5.0                       # descriptor cut of Molecule.generate_arad_descriptor


@dataclass
class Request:
    model: int
    charges: np.ndarray          # packed atoms of the query molecules
    coords: np.ndarray           # (atoms, 3)
    offsets: np.ndarray          # (nmol + 1,)
    arrival: float = 0.0         # seconds after the start of ``serve``
    y: np.ndarray = None         # retrain: targets of the appended molecules
    retrain: bool = False
    rid: int = -1
    result: np.ndarray = None    # predictions (nmol,)
    admitted: float = None
    done: float = None

    @property
    def nmol(self):
        return len(self.offsets) - 1


def _ptp_packed(charges, offsets, amax):
    """PTP (nmol, amax, 2) float64 and atom counts (nmol,) int32 for packed molecules
    (the marshalling of fml/kernels/kernels.py:261-292)."""
    nm = len(offsets) - 1
    counts = np.diff(offsets).astype(np.int32)
    zi = np.asarray(charges).astype(np.int64)
    ptp = np.zeros((nm, amax, 2))
    if len(zi):
        if (zi < 0).any() or (zi > 127).any() or (PTP_ROW[np.clip(zi, 0, 127)] < 0).any():
            raise KeyError("a nuclear charge outside the periodic-table map")
        mol = np.repeat(np.arange(nm), counts)
        slot = np.arange(len(zi)) - np.repeat(offsets[:-1], counts)
        ptp[mol, slot, 0] = PTP_ROW[zi]
        ptp[mol, slot, 1] = PTP_COL[zi]
    return ptp, counts


def _aligned(nbytes):
    return (int(nbytes) + 255) // 256 * 256


def _layout_bytes(specs):
    return sum(_aligned(int(np.prod(shape)) * torch.empty(0, dtype=dt).element_size())
               for shape, dt in specs)


def _carve(buf, specs):
    """Typed views of a uint8 buffer, one per (shape, dtype), 256-byte aligned."""
    out, off = [], 0
    for shape, dt in specs:
        nb = int(np.prod(shape)) * torch.empty(0, dtype=dt).element_size()
        out.append(buf[off:off + nb].view(dt).view(shape))
        off += _aligned(nb)
    return out


class _Version:
    """One trained state of a model (immutable once built)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in self.__dict__.values()
                   if isinstance(t, torch.Tensor))


class Model:
    def __init__(self, mid, kind, size, sigma, lam, precision="fp32"):
        if kind not in ("cm", "arad"):
            raise ValueError("kind must be 'cm' or 'arad'")
        self.mid, self.kind, self.size = mid, kind, int(size)
        self.sigma, self.lam = float(sigma), float(lam)
        self.precision = precision
        self.d = self.size * (self.size + 1) // 2
        self._sig = (ctypes.c_double * 1)(self.sigma)
        self.sig_ptr = ctypes.cast(self._sig, ctypes.POINTER(ctypes.c_double))
        self.version = None
        self.host = None  # training molecules (charges, coords, offsets, y) on the host
        self.retrain_pending = []
        self.retrain_active = None


class KRRServer:
    def __init__(self, hbm_budget=150e9, max_inflight=8, max_batch_molecules=1024,
                 high_priority_slots=3):
        _lib.load()
        self.dev = device()
        self.budget = float(hbm_budget)
        self.max_batch = int(max_batch_molecules)
        self.models = {}
        if max_inflight < 1:
            raise ValueError("max_inflight must be >= 1")
        conn = int(os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8"))
        if conn < max_inflight + 4:
            warnings.warn("CUDA_DEVICE_MAX_CONNECTIONS=%d: streams of the %d slots share hardware "
                          "queues, so batches can wait behind unrelated ones; set it to >= %d "
                          "before CUDA initialises" % (conn, max_inflight, max_inflight + 4))
        # at least one slot takes ARAD batches
        high_priority_slots = min(high_priority_slots, max_inflight - 1)
        pr = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream,
                                                          "priority_range") else (0, -1)
        lo, hi = max(pr), min(pr)  # a lower number is a higher priority
        self.slots = []
        for k in range(max_inflight):
            pri = hi if k < high_priority_slots else lo
            st = torch.cuda.Stream(device=self.dev, priority=pri)
            self.slots.append({"stream": st, "high": k < high_priority_slots, "busy": None,
                               "dev": None, "pin": None})
        # retrains above the ARAD slots: their thousands of small kernels would
        # otherwise wait behind whole ARAD grids and back up the launch queue
        self._have_high = high_priority_slots > 0
        self.retrain_stream = torch.cuda.Stream(device=self.dev, priority=(lo + hi) // 2
                                                if lo - hi >= 2 else hi)
        self.inflight_bytes = 0  # retrains in flight
        self.launches = 0
        self._count_lock = threading.Lock()
        # retrains are launched from one worker thread: a retrain enqueues
        # thousands of kernels, and a launch blocks while the stream's queue
        # is full, which must not stall the admission of prediction batches
        self._retrain_pool = concurrent.futures.ThreadPoolExecutor(
            max_workers=1, thread_name_prefix="fmlb-retrain")
        self._retrain_pool.submit(self._warm_worker).result()
        self.stats = collections.Counter()
        # (kind, host launch s, device s, requests, admitted at, completion seen at)
        self.batch_log = []
        self.retrain_host_s = []  # host seconds spent launching each retrain
        self.phase_max = collections.Counter()  # longest loop iteration / phase (seconds)

    def _warm_worker(self):
        """A 1 x 1 factorisation on the worker thread, outside any capture: it
        creates the library's per-thread lookahead stream and events."""
        torch.cuda.set_device(self.dev)
        lib = _lib.load()
        with torch.cuda.stream(self.retrain_stream):
            A = torch.ones((1, 1), dtype=torch.float64, device=self.dev)
            work = torch.empty(lib.fmlb_potrf_workspace_bytes(1), dtype=torch.uint8,
                               device=self.dev)
            info = torch.zeros(1, dtype=torch.int32, device=self.dev)
            _lib.call("fmlb_potrf_f64", _lib.ptr(A), 1, 1, _lib.ptr(work), _lib.ptr(info),
                      _lib.stream_handle(self.retrain_stream))
        self.retrain_stream.synchronize()

    def _count(self, k):
        with self._count_lock:
            self.launches += k

    # ------------------------------------------------------------------ memory
    def resident_bytes(self):
        total = 0
        for m in self.models.values():
            if m.version is not None:
                total += m.version.nbytes()
        return total

    def arena_bytes(self):
        return sum(sl["dev"].numel() for sl in self.slots if sl["dev"] is not None)

    def _fits(self, nbytes):
        return self.resident_bytes() + self.arena_bytes() + self.inflight_bytes + nbytes <= \
            self.budget

    def _predict_specs(self, m, nq, atoms):
        """(pinned host, device) layouts of one prediction batch."""
        lib = _lib.load()
        f64, i32, u8 = torch.float64, torch.int32, torch.uint8
        n, a = m.version.n, m.size
        pin = [((atoms,), f64), ((atoms, 3), f64), ((nq + 1,), i32), ((nq,), f64)]
        dev = [((atoms,), f64), ((atoms, 3), f64), ((nq + 1,), i32), ((nq,), f64)]
        if m.kind == "cm":
            dev += [((nq, m.d), f64),
                    ((lib.fmlb_kernel_predict_workspace_bytes(nq, n, 1),), u8)]
        else:
            pin += [((nq, a, 2), f64), ((nq,), i32)]
            dev += [((nq, a, 5, a), f64), ((nq, a, 2), f64), ((nq,), i32), ((nq, n), f64),
                    ((lib.fmlb_arad_workspace_bytes(nq, n, a, 0),), u8)]
        return pin, dev

    def reserve(self):
        """Size every slot's arenas for a full batch (``max_batch_molecules`` of
        the largest molecules) of any resident model the slot may serve."""
        for slot in self.slots:
            dev = pin = 0
            for m in self.models.values():
                if slot["high"] and m.kind == "arad":
                    continue
                p, d = self._predict_specs(m, self.max_batch, self.max_batch * m.size)
                dev, pin = max(dev, _layout_bytes(d)), max(pin, _layout_bytes(p))
            extra = dev - (slot["dev"].numel() if slot["dev"] is not None else 0)
            if extra > 0:
                if not self._fits(extra):
                    raise MemoryError("slot arenas do not fit the HBM budget")
                slot["dev"] = None
                slot["dev"] = torch.empty(dev, dtype=torch.uint8, device=self.dev)
            if slot["pin"] is None or slot["pin"].numel() < pin:
                slot["pin"] = torch.empty(pin, dtype=torch.uint8, pin_memory=True)

    def _slot_growth(self, slot, m, nq, atoms):
        need = _layout_bytes(self._predict_specs(m, nq, atoms)[1])
        have = slot["dev"].numel() if slot["dev"] is not None else 0
        return max(0, need - have)

    def _train_bytes(self, m, n_new, m_add):
        lib = _lib.load()
        n = n_new
        b = n * n * 8 + n * 8 + lib.fmlb_potrf_workspace_bytes(n)
        if m.kind == "cm":
            return b + n * m.d * 8
        a = m.size
        return b + n * n * 8 + n * (a * 5 * a + 2 * a) * 8 + n * 4 + m_add * (n + m_add) * 8 + \
            lib.fmlb_arad_workspace_bytes(max(m_add, 1), n, a, 0) + \
            lib.fmlb_arad_workspace_bytes(n, n, a, 1)

    # ------------------------------------------------------------------ descriptors
    def _upload(self, charges, coords, offsets, stream):
        """Pinned host copies -> device, asynchronously on ``stream``."""
        z = torch.from_numpy(np.ascontiguousarray(charges, np.float64)).pin_memory()
        r = torch.from_numpy(np.ascontiguousarray(coords, np.float64).reshape(-1, 3)).pin_memory()
        o = torch.from_numpy(np.ascontiguousarray(offsets, np.int32)).pin_memory()
        with torch.cuda.stream(stream):
            zd = z.to(self.dev, non_blocking=True)
            rd = r.to(self.dev, non_blocking=True)
            od = o.to(self.dev, non_blocking=True)
        return (zd, rd, od), (z, r, o)

    def _describe(self, m, dev_in, nmol, charges, offsets, stream):
        """Descriptor launch for packed molecules; returns device tensors."""
        zd, rd, od = dev_in
        st = _lib.stream_handle(stream)
        P = _lib.ptr
        counts = np.diff(offsets)
        if nmol and counts.max() > m.size:
            raise ValueError("a molecule has %d atoms, more than the model size %d"
                             % (int(counts.max()), m.size))
        with torch.cuda.stream(stream):
            if m.kind == "cm":
                X = torch.empty((nmol, m.d), dtype=torch.float64, device=self.dev)
                _lib.call("fmlb_coulomb_matrices", P(zd), P(rd), P(od), nmol, m.size, P(X), m.d,
                          None, 0, None, None, st)
                self._count(1)
                return {"X": X}
            a = m.size
            X = torch.empty((nmol, a, 5, a), dtype=torch.float64, device=self.dev)
            _lib.call("fmlb_arad_descriptors", P(zd), P(rd), P(od), nmol, a, ARAD_CUT, P(X), None,
                      st)
            ptp, cnt = _ptp_packed(charges, offsets, a)
            Z = torch.from_numpy(ptp).pin_memory().to(self.dev, non_blocking=True)
            N = torch.from_numpy(cnt).pin_memory().to(self.dev, non_blocking=True)
            self._count(1)
            return {"X": X, "Z": Z, "N": N}

    # ------------------------------------------------------------------ training
    def _arad_call(self, m, A, B, out, stream, symmetric):
        """out (nA, nB) = ARAD kernel between prepared sets A and B (dicts X/Z/N)."""
        lib = _lib.load()
        P = _lib.ptr
        a = m.size
        nA = A["X"].shape[0]
        nB = nA if symmetric else B["X"].shape[0]
        ws = torch.empty(max(lib.fmlb_arad_workspace_bytes(nA, nB, a, 1 if symmetric else 0),
                             256), dtype=torch.uint8, device=self.dev)
        if symmetric:
            B = {"X": None, "Z": None, "N": None}
        _lib.call("fmlb_arad_kernels", P(A["X"]), P(A["Z"]), P(A["N"]), nA, P(B["X"]), P(B["Z"]),
                  P(B["N"]), nB, a, m.sig_ptr, 1, *ARAD_PARAMS, 1 if symmetric else 0,
                  PRECISIONS[m.precision], P(out), P(ws), ws.numel(), _lib.stream_handle(stream))
        self._count(arad_launches(symmetric, m.precision, a, 1))
        return ws

    def _factor(self, m, K, y, stream, keep_K, graphs=None):
        """L = chol(K + lam I) (a copy when K is kept), alpha = solve; returns tensors.

        With ``graphs`` (a list) the factorisation and solve are captured into
        one CUDA graph and replayed, so that their thousands of kernels reach
        the GPU as one submission; the graph is appended to ``graphs``.
        """
        lib = _lib.load()
        P = _lib.ptr
        n = K.shape[0]
        with torch.cuda.stream(stream):
            L = K.clone() if keep_K else K
            work = torch.empty(lib.fmlb_potrf_workspace_bytes(n), dtype=torch.uint8,
                               device=self.dev)
            info = torch.zeros(1, dtype=torch.int32, device=self.dev)
            alpha = torch.from_numpy(np.ascontiguousarray(y, np.float64)).pin_memory().to(
                self.dev, non_blocking=True)

        def launches():
            st = _lib.stream_handle(stream)
            _lib.call("fmlb_add_diagonal_f64", P(L), n, n, m.lam, st)
            _lib.call("fmlb_potrf_f64", P(L), n, n, P(work), P(info), st)
            _lib.call("fmlb_potrs_f64", P(L), n, n, P(work), P(alpha), st)

        if graphs is None:
            with torch.cuda.stream(stream):
                launches()
        else:
            # capture_begin/end directly: the torch.cuda.graph context manager
            # synchronises the device and empties the allocator caches, which
            # would stall the serving loop
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(stream):
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    launches()
                finally:
                    g.capture_end()
                g.replay()
            graphs.append(g)
        self._count(1 + potrf_launches(n) + 2 * -(-n // 128))
        return L, work, info, alpha

    def _build_version(self, m, charges, coords, offsets, y, stream, old=None, old_nmol=0,
                       graphs=None):
        """Train on the given molecules; with ``old`` (ARAD) only the kernel rows
        of the appended molecules are computed and the old K is reused."""
        n = len(offsets) - 1
        P = _lib.ptr
        st = _lib.stream_handle(stream)
        keep = []
        if m.kind == "cm":
            dev_in, pins = self._upload(charges, coords, offsets, stream)
            D = self._describe(m, dev_in, n, charges, offsets, stream)
            with torch.cuda.stream(stream):
                K = torch.empty((n, n), dtype=torch.float64, device=self.dev)
                _lib.call("fmlb_gaussian_kernel_f64", P(D["X"]), n, m.d, P(D["X"]), n, m.d, m.d,
                          m.sig_ptr, 1, P(K), n, n * n, 1, st)
            self._count(1)
            L, work, info, alpha = self._factor(m, K, y, stream, keep_K=False, graphs=graphs)
            keep += [dev_in, pins]
            return _Version(n=n, X=D["X"], L=L, work=work, info=info, alpha=alpha), keep
        if old is None:
            dev_in, pins = self._upload(charges, coords, offsets, stream)
            D = self._describe(m, dev_in, n, charges, offsets, stream)
            with torch.cuda.stream(stream):
                K = torch.empty((n, n), dtype=torch.float64, device=self.dev)
                keep.append(self._arad_call(m, D, None, K, stream, True))
            keep += [dev_in, pins]
        else:
            n0 = old_nmol
            add = slice(offsets[n0], offsets[n])
            aoff = offsets[n0:] - offsets[n0]
            dev_in, pins = self._upload(charges[add], coords[add], aoff, stream)
            Dn = self._describe(m, dev_in, n - n0, charges[add], aoff, stream)
            madd = n - n0
            with torch.cuda.stream(stream):
                C = torch.empty((madd, n0), dtype=torch.float64, device=self.dev)
                Dm = torch.empty((madd, madd), dtype=torch.float64, device=self.dev)
                keep.append(self._arad_call(m, Dn, {"X": old.X, "Z": old.Z, "N": old.N}, C,
                                            stream, False))
                keep.append(self._arad_call(m, Dn, None, Dm, stream, True))
                K = torch.empty((n, n), dtype=torch.float64, device=self.dev)
                K[:n0, :n0].copy_(old.K)
                K[n0:, :n0].copy_(C)
                K[:n0, n0:].copy_(C.t())
                K[n0:, n0:].copy_(Dm)
                D = {"X": torch.cat([old.X, Dn["X"]]), "Z": torch.cat([old.Z, Dn["Z"]]),
                     "N": torch.cat([old.N, Dn["N"]])}
            keep += [dev_in, pins, C, Dm, Dn]
        L, work, info, alpha = self._factor(m, K, y, stream, keep_K=True, graphs=graphs)
        return _Version(n=n, X=D["X"], Z=D["Z"], N=D["N"], K=K, L=L, work=work, info=info,
                        alpha=alpha), keep

    def add_model(self, mid, kind, charges, coords, offsets, y, sigma, lam, size=29,
                  precision="fp32"):
        """Train a model (blocking) and keep it resident."""
        m = Model(mid, kind, size, sigma, lam, precision)
        offsets = np.asarray(offsets, np.int64)
        if not self._fits(self._train_bytes(m, len(offsets) - 1, 0)):
            raise MemoryError("model %r does not fit the HBM budget" % (mid,))
        v, keep = self._build_version(m, np.asarray(charges), np.asarray(coords), offsets,
                                      np.asarray(y), self.retrain_stream)
        self.retrain_stream.synchronize()
        del keep
        info = int(v.info.item())
        if info:
            raise np.linalg.LinAlgError("model %r: Cholesky failed at column %d" % (mid, info))
        m.version = v
        m.host = (np.asarray(charges, np.float64), np.asarray(coords, np.float64).reshape(-1, 3),
                  offsets, np.asarray(y, np.float64))
        self.models[mid] = m
        return m

    # ------------------------------------------------------------------ prediction
    def _launch_predict(self, slot, m, reqs):
        t_host = time.perf_counter()
        stream = slot["stream"]
        charges = np.concatenate([r.charges for r in reqs])
        coords = np.concatenate([np.asarray(r.coords).reshape(-1, 3) for r in reqs])
        counts = np.concatenate([np.diff(r.offsets) for r in reqs])
        offsets = np.zeros(len(counts) + 1, np.int64)
        np.cumsum(counts, out=offsets[1:])
        nq, atoms = len(counts), len(charges)
        if counts.max() > m.size:
            raise ValueError("a molecule has %d atoms, more than the model size %d"
                             % (int(counts.max()), m.size))
        v = m.version
        pin_specs, dev_specs = self._predict_specs(m, nq, atoms)
        # per-slot arenas, grown when a batch needs more (never inside the steady state)
        need_dev, need_pin = _layout_bytes(dev_specs), _layout_bytes(pin_specs)
        if slot["dev"] is None or slot["dev"].numel() < need_dev:
            slot["dev"] = None
            slot["dev"] = torch.empty(need_dev, dtype=torch.uint8, device=self.dev)
        if slot["pin"] is None or slot["pin"].numel() < need_pin:
            slot["pin"] = torch.empty(need_pin, dtype=torch.uint8, pin_memory=True)
        hp = _carve(slot["pin"], pin_specs)
        dv = _carve(slot["dev"], dev_specs)
        hp[0].numpy()[:] = charges
        hp[1].numpy()[:] = coords
        hp[2].numpy()[:] = offsets
        P = _lib.ptr
        st = _lib.stream_handle(stream)
        a = m.size
        with torch.cuda.stream(stream):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for k in range(3):
                dv[k].copy_(hp[k], non_blocking=True)
            zd, rd, od, pred = dv[:4]
            if m.kind == "cm":
                X, pw = dv[4:6]
                _lib.call("fmlb_coulomb_matrices", P(zd), P(rd), P(od), nq, a, P(X), m.d, None,
                          0, None, None, st)
                _lib.call("fmlb_kernel_predict_f64", 0, P(X), nq, m.d, P(v.X), v.n, m.d, m.d,
                          m.sig_ptr, 1, P(v.alpha), v.n, P(pred), nq, P(pw), pw.numel(), st)
                self._count(3)
            else:
                X, Z, N, Kt, ws = dv[4:9]
                ptp, cnt = _ptp_packed(charges, offsets, a)
                hp[4].numpy()[:] = ptp
                hp[5].numpy()[:] = cnt
                Z.copy_(hp[4], non_blocking=True)
                N.copy_(hp[5], non_blocking=True)
                _lib.call("fmlb_arad_descriptors", P(zd), P(rd), P(od), nq, a, ARAD_CUT, P(X),
                          None, st)
                _lib.call("fmlb_arad_kernels", P(X), P(Z), P(N), nq, P(v.X), P(v.Z), P(v.N), v.n,
                          a, m.sig_ptr, 1, *ARAD_PARAMS, 0, PRECISIONS[m.precision], P(Kt), P(ws),
                          ws.numel(), st)
                _lib.call("fmlb_gemv_f64", P(Kt), v.n, nq, v.n, P(v.alpha), P(pred), st)
                self._count(2 + arad_launches(False, m.precision, a, 1))
            hp[3].copy_(pred, non_blocking=True)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
        slot["busy"] = {"reqs": reqs, "event": ev, "start": ev0, "out": hp[3], "version": v,
                        "kind": m.kind, "host_s": time.perf_counter() - t_host,
                        "t_admit": reqs[0].admitted}
        self.stats["batches"] += 1
        self.stats["batched_requests"] += len(reqs)

    def _finish_predict(self, slot, now):
        b = slot["busy"]
        # per-batch record: host time to launch, device time from first copy to last
        self.batch_log.append((b["kind"], b["host_s"], b["start"].elapsed_time(b["event"]) * 1e-3,
                               len(b["reqs"]), b["t_admit"], now))
        out = b["out"].numpy()
        k = 0
        for r in b["reqs"]:
            r.result = out[k:k + r.nmol].copy()
            r.done = now
            k += r.nmol
        slot["busy"] = None

    # ------------------------------------------------------------------ retraining
    def _launch_retrain(self, m, now):
        t_host = time.perf_counter()
        reqs = m.retrain_pending
        m.retrain_pending = []
        z0, r0, o0, y0 = m.host
        n0 = len(o0) - 1
        zs, rs, ys, cnts = [z0], [r0], [y0], [np.diff(o0)]
        for r in reqs:
            zs.append(np.asarray(r.charges, np.float64))
            rs.append(np.asarray(r.coords, np.float64).reshape(-1, 3))
            ys.append(np.asarray(r.y, np.float64))
            cnts.append(np.diff(r.offsets))
            r.admitted = now
        counts = np.concatenate(cnts)
        offsets = np.zeros(len(counts) + 1, np.int64)
        np.cumsum(counts, out=offsets[1:])
        host = (np.concatenate(zs), np.concatenate(rs), offsets, np.concatenate(ys))
        nbytes = self._train_bytes(m, len(counts), len(counts) - n0)
        old = m.version if m.kind == "arad" else None
        dev = self.dev

        def job():
            torch.cuda.set_device(dev)
            graphs = []
            v, keep = self._build_version(m, *host, self.retrain_stream, old=old, old_nmol=n0,
                                          graphs=graphs)
            keep.append(graphs)
            with torch.cuda.stream(self.retrain_stream):
                info_host = torch.empty(1, dtype=torch.int32, pin_memory=True)
                info_host.copy_(v.info, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.retrain_stream)
            return v, keep, info_host, ev

        self.inflight_bytes += nbytes
        m.retrain_active = {"reqs": reqs, "future": self._retrain_pool.submit(job),
                            "host": host, "bytes": nbytes}
        self.stats["retrains"] += 1
        self.retrain_host_s.append(time.perf_counter() - t_host)

    def _retrain_done(self, m):
        """True once the retrain's launches were issued and its work finished."""
        a = m.retrain_active
        if "event" not in a:
            if not a["future"].done():
                return False
            a["version"], a["keep"], a["info"], a["event"] = a["future"].result()
        return a["event"].query()

    def _finish_retrain(self, m, now):
        a = m.retrain_active
        info = int(a["info"][0])
        self.inflight_bytes -= a["bytes"]
        m.retrain_active = None
        for r in a["reqs"]:
            r.done = now
            r.result = np.array([float(info)])
        if info == 0:
            m.version = a["version"]
            m.host = a["host"]
        else:
            self.stats["retrain_failures"] += 1

    # ------------------------------------------------------------------ loop
    def serve(self, requests, realtime=True, poll_sleep=50e-6):
        """Run the loop until every request is done. ``requests`` carry arrival
        times (seconds from the start); with ``realtime=False`` all arrive at
        once. Returns the wall time in seconds."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for i, r in enumerate(reqs):
            if r.rid < 0:
                r.rid = i
            if r.model not in self.models:
                raise KeyError("unknown model %r" % (r.model,))
        queues = collections.defaultdict(collections.deque)
        nxt, remaining = 0, len(reqs)
        t0 = time.perf_counter()
        t_prev = time.perf_counter()
        while remaining:
            t_now = time.perf_counter()
            self.phase_max["iteration"] = max(self.phase_max["iteration"], t_now - t_prev)
            t_prev = t_now
            now = t_now - t0
            progressed = False
            while nxt < len(reqs) and (not realtime or reqs[nxt].arrival <= now):
                r = reqs[nxt]
                nxt += 1
                if r.retrain:
                    self.models[r.model].retrain_pending.append(r)
                else:
                    queues[r.model].append(r)
                progressed = True
            t_ph = time.perf_counter()
            # completions
            for slot in self.slots:
                if slot["busy"] is not None and slot["busy"]["event"].query():
                    remaining -= len(slot["busy"]["reqs"])
                    self._finish_predict(slot, time.perf_counter() - t0)
                    progressed = True
            for m in self.models.values():
                if m.retrain_active is not None and self._retrain_done(m):
                    remaining -= len(m.retrain_active["reqs"])
                    self._finish_retrain(m, time.perf_counter() - t0)
                    progressed = True
            t_adm = time.perf_counter()
            self.phase_max["completions"] = max(self.phase_max["completions"], t_adm - t_ph)
            # admission of prediction batches: the model with the oldest waiting
            # request first; CM batches take only the high-priority slots, ARAD
            # batches only the others
            for _, mid in sorted((q[0].arrival, mid) for mid, q in queues.items() if q):
                m = self.models[mid]
                q = queues[mid]
                while q and q[0].nmol == 0:  # nothing to compute
                    r = q.popleft()
                    r.admitted, r.done, r.result = now, now, np.zeros(0)
                    remaining -= 1
                    progressed = True
                if not q:
                    continue
                # a CM batch in a low-priority slot would wait behind whole ARAD
                # grids, so CM batches use only the high-priority slots
                free = [s for s in self.slots if s["busy"] is None and
                        (s["high"] == (m.kind == "cm") or not self._have_high)]
                if not free:
                    self.stats["no_free_slot_" + m.kind] += 1
                    continue
                slot = free[0]
                take, mols, atoms = [], 0, 0
                while q and q[0].nmol and (not take or mols + q[0].nmol <= self.max_batch):
                    mols += q[0].nmol
                    atoms += len(q[0].charges)
                    take.append(q.popleft())
                while take and not self._fits(self._slot_growth(slot, m, mols, atoms)):
                    r = take.pop()  # shrink the batch until it fits
                    q.appendleft(r)
                    mols -= r.nmol
                    atoms -= len(r.charges)
                if not take:
                    if self.inflight_bytes == 0 and all(sl["busy"] is None for sl in self.slots):
                        raise MemoryError("a request for model %r needs more device memory than "
                                          "the HBM budget leaves" % (mid,))
                    self.stats["budget_waits"] += 1
                    continue
                for r in take:
                    r.admitted = now
                self._launch_predict(slot, m, take)
                progressed = True
            t_rt = time.perf_counter()
            self.phase_max["admission"] = max(self.phase_max["admission"], t_rt - t_adm)
            # retrains: one at a time per model, when the budget allows
            for m in self.models.values():
                if m.retrain_pending and m.retrain_active is None:
                    n_new = len(m.host[2]) - 1 + sum(r.nmol for r in m.retrain_pending)
                    need = self._train_bytes(m, n_new, n_new - len(m.host[2]) + 1)
                    if self._fits(need):
                        self._launch_retrain(m, now)
                        progressed = True
                    elif self.inflight_bytes == 0 and all(sl["busy"] is None
                                                          for sl in self.slots):
                        raise MemoryError("retraining model %r needs more device memory than "
                                          "the HBM budget leaves" % (m.mid,))
            if not progressed and nxt == len(reqs) and self.inflight_bytes == 0 and \
                    all(s["busy"] is None for s in self.slots) and \
                    all(m.retrain_active is None for m in self.models.values()):
                raise RuntimeError("serve: %d requests can be neither admitted nor completed"
                                   % remaining)
            if not progressed:
                if realtime and nxt < len(reqs):
                    wait = reqs[nxt].arrival - (time.perf_counter() - t0)
                    time.sleep(min(max(wait, 0.0), poll_sleep))
                else:
                    time.sleep(poll_sleep)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    def predict(self, mid, charges, coords, offsets):
        """One request served alone (blocking)."""
        r = Request(mid, np.asarray(charges), np.asarray(coords), np.asarray(offsets, np.int64))
        self.serve([r], realtime=False)
        return r.result


def latency_summary(requests):
    lat = np.array([r.done - r.arrival for r in requests if not r.retrain])
    if not len(lat):
        return {}
    wait = np.array([r.admitted - r.arrival for r in requests if not r.retrain])
    service = np.array([r.done - r.admitted for r in requests if not r.retrain])
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "n": int(len(lat)),
            "queue_wait_p50_ms": float(np.percentile(wait, 50) * 1e3),
            "service_p50_ms": float(np.percentile(service, 50) * 1e3)}
