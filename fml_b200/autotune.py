"""Project-written autotuner for the batched KRR launch.

Chooses, by timing candidates on the GPU, how many training points a problem
may have to run inside the persistent batched kernel (larger ones take the
multi-CTA path) and the persistent grid size. Results are cached as JSON keyed
by (tuned quantity, problem-size class, GPU name) in
``$FMLB_AUTOTUNE_CACHE`` (default ``~/.cache/fml_b200/autotune.json``).
"""

import json
import os
import threading

import numpy as np
import torch

_LOCK = threading.Lock()
DEFAULT = {"split_threshold": 1536, "grid": 0}
CANDIDATE_THRESHOLDS = (1024, 1536, 2048, 3072, 1 << 30)
CANDIDATE_GRID_MULT = (1, 2)


def cache_path():
    return os.environ.get("FMLB_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "fml_b200",
                                       "autotune.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(data):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def shape_class(problems):
    """Coarse key: problem count and the training-size distribution (log2 bins)."""
    from .batched import n_train_of
    ns = np.array([n_train_of(p) for p in problems])
    if len(ns) == 0:
        return "empty"
    hist = np.bincount(np.clip(np.log2(np.maximum(ns, 1)).astype(int), 0, 20), minlength=21)
    return "np%d_max%d_h%s" % (len(ns), int(2 ** np.ceil(np.log2(ns.max()))),
                               "-".join(str(int(h)) for h in hist[5:14]))


def gpu_key():
    if not torch.cuda.is_available():
        return "nogpu"
    return torch.cuda.get_device_name(torch.cuda.current_device()).replace(" ", "_")


def batched_config(problems, tune=None, batch=None):
    """Cached or default configuration; tunes when FMLB_AUTOTUNE=1 or tune=True
    (on ``batch``, an existing BatchedKRR of these problems, when given)."""
    key = "batched_krr|%s|%s" % (shape_class(problems), gpu_key())
    with _LOCK:
        cached = _load().get(key)
    if cached:
        return cached
    if tune is None:
        tune = os.environ.get("FMLB_AUTOTUNE", "0") == "1"
    if not tune:
        return dict(DEFAULT)
    return tune_batched(problems, key, batch=batch)


def tune_batched(problems, key=None, reps=2, batch=None):
    """Time every candidate (threshold x grid) and keep the fastest.

    The kernel builds that do not depend on the candidate (the ARAD kernels)
    run once; every candidate then times the solve pass with them restored.
    """
    from . import _lib
    from .batched import BatchedKRR
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    b = batch if batch is not None else BatchedKRR(problems, split_threshold=DEFAULT[
        "split_threshold"], grid=DEFAULT["grid"])
    b.keep_kernels()
    results = []
    for thr in CANDIDATE_THRESHOLDS:
        for gm in CANDIDATE_GRID_MULT:
            b.configure(thr, gm * sms)
            b.run(builds=False)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                b.run(builds=False)
            e1.record()
            torch.cuda.synchronize()
            results.append((e0.elapsed_time(e1) / reps, thr, gm * sms))
    b._pristine = None
    ms, thr, grid = min(results)
    cfg = {"split_threshold": thr, "grid": grid, "ms": ms,
           "candidates": [[r[1], r[2], r[0]] for r in results]}
    if key is None:
        key = "batched_krr|%s|%s" % (shape_class(problems), gpu_key())
    with _LOCK:
        data = _load()
        data[key] = cfg
        _store(data)
    _lib.load()
    return cfg
