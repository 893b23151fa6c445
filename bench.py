"""Benchmark of the KRR hot path on B200.

Workload (default): large-N Gaussian KRR on sorted Coulomb matrices —
N_train = 32768, N_test = 8192 synthetic molecules with 4..29 atoms
(descriptor length 435), sigma in {100, 400, 1600}, lambda = 1e-8, FP64.
One step = one full pass of the hot path over the batch: sorted Coulomb
matrices from coordinates, the symmetric training kernel for all sigmas,
K + lambda I, Cholesky factorisation and solve per sigma, and the fused
prediction of all test molecules for every sigma.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs are independent replicas (one problem per GPU, no data-path
collective; the KRR problem does not shard), so scaling is weak.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the CPU baseline's OpenMP / OpenBLAS thread counts must be set before those
# libraries initialise
_CORES = len(os.sched_getaffinity(0))
os.environ.setdefault("OMP_NUM_THREADS", str(_CORES))
os.environ.setdefault("OPENBLAS_NUM_THREADS", str(_CORES))
# independent hardware work queues for the serving slots and the batched side
# streams (the default of 8 makes unrelated streams wait behind each other);
# read when the CUDA context is created
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np  # noqa: E402

METRIC = "kernel entries/s & KRR solves/s at stated MAE vs FP64 oracle; p50/p99 latency"
UNIT = "kernel entries/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--ntrain", type=int, default=32768)
    p.add_argument("--ntest", type=int, default=8192)
    p.add_argument("--nmax", type=int, default=29)
    p.add_argument("--sigmas", default="100,400,1600")
    p.add_argument("--lam", type=float, default=1e-8)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--factor", default="ozaki", choices=["ozaki", "fp64"],
                   help="factorisation of the headline step: 'ozaki' (default: trailing "
                        "updates on the int8 tensor cores, then double-double refinement) or "
                        "'fp64' (FP64 tensor cores, no refinement; also reported beside the "
                        "headline)")
    p.add_argument("--slices", type=int, default=6, help="digit planes of the int8 factor")
    p.add_argument("--refine", type=int, default=None,
                   help="double-double refinement steps (default 2 with the int8 factor, 0 "
                        "with the FP64 one)")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the measurements reported beside the headline (FP64-factor "
                        "path, Laplacian and lambda=1e-6 legs, mixed kernels, batched, "
                        "serving)")
    p.add_argument("--cpu-ntrain", type=int, default=4096)
    p.add_argument("--cpu-ntest", type=int, default=1024)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--stages", nargs="?", const="all", default=None,
                   help="time each hot-path kernel on its own (one JSON line per stage); "
                        "'arad' times only the ARAD kernels, 'build' only the descriptors "
                        "and kernel-matrix builds, 'factor' only the factorisations, "
                        "'update' one int8 and one FP64 trailing update (m = --ntrain, "
                        "k = 1024) on seeded normal data")
    p.add_argument("--workload", default="krr",
                   choices=["krr", "batched", "serving", "small", "arad"],
                   help="krr: the large-N KRR step (default, the headline line); batched: "
                        "256 uneven problems in one persistent launch; serving: the request loop")
    p.add_argument("--nprob", type=int, default=256)
    p.add_argument("--serve-rates", default="200,1000,5000")
    p.add_argument("--serve-requests", type=int, default=400,
                   help="requests per arrival rate")
    p.add_argument("--serve-max-train", type=int, default=32768)
    p.add_argument("--serve-baseline-seconds", type=float, default=30.0)
    p.add_argument("--serve-retrain-frac", type=float, default=0.02)
    p.add_argument("--serve-trace", default=None,
                   help="write every request's model, arrival, admission and completion (JSON)")
    p.add_argument("--arad-nmol", type=int, default=4000,
                   help="molecules of the ARAD stage (the first 3/4 form the symmetric set)")
    return p.parse_args()


def entries_per_step(ntrain, ntest, nsig):
    return (ntrain * ntrain + ntest * ntrain) * nsig


def workload_name(a, nsig):
    return ("gaussian KRR on sorted Coulomb matrices: N_train=%d, N_test=%d, nmax=%d (d=%d), "
            "sigma=%s, lambda=%g, FP64" % (a.ntrain, a.ntest, a.nmax, a.nmax * (a.nmax + 1) // 2,
                                          a.sigmas, a.lam))


def headline_config(a, sigmas, world):
    """The workload both arms report as `config`: the reference arm runs a
    bounded sample of it per step and says so in its `cpu_baseline.sample`."""
    return {"workload": workload_name(a, len(sigmas)), "n_train": a.ntrain, "n_test": a.ntest,
            "sigmas": list(sigmas), "lambda": a.lam,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (each K is %.1f GB)" % (a.ntrain ** 2 * 8 / 1e9)}


def refine_steps(a):
    return (2 if a.factor == "ozaki" else 0) if a.refine is None else a.refine


def factor_name(a):
    if a.factor == "ozaki":
        return ("int8 tensor-core (Ozaki, %d digit planes) trailing updates + %d double-double "
                "refinement steps" % (a.slices, refine_steps(a)))
    return "FP64 tensor-core factorisation" + (
        " + %d double-double refinement steps" % refine_steps(a) if refine_steps(a) else "")


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        with open(self.path) as fh:
            lines = fh.readlines()
        os.unlink(self.path)
        return clock_summary(lines)


def clock_summary(lines):
    """Median SM clock under load, the maximum SM clock and the throttle
    reasons seen, from `nvidia-smi --query-gpu=<ClockSampler.FIELDS>
    --format=csv,noheader,nounits` lines. Samples below half the maximum
    clock (idle moments) are left out of the median; fields that are not
    numbers ("[N/A]") are skipped."""
    def num(x):
        try:
            return float(x)
        except ValueError:
            return None

    rows = [p for p in ([x.strip() for x in line.split(",")] for line in lines) if len(p) >= 9]
    sm = [v for v in (num(r[1]) for r in rows) if v is not None]
    smaxes = [v for v in (num(r[2]) for r in rows) if v is not None]
    if not rows or not sm or not smaxes:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"],
                "samples": len(rows)}
    smax = max(smaxes)
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows for i in range(4)
                      if r[5 + i].lower().startswith("active")})
    loaded = [v for v in sm if v > 0.5 * smax] or sm
    return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": smax, "reasons": reasons,
            "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port (C/OpenMP restatement + LAPACK via scipy)
# ---------------------------------------------------------------------------
def cpu_krr_sample(a, sigmas, seed):
    import oracle
    from fml_b200 import synthetic
    oracle.build()
    b = synthetic.generate(a.cpu_ntrain + a.cpu_ntest, nmax=a.nmax, seed=seed)

    def one():
        X = oracle.coulomb_matrices(b.charges, b.coords, b.offsets, a.nmax)
        tr, te = X[:a.cpu_ntrain], X[a.cpu_ntrain:]
        preds = []
        for s in sigmas:  # the reference builds one sigma per call
            K = oracle.gaussian_kernel(tr.T, tr.T, s)
            K[np.diag_indices_from(K)] += a.lam
            alpha, _ = oracle.cho_solve(K, b.energies[:a.cpu_ntrain])
            preds.append(oracle.gaussian_kernel(te.T, tr.T, s) @ alpha)
        return np.array(preds)

    return one, b


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sigmas = [float(s) for s in a.sigmas.split(",")]
    one, _ = cpu_krr_sample(a, sigmas, a.seed)
    for _ in range(a.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        one()
    dt = (time.perf_counter() - t0) / a.steps
    v = entries_per_step(a.cpu_ntrain, a.cpu_ntest, len(sigmas)) / dt
    sample = ("N_train=%d, N_test=%d per step (bounded sample of the workload; same descriptors, "
              "sigmas and lambda; the cost per entry grows with N, so entries/s at N_train=%d is "
              "lower still)" % (a.cpu_ntrain, a.cpu_ntest, a.ntrain))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(a, sigmas, int(os.environ.get("WORLD_SIZE", "1"))),
        "factorisation": "LAPACK dpotrf/dpotrs (OpenBLAS), as the reference calls them",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": _CORES, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def measure_syrk(pipe, torch, lib_call, ptr, stream, factor="fp64", slices=7):
    """Per-launch timing of the dominant kernel (the trailing update) over the
    launch sequence of one factorisation (the strip of each next outer block
    and the bulk past it, with k = the outer panel width), on the pipeline's K
    buffer. factor "ozaki" times fmlb_syrk_lower_ozaki (digit split + int8
    tensor-core update per launch), "fp64" fmlb_syrk_lower_f64."""
    from fml_b200 import _lib
    from fml_b200.krr import outer_panel
    n = pipe.n_train
    W = outer_panel(n)
    K = pipe.K[0]
    evs = []
    flops = 0.0
    if factor == "ozaki":
        lib = _lib.load()
        ws = torch.empty(lib.fmlb_syrk_ozaki_workspace_bytes(n, W, slices), dtype=torch.uint8,
                         device=K.device)
        info = torch.zeros(1, dtype=torch.int32, device=K.device)

    def timed(Cv, m, Pv, strip):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        if factor == "ozaki":
            lib_call("fmlb_syrk_lower_ozaki", ptr(Cv), n, m, ptr(Pv), n, W, strip, slices,
                     ptr(ws), ws.numel(), ptr(info), stream)
        else:
            lib_call("fmlb_syrk_lower_f64", ptr(Cv), n, m, ptr(Pv), n, W, strip, None, stream)
        e1.record()
        evs.append((e0, e1))

    for K0 in range(0, n - W, W):
        base = K0 + W
        m = n - base
        w = min(W, m)
        timed(K[base:, base:], m, K[base:, K0:K0 + W], W)
        flops += 2.0 * W * (w * m - w * (w - 1) / 2)
        m2 = m - W
        if m2 > 0:
            b2 = base + W
            timed(K[b2:, b2:], m2, K[b2:, K0:K0 + W], 0)
            flops += 2.0 * W * m2 * (m2 + 1) / 2
    torch.cuda.synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    return flops, ms, len(evs)


def measure_int8_peak(torch):
    """Dense int8 tensor-core throughput of a library GEMM (torch._int_mm,
    cuBLASLt) at 8192^3, best of 4; None if unavailable."""
    try:
        n = 8192
        a = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda")
        b = torch.randint(-127, 127, (n, n), dtype=torch.int8, device="cuda")
        torch._int_mm(a, b)
        best = 1e30
        for _ in range(4):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except Exception:  # noqa: BLE001 - a missing library path only loses the figure
        return None


def measure_dgemm_peak(torch):
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    best = 1e30
    for _ in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def max_over_ranks(torch, dist, value, device):
    """The slowest rank's time: every replica's step is timed on its own device,
    the job's time is the maximum (barrier before and after the timed region)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(seed, rank):
    """Each replica solves its own problem (independent molecules per rank)."""
    return seed + 1000 * rank


def run_ours(a):
    import torch
    import torch.distributed as dist

    from fml_b200 import _lib, krr, synthetic

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    sigmas = [float(s) for s in a.sigmas.split(",")]
    nsig = len(sigmas)
    n_mol = a.ntrain + a.ntest
    b = synthetic.generate(n_mol, nmax=a.nmax, seed=replica_seed(a.seed, rank))
    dev = torch.device("cuda", local)
    z = torch.from_numpy(b.charges).to(dev)
    r = torch.from_numpy(b.coords).to(dev)
    o = torch.from_numpy(b.offsets).to(dev)
    y = torch.from_numpy(np.ascontiguousarray(b.energies[:a.ntrain])).to(dev)
    nref = refine_steps(a)
    pipe = krr.KRRPipeline(n_mol, a.ntrain, a.nmax, sigmas, a.lam, factor=a.factor,
                           slices=a.slices, refine=nref)

    for _ in range(a.warmup):
        pipe.run(z, r, o, y)
    torch.cuda.synchronize()
    info = pipe.info.cpu().numpy()
    pred = pipe.pred[:, :a.ntest].cpu().numpy()
    yt = b.energies[a.ntrain:]
    mae = {str(s): float(np.abs(pred[k] - yt).mean()) for k, s in enumerate(sigmas)}

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        pipe.run(z, r, o, y)
    e1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / a.steps
    if world > 1:
        ms = max_over_ranks(torch, dist, ms, dev)
    per_step = entries_per_step(a.ntrain, a.ntest, nsig)
    value = world * per_step / (ms * 1e-3)

    # end to end through the public API with host (pinned) inputs
    e2e = None
    if not a.no_e2e:
        hz = torch.from_numpy(b.charges).pin_memory()
        hr = torch.from_numpy(b.coords).pin_memory()
        ho = torch.from_numpy(b.offsets).pin_memory()
        hy = torch.from_numpy(np.ascontiguousarray(b.energies[:a.ntrain])).pin_memory()
        h2d = sum(t.numel() * t.element_size() for t in (hz, hr, ho, hy))
        out_host = torch.empty((nsig, a.ntest), dtype=torch.float64).pin_memory()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(a.steps):
            dz, dr = hz.to(dev, non_blocking=True), hr.to(dev, non_blocking=True)
            do, dy = ho.to(dev, non_blocking=True), hy.to(dev, non_blocking=True)
            p = pipe.run(dz, dr, do, dy)
            out_host.copy_(p, non_blocking=True)
        s1.record()
        torch.cuda.synchronize()
        ems = s0.elapsed_time(s1) / a.steps
        if world > 1:
            ems = max_over_ranks(torch, dist, ems, dev)
        e2e = {"value": world * per_step / (ems * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(nsig * a.ntest * 8),
               "ms_per_step": ems, "api": "fml_b200.krr.KRRPipeline.run on host-pinned inputs"}

    # relative residuals ||y - (K + lambda I) alpha|| / ||y|| in double-double
    # (K from the strict upper triangle the factorisation leaves in place)
    if nref > 0:
        rr = pipe.relative_residuals()
        residuals = {str(s): [float(v) for v in rr[k]] for k, s in enumerate(sigmas)}
        res_key = "relative_residual_per_refinement_step"
    else:
        rr = pipe.residual_now()
        residuals = {str(s): float(rr[k]) for k, s in enumerate(sigmas)}
        res_key = "relative_residual"

    # dominant kernel: the trailing update of the factorisation
    flops, syrk_ms, nl = measure_syrk(pipe, torch, _lib.call, _lib.ptr, _lib.stream_handle(),
                                      a.factor, a.slices)
    dgemm = measure_dgemm_peak(torch)
    fp64_equiv = flops / (syrk_ms * 1e-3) / 1e12
    traffic = None
    if a.factor == "ozaki":
        nprod = a.slices * (a.slices + 1) // 2
        int8_peak = measure_int8_peak(torch)
        peaks = _measured_peaks()
        peak, peak_src = int8_peak, "torch._int_mm (cuBLASLt int8) 8192^3 measured in this run"
        if peak is None:
            peak = 2.0 * peaks["bf16_tflops"]
            peak_src = "2 x measured dense bf16 (MEASURED_PEAKS.json): no int8 GEMM measured"
        achieved = flops * nprod / (syrk_ms * 1e-3) / 1e12
        tpath = os.path.join(ROOT, "profiles", "ozaki_syrk_traffic.json")
        roofline = {"bound": "tensor", "pipe": "int8 tensor cores (tcgen05.mma kind::i8)",
                    "kernel": "ozaki_syrk_kernel (int8 emulated FP64 trailing update, %d "
                              "digit products per FP64 product; timing includes the digit "
                              "split)" % nprod,
                    "achieved": achieved, "peak": peak, "unit": "TOPS (int8)",
                    "frac": achieved / peak, "peak_source": peak_src,
                    "fp64_equivalent_tflops": fp64_equiv, "dgemm_tflops_measured": dgemm,
                    "fp64_equivalent_vs_dgemm": fp64_equiv / dgemm}
    else:
        tpath = os.path.join(ROOT, "profiles", "syrk_update_f64_traffic.json")
        roofline = {"bound": "tensor", "pipe": "FP64 DMMA (mma.sync m8n8k4 f64)",
                    "kernel": "syrk_dmma_kernel (FP64 trailing update)",
                    "achieved": fp64_equiv, "peak": dgemm, "unit": "TFLOP/s",
                    "frac": fp64_equiv / dgemm,
                    "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json "
                                   "holds no FP64 figure)"}
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("bytes_per_launch")
        except (OSError, ValueError):
            traffic = None
    roofline.update({"traffic": traffic, "launches": nl, "avg_launch_ms": syrk_ms / nl,
                     "share_of_step": syrk_ms * nsig / ms,
                     "algorithmic_fp64_flops_per_launch": flops / nl})

    extras = None
    if rank == 0 and world == 1 and not a.no_extras:
        extras = headline_extras(a, torch, pipe, b, sigmas, dev, z, r, o, y, pred, ms)

    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        one, _ = cpu_krr_sample(a, sigmas, a.seed)
        one()
        t0 = time.perf_counter()
        one()
        dt = time.perf_counter() - t0
        cpu = {"value": entries_per_step(a.cpu_ntrain, a.cpu_ntest, nsig) / dt, "unit": UNIT,
               "cores": _CORES, "kind": "port",
               "sample": "N_train=%d, N_test=%d, same sigmas/lambda, one step of %.1f s; the "
                         "port's cost per entry grows with N (kernels ~N^2 d, factorisation "
                         "~N^3), so entries/s at N_train=%d is lower still"
                         % (a.cpu_ntrain, a.cpu_ntest, dt, a.ntrain)}

    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if a.factor == "fp64" else
            "f64 (int8 tensor-core emulated trailing updates, double-double refinement)",
            "data": "synthetic seeded molecules (fml_b200/synthetic.py)",
            "config": headline_config(a, sigmas, world), "factorisation": factor_name(a),
            "solves_per_s": world * nsig / (ms * 1e-3),
            "mae": mae, "potrf_info": [int(v) for v in info], res_key: residuals,
            "clocks": clocks, "e2e": e2e, "gpu_launches": pipe.launches_per_run() * a.steps,
            "roofline": roofline, "cpu_baseline": cpu, "extras": extras,
        }))
    if world > 1:
        dist.destroy_process_group()


def _guarded(out, name, fn):
    """Runs one extra measurement; a failure is recorded, not raised."""
    t0 = time.perf_counter()
    try:
        res = fn()
    except Exception as e:  # noqa: BLE001 - the headline line must still print
        res = {"error": repr(e)[:400]}
    res["wall_s"] = time.perf_counter() - t0
    out[name] = res


def headline_extras(a, torch, pipe, b, sigmas, dev, z, r, o, y, pred, ms_head):
    """Measurements reported beside the headline, outside its timed region."""
    from fml_b200 import _lib, krr

    out = {}
    yt = b.energies[a.ntrain:]
    n_mol = a.ntrain + a.ntest
    per_step = entries_per_step(a.ntrain, a.ntest, len(sigmas))

    def time_pipe(p, steps=2):
        p.run(z, r, o, y)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            p.run(z, r, o, y)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def leg(kind, lam, factor, refine):
        p = krr.KRRPipeline(n_mol, a.ntrain, a.nmax, sigmas, lam, kind, factor=factor,
                            slices=a.slices, refine=refine)
        ms = time_pipe(p, 1)
        pr = p.pred[:, :a.ntest].cpu().numpy()
        res = p.residual_now()
        d = {"kind": kind, "lambda": lam, "factor": factor, "refine": refine, "ms_per_step": ms,
             "entries_per_s": per_step / (ms * 1e-3),
             "solves_per_s": len(sigmas) / (ms * 1e-3),
             "info": [int(v) for v in p.info.cpu().numpy()],
             "mae": {str(s): float(np.abs(pr[k] - yt).mean()) for k, s in enumerate(sigmas)},
             "relative_residual": {str(s): float(res[k]) for k, s in enumerate(sigmas)}}
        return d, pr, p

    if a.factor != "fp64":
        def fp64_path():
            d, pr, p = leg("gaussian", a.lam, "fp64", 0)
            del p
            ms_fp = d["ms_per_step"]
            d["headline_speedup_vs_fp64_factor_path"] = ms_fp / ms_head
            d["max_rel_pred_diff_headline_vs_fp64"] = {
                str(s): float(np.abs(pred[k] - pr[k]).max() / np.abs(pr[k]).max())
                for k, s in enumerate(sigmas)}
            d["rel_mae_diff_headline_vs_fp64"] = {
                str(s): float(abs(np.abs(pred[k] - yt).mean() - np.abs(pr[k] - yt).mean())
                              / np.abs(pr[k] - yt).mean()) for k, s in enumerate(sigmas)}
            return d
        _guarded(out, "plain_fp64_factor_path", fp64_path)
        torch.cuda.empty_cache()

    nref = refine_steps(a)

    def lap():
        d, _, p = leg("laplacian", a.lam, a.factor, nref)
        del p
        return d
    _guarded(out, "laplacian_leg", lap)
    torch.cuda.empty_cache()

    def lam6():
        d, _, p = leg("gaussian", 1e-6, a.factor, nref)
        del p
        return d
    _guarded(out, "lambda_1e-06_leg", lam6)
    torch.cuda.empty_cache()

    def mixed():
        return mixed_kernel_builds(a, torch, pipe, sigmas, dev)
    _guarded(out, "mixed_precision_kernel_builds", mixed)
    torch.cuda.empty_cache()

    def batched():
        return batched_once(a, torch)
    _guarded(out, "batched_256_problems", batched)
    torch.cuda.empty_cache()

    def serving():
        return serving_once(a, torch)
    _guarded(out, "serving_one_rate", serving)
    torch.cuda.empty_cache()
    return out


def mixed_kernel_builds(a, torch, pipe, sigmas, dev):
    """The tcgen05 BF16x3 Gaussian and the FP32 Laplacian builds of the
    training kernels (all sigmas, symmetric, FP32 out) at N_train, with their
    max-abs error against the FP64 builds on the leading 8192 x 8192 block.
    Neither can feed the lambda = 1e-8 factorisation: its entries carry
    ~1e-4 absolute error, four orders above lambda."""
    from fml_b200 import _lib
    lib = _lib.load()
    P, st = _lib.ptr, _lib.stream_handle()
    n, L, ns = a.ntrain, pipe.d, len(sigmas)
    X = pipe.X[:n]
    sp, keep = _lib.host_doubles(sigmas)
    peaks = _measured_peaks()
    K32 = torch.empty((ns, n, n), dtype=torch.float32, device=dev)
    mu = torch.empty(L, dtype=torch.float64, device=dev)
    ws = torch.empty(lib.fmlb_tc_operand_bytes(n, L), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)

    def tc():
        _lib.call("fmlb_column_mean_f64", P(X), n, L, L, P(mu), st)
        _lib.call("fmlb_gaussian_kernel_tc", P(X), n, L, P(X), n, L, L, P(mu), sp, ns, P(K32), n,
                  n * n, 1, P(ws), ws.numel(), P(status), st)
    ms_tc = _time(torch, tc, reps=3)
    nb = min(n, 8192)
    Kd = torch.empty((ns, nb, nb), dtype=torch.float64, device=dev)
    _lib.call("fmlb_gaussian_kernel_f64", P(X), nb, L, P(X), nb, L, L, sp, ns, P(Kd), nb, nb * nb,
              1, st)
    err_tc = _max_abs_diff(torch, K32[:, :nb, :nb], Kd)
    ms_l = _time(torch, lambda: _lib.call("fmlb_laplacian_kernel_f32", P(X), n, L, P(X), n, L, L,
                                          sp, ns, P(K32), n, n * n, 1, st), reps=2)
    _lib.call("fmlb_laplacian_kernel_f64", P(X), nb, L, P(X), nb, L, L, sp, ns, P(Kd), nb, nb * nb,
              1, st)
    err_l = _max_abs_diff(torch, K32[:, :nb, :nb], Kd)
    del keep
    wbytes = 4.0 * n * n * ns
    return {"n": n, "sigmas": sigmas, "error_sample": "leading %d x %d block" % (nb, nb),
            "gaussian_bf16x3_tcgen05": {
                "ms": ms_tc, "entries_per_s": n * n * ns / (ms_tc * 1e-3),
                "hbm_write_gbs": wbytes / ms_tc / 1e6,
                "hbm_write_frac_of_copy_peak": wbytes / ms_tc / 1e6 / peaks["hbm_gbs"],
                "copy_peak_source": peaks["source"],
                "max_abs_err_vs_fp64": err_tc, "status": int(status.item())},
            "laplacian_fp32": {"ms": ms_l, "entries_per_s": n * n * ns / (ms_l * 1e-3),
                               "max_abs_err_vs_fp64": err_l}}


def batched_once(a, torch):
    """The 256-problem batched workload (default tile configuration, no
    autotuning): one captured pass replayed twice after a warm-up."""
    from fml_b200 import autotune
    from fml_b200.batched import BatchedKRR
    probs, kinds, ytest, nt = batched_problems(a.nprob)
    bk = BatchedKRR(probs, split_threshold=autotune.DEFAULT["split_threshold"],
                    grid=autotune.DEFAULT["grid"])
    g = bk.capture()
    g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(2):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 2
    info = bk.infos()
    preds = bk.predictions()
    mae = [float(np.mean(np.abs(p - yt))) for p, yt in zip(preds, ytest)]
    ns = np.array([len(p.y) for p in probs])
    entries = float(np.sum(ns.astype(np.float64) ** 2 + nt * ns))
    del g
    return {"problems": a.nprob, "ms_per_pass": ms, "solves_per_s": a.nprob / (ms * 1e-3),
            "kernel_entries_per_s": entries / (ms * 1e-3),
            "cholesky_failures": int((info != 0).sum()), "median_mae": float(np.median(mae)),
            "config": "default split threshold / grid (autotuning off here)"}


def serving_once(a, torch):
    """The serving loop at one offered rate: 16 resident models (8 CM, 8 ARAD)
    with n_train log-spaced 2000..8192 (the full configuration goes to 32768:
    bench.py --workload serving), 100 Poisson requests at 200 req/s."""
    from fml_b200 import synthetic
    from fml_b200.serving import KRRServer, latency_summary
    size = 29
    srv = KRRServer(hbm_budget=150e9, max_inflight=8, max_batch_molecules=1024)
    specs = serving_models(8192, size)
    for m, kind, bb, sigma, lam in specs:
        srv.add_model(m, kind, bb.charges, bb.coords, bb.offsets, bb.energies, sigma, lam,
                      size=size)
    srv.reserve()
    train_sizes = [bb.nmol for _, _, bb, _, _ in specs]
    pool = synthetic.generate(20000, nmax=size, seed=4000)
    warm = serving_requests(16, 1e6, pool, 16, 3999, train_sizes, retrain_frac=0.0)
    for k, q in enumerate(warm):
        q.model = k
    srv.serve(warm, realtime=False)
    reqs = serving_requests(100, 200.0, pool, 16, 4000, train_sizes, retrain_frac=0.02)
    wall = srv.serve(reqs, realtime=True)
    preds = [q for q in reqs if not q.retrain]
    res = latency_summary(reqs)
    res.update({"offered_req_per_s": 200.0, "requests": len(reqs),
                "molecules_per_s": sum(q.nmol for q in preds) / wall,
                "cm": latency_summary([q for q in preds if q.model < 8]),
                "arad": latency_summary([q for q in preds if q.model >= 8]),
                "models": "16 (8 CM-Gaussian, 8 ARAD), n_train 2000..8192"})
    del srv
    return res


# ---------------------------------------------------------------------------
# per-stage measurements (one JSON line each; not the headline number)
# ---------------------------------------------------------------------------
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # nominal CUDA-core FP32 (FFMA = 2 flops)
MUFU_PEAK_PER_S = 148 * 16 * 1.965e9                 # nominal ex2 throughput


def _measured_peaks():
    """HBM copy GB/s and dense BF16 TFLOP/s of this pool's B200s: the measured
    file when present, else the earlier measurement on this pool (fallback)."""
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        d.setdefault("source", "measured (MEASURED_PEAKS.json)")
        return d
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0,
                "source": "fallback (MEASURED_PEAKS.json absent): 6.65 TB/s copy, 1.59 "
                          "PFLOP/s BF16 measured earlier on this pool"}


def _max_abs_diff(torch, A, B):
    """max |A - B| over (nsigma, n, n) stacks, one row block at a time (measurement only)."""
    worst = 0.0
    for k in range(A.shape[0]):
        for r0 in range(0, A.shape[1], 2048):
            d = (A[k, r0:r0 + 2048].double() - B[k, r0:r0 + 2048].double()).abs().max()
            worst = max(worst, float(d.item()))
    return worst


def _time(torch, fn, reps=3, warmup=1):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def run_stages(a):
    import torch

    from fml_b200 import _lib, synthetic
    from fml_b200.kernels import _ptp_arrays

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    st = _lib.stream_handle()
    P = _lib.ptr
    peaks = _measured_peaks()
    hbm = peaks["hbm_gbs"]
    dgemm = measure_dgemm_peak(torch)
    out = []

    def emit(d):
        d["stage_of"] = "fml_b200 hot path"
        out.append(d)
        print(json.dumps(d), flush=True)

    if a.stages == "arad":
        return run_arad_stage(a, torch, lib, st, P)
    if a.stages == "factor":
        return run_factor_stages(a, torch, lib, st, P, emit)
    if a.stages == "update":
        return run_update_stage(a, torch, lib, st, P, emit)
    # --- descriptors ---------------------------------------------------------
    b = synthetic.generate(40960, nmax=29, seed=2)
    z = torch.from_numpy(b.charges).to(dev)
    r = torch.from_numpy(b.coords).to(dev)
    o = torch.from_numpy(b.offsets).to(dev)
    L = 435
    X = torch.empty((40960, L), dtype=torch.float64, device=dev)
    ms = _time(torch, lambda: _lib.call("fmlb_coulomb_matrices", P(z), P(r), P(o), 40960, 29,
                                        P(X), L, None, 0, None, None, st), reps=5)
    byt = 40960 * L * 8 + len(b.charges) * 32 + 40961 * 4
    emit({"stage": "coulomb_matrices", "config": "40960 molecules, nmax 29", "ms": ms,
          "molecules_per_s": 40960 / (ms * 1e-3), "bound": "hbm", "achieved_gbs": byt / ms / 1e6,
          "peak_gbs": hbm, "peak_source": peaks["source"], "frac": byt / ms / 1e6 / hbm})

    ba = synthetic.generate(4000, nmax=23, seed=1)
    za = torch.from_numpy(ba.charges).to(dev)
    ra = torch.from_numpy(ba.coords).to(dev)
    oa = torch.from_numpy(ba.offsets).to(dev)
    D = torch.empty((4000, 23, 5, 23), dtype=torch.float64, device=dev)
    ms = _time(torch, lambda: _lib.call("fmlb_arad_descriptors", P(za), P(ra), P(oa), 4000, 23,
                                        1e6, P(D), None, st), reps=5)
    emit({"stage": "arad_descriptors", "config": "4000 molecules, size 23, cut 1e6", "ms": ms,
          "molecules_per_s": 4000 / (ms * 1e-3), "bound": "fp64 issue (O(n^3) per molecule)"})

    # --- Gaussian / Laplacian -----------------------------------------------
    n = a.ntrain
    sig = [float(v) for v in a.sigmas.split(",")]
    ns = len(sig)
    sp, keep = _lib.host_doubles(sig)
    Xt = X[:n]
    K = torch.empty((ns, n, n), dtype=torch.float64, device=dev)
    ms = _time(torch, lambda: _lib.call("fmlb_gaussian_kernel_f64", P(Xt), n, L, P(Xt), n, L, L,
                                        sp, ns, P(K), n, n * n, 1, st), reps=2)
    fl = 3.0 * L * n * (n + 1) / 2
    emit({"stage": "gaussian_f64_symmetric", "config": "N=%d, d=%d, %d sigmas" % (n, L, ns),
          "ms": ms, "entries_per_s": n * n * ns / (ms * 1e-3), "bound": "fp64",
          "achieved_tflops": fl / ms / 1e9, "peak_tflops": dgemm,
          "frac": fl / ms / 1e9 / dgemm, "peak_source": "cuBLAS DGEMM measured in this run"})
    K32 = torch.empty((ns, n, n), dtype=torch.float32, device=dev)
    mu = torch.empty(L, dtype=torch.float64, device=dev)
    ws = torch.empty(lib.fmlb_tc_operand_bytes(n, L), dtype=torch.uint8, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)

    def tc():
        _lib.call("fmlb_column_mean_f64", P(Xt), n, L, L, P(mu), st)
        _lib.call("fmlb_gaussian_kernel_tc", P(Xt), n, L, P(Xt), n, L, L, P(mu), sp, ns, P(K32), n,
                  n * n, 1, P(ws), ws.numel(), P(status), st)
    ms = _time(torch, tc, reps=3)
    wbytes = 4.0 * n * n * ns
    tfl = 3 * 2.0 * 448 * n * (n + 1) / 2
    emit({"stage": "gaussian_tc_bf16x3_symmetric", "config": "N=%d, d=%d (448 padded), %d sigmas"
          % (n, L, ns), "ms": ms, "entries_per_s": n * n * ns / (ms * 1e-3), "bound": "hbm",
          "achieved_gbs": wbytes / ms / 1e6, "peak_gbs": hbm, "peak_source": peaks["source"], "frac": wbytes / ms / 1e6 / hbm,
          "tensor_tflops": tfl / ms / 1e9, "tensor_frac_of_bf16": tfl / ms / 1e9 / peaks["bf16_tflops"],
          "max_abs_err_vs_fp64": _max_abs_diff(torch, K32, K), "status": int(status.item())})
    del K32, ws, K
    nl = min(n, 16384)
    Kl = torch.empty((ns, nl, nl), dtype=torch.float64, device=dev)
    Xl = X[:nl]
    ms = _time(torch, lambda: _lib.call("fmlb_laplacian_kernel_f64", P(Xl), nl, L, P(Xl), nl, L, L,
                                        sp, ns, P(Kl), nl, nl * nl, 1, st), reps=2)
    fl = 3.0 * L * nl * (nl + 1) / 2
    emit({"stage": "laplacian_f64_symmetric", "config": "N=%d, d=%d, %d sigmas" % (nl, L, ns),
          "ms": ms, "entries_per_s": nl * nl * ns / (ms * 1e-3), "bound": "fp64",
          "achieved_tflops": fl / ms / 1e9, "peak_tflops": dgemm, "frac": fl / ms / 1e9 / dgemm})
    Kl32 = torch.empty((ns, n, n), dtype=torch.float32, device=dev)
    ms = _time(torch, lambda: _lib.call("fmlb_laplacian_kernel_f32", P(Xt), n, L, P(Xt), n, L, L,
                                        sp, ns, P(Kl32), n, n * n, 1, st), reps=2)
    terms = float(L) * n * (n + 1) / 2
    # 2 FP32 lane operations (sub, abs-add) per term, issued as FP32x2 pairs
    fp32_tf = 2.0 * terms / ms / 1e9
    emit({"stage": "laplacian_f32_symmetric", "config": "N=%d, d=%d, %d sigmas" % (n, L, ns),
          "ms": ms, "entries_per_s": n * n * ns / (ms * 1e-3),
          "bound": "FP32 pipe (70 % FMA-pipe active in the ncu profile)",
          "achieved_fp32_tops": fp32_tf, "peak_fp32_tops_nominal": FP32_PEAK_TFLOPS / 2,
          "frac": fp32_tf / (FP32_PEAK_TFLOPS / 2),
          "max_abs_err_vs_fp64": _max_abs_diff(torch, Kl32[:, :nl, :nl], Kl),
          "error_sample": "leading %d x %d block" % (nl, nl)})
    del Kl32, Kl
    if a.stages == "build":  # descriptors and kernel builds only (small ncu captures)
        del keep
        return out

    # --- Cholesky, solve, prediction ------------------------------------------
    K1 = torch.empty((n, n), dtype=torch.float64, device=dev)
    one = (ctypes_double_arr := _lib.host_doubles([sig[-1]]))[0]
    work = torch.empty(lib.fmlb_potrf_workspace_bytes(n), dtype=torch.uint8, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)

    def factor():
        _lib.call("fmlb_gaussian_kernel_f64", P(Xt), n, L, P(Xt), n, L, L, one, 1, P(K1), n, n * n,
                  1, st)
        _lib.call("fmlb_add_diagonal_f64", P(K1), n, n, a.lam, st)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.call("fmlb_potrf_f64", P(K1), n, n, P(work), P(info), st)
        e1.record()
        return e0, e1
    factor()
    torch.cuda.synchronize()
    tms = []
    for _ in range(2):
        e0, e1 = factor()
        torch.cuda.synchronize()
        tms.append(e0.elapsed_time(e1))
    ms = float(np.median(tms))
    fl = n ** 3 / 3.0
    emit({"stage": "potrf_f64", "config": "N=%d" % n, "ms": ms, "solves_per_s_factor": 1e3 / ms,
          "bound": "fp64", "achieved_tflops": fl / ms / 1e9, "peak_tflops": dgemm,
          "frac": fl / ms / 1e9 / dgemm, "info": int(info.item())})
    x = torch.from_numpy(np.ascontiguousarray(b.energies[:n])).to(dev)
    ms = _time(torch, lambda: _lib.call("fmlb_potrs_f64", P(K1), n, n, P(work), P(x), st), reps=3)
    byt = n * n * 8.0
    emit({"stage": "potrs_f64", "config": "N=%d, 1 right-hand side" % n, "ms": ms, "bound": "hbm",
          "achieved_gbs": byt / ms / 1e6, "peak_gbs": hbm, "peak_source": peaks["source"], "frac": byt / ms / 1e6 / hbm})
    nq = a.ntest
    alpha = torch.randn((ns, n), dtype=torch.float64, device=dev)
    y = torch.empty((ns, nq), dtype=torch.float64, device=dev)
    pw = torch.empty(lib.fmlb_kernel_predict_workspace_bytes(nq, n, ns), dtype=torch.uint8,
                     device=dev)
    Xq = X[n:n + nq]
    ms = _time(torch, lambda: _lib.call("fmlb_kernel_predict_f64", 0, P(Xq), nq, L, P(Xt), n, L, L,
                                        sp, ns, P(alpha), n, P(y), nq, P(pw), pw.numel(), st), reps=3)
    fl = 3.0 * L * nq * n
    emit({"stage": "predict_f64_fused", "config": "N_test=%d, N_train=%d, %d sigmas" % (nq, n, ns),
          "ms": ms, "bound": "fp64", "achieved_tflops": fl / ms / 1e9, "peak_tflops": dgemm,
          "frac": fl / ms / 1e9 / dgemm})
    del K1, work

    del keep
    out += run_arad_stage(a, torch, lib, st, P)
    return out


def run_update_stage(a, torch, lib, st, P, emit):
    """One trailing update C -= P P^T (lower triangle) of each kind at
    m = --ntrain, k = 1024, on a seeded normal panel and C: the int8 update
    (--slices digit planes, the digit split included) and the FP64 one,
    three launches each (the second is the one a profiler captures)."""
    from fml_b200 import _lib
    dev = torch.device("cuda", 0)
    m, k = a.ntrain, 1024
    g = torch.Generator(device=dev).manual_seed(a.seed)
    Pm = torch.randn((m, k), dtype=torch.float64, device=dev, generator=g)
    C = torch.randn((m, m), dtype=torch.float64, device=dev, generator=g)
    ws = torch.empty(lib.fmlb_syrk_ozaki_workspace_bytes(m, k, a.slices), dtype=torch.uint8,
                     device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    fl = 2.0 * k * m * (m + 1) / 2
    ms = _time(torch, lambda: _lib.call("fmlb_syrk_lower_ozaki", P(C), m, m, P(Pm), k, k, 0,
                                        a.slices, P(ws), ws.numel(), P(info), st), reps=2)
    emit({"stage": "update_ozaki", "config": "m=%d, k=%d, %d digit planes" % (m, k, a.slices),
          "ms": ms, "fp64_equivalent_tflops": fl / ms / 1e9,
          "int8_tops": fl * a.slices * (a.slices + 1) / 2 / ms / 1e9, "info": int(info.item())})
    ms = _time(torch, lambda: _lib.call("fmlb_syrk_lower_f64", P(C), m, m, P(Pm), k, k, 0, None,
                                        st), reps=2)
    emit({"stage": "update_fp64", "config": "m=%d, k=%d" % (m, k), "ms": ms,
          "tflops": fl / ms / 1e9})


def run_factor_stages(a, torch, lib, st, P, emit):
    """The factorisations alone at N = --ntrain on the Gaussian kernel of the
    sorted CMs (sigma = last of --sigmas, lambda = --lam): FP64 and int8
    (Ozaki) factors, and one bulk trailing update of each kind (m = N - 1024,
    k = 1024)."""
    from fml_b200 import _lib, synthetic
    dev = torch.device("cuda", 0)
    n = a.ntrain
    b = synthetic.generate(n, nmax=a.nmax, seed=2)
    L = a.nmax * (a.nmax + 1) // 2
    z = torch.from_numpy(b.charges).to(dev)
    r = torch.from_numpy(b.coords).to(dev)
    o = torch.from_numpy(b.offsets).to(dev)
    X = torch.empty((n, L), dtype=torch.float64, device=dev)
    _lib.call("fmlb_coulomb_matrices", P(z), P(r), P(o), n, a.nmax, P(X), L, None, 0, None, None,
              st)
    sig = [float(v) for v in a.sigmas.split(",")][-1]
    one, keep = _lib.host_doubles([sig])
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    dgemm = measure_dgemm_peak(torch)
    w64 = torch.empty(lib.fmlb_potrf_workspace_bytes(n), dtype=torch.uint8, device=dev)
    woz = torch.empty(lib.fmlb_potrf_ozaki_workspace_bytes(n, a.slices), dtype=torch.uint8,
                      device=dev)

    def build():
        _lib.call("fmlb_gaussian_kernel_f64", P(X), n, L, P(X), n, L, L, one, 1, P(K), n, n * n,
                  1, st)
        _lib.call("fmlb_add_diagonal_f64", P(K), n, n, a.lam, st)

    for name in ("fp64", "ozaki"):
        tms = []
        for _ in range(3):
            build()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            if name == "fp64":
                _lib.call("fmlb_potrf_f64", P(K), n, n, P(w64), P(info), st)
            else:
                _lib.call("fmlb_potrf_ozaki_f64", P(K), n, n, a.slices, P(woz), woz.numel(),
                          P(info), st)
            e1.record()
            torch.cuda.synchronize()
            tms.append(e0.elapsed_time(e1))
        ms = float(np.median(tms[1:]))
        fl = n ** 3 / 3.0
        emit({"stage": "potrf_" + name, "config": "N=%d, sigma=%g, lambda=%g" % (n, sig, a.lam),
              "ms": ms, "fp64_equivalent_tflops": fl / ms / 1e9, "dgemm_tflops": dgemm,
              "info": int(info.item())})
    # the triangular solves with the FP64 factor (forward + backward, one right-hand side)
    build()
    _lib.call("fmlb_potrf_f64", P(K), n, n, P(w64), P(info), st)
    x = torch.ones(n, dtype=torch.float64, device=dev)
    ms = _time(torch, lambda: _lib.call("fmlb_potrs_f64", P(K), n, n, P(w64), P(x), st), reps=3)
    emit({"stage": "potrs_f64", "config": "N=%d, 1 right-hand side" % n, "ms": ms,
          "bound": "hbm (the factor is read twice)", "achieved_gbs": n * n * 8.0 / ms / 1e6})
    # one bulk update of each kind: C = K[1024:, 1024:], P = K[1024:, :1024]
    m, k = n - 1024, 1024
    Cv, Pv = K[1024:, 1024:], K[1024:, :1024]
    ws = torch.empty(lib.fmlb_syrk_ozaki_workspace_bytes(m, k, a.slices), dtype=torch.uint8,
                     device=dev)
    info.zero_()
    fl = 2.0 * k * m * (m + 1) / 2
    ms = _time(torch, lambda: _lib.call("fmlb_syrk_lower_f64", P(Cv), n, m, P(Pv), n, k, 0, None,
                                        st), reps=3)
    emit({"stage": "syrk_fp64", "config": "m=%d, k=%d" % (m, k), "ms": ms,
          "tflops": fl / ms / 1e9, "frac_of_dgemm": fl / ms / 1e9 / dgemm})
    ms = _time(torch, lambda: _lib.call("fmlb_syrk_lower_ozaki", P(Cv), n, m, P(Pv), n, k, 0,
                                        a.slices, P(ws), ws.numel(), P(info), st), reps=3)
    nprod = a.slices * (a.slices + 1) // 2
    int8 = measure_int8_peak(torch)
    emit({"stage": "syrk_ozaki", "config": "m=%d, k=%d, %d digit planes (%d int8 products)"
          % (m, k, a.slices, nprod), "ms": ms, "fp64_equivalent_tflops": fl / ms / 1e9,
          "int8_tops": fl * nprod / ms / 1e9, "int8_peak_tops_measured": int8,
          "frac_of_int8_peak": (fl * nprod / ms / 1e9 / int8) if int8 else None,
          "vs_dgemm": fl / ms / 1e9 / dgemm, "info": int(info.item())})
    del keep
    return []


def run_arad_stage(a, torch, lib, st, P):
    """ARAD kernels: symmetric set of 3/4 of --arad-nmol molecules (3000 of the
    4000-molecule configuration), size 23, descriptor cut 1e6, 5 sigmas."""
    import fml_b200
    from fml_b200 import _lib, synthetic
    from fml_b200.kernels import _ptp_arrays

    out = []
    dev = torch.device("cuda", 0)
    ba = synthetic.generate(a.arad_nmol, nmax=23, seed=1)
    Xa = fml_b200.generate_arad_descriptors(ba.charges, ba.coords, ba.offsets, size=23, cut=1e6)
    Z = [ba.molecule(i)[0] for i in range(ba.nmol)]
    ntr = (3 * a.arad_nmol) // 4
    asig = [0.1, 0.5, 1.0, 2.0, 5.0]
    asp, akeep = _lib.host_doubles(asig)
    # neighbour pairs evaluated: per atom the prefix of neighbours within the kernel cut (6.0)
    Pm = np.array([int(((Xa[m, :len(Z[m]), 0, :len(Z[m])] <= 6.0)).sum()) for m in range(ba.nmol)],
                  dtype=np.float64)
    Ptr = Pm[:ntr]
    evals_sym = (Ptr.sum() ** 2 + (Ptr ** 2).sum()) / 2.0
    zp, nn = _ptp_arrays(Z[:ntr], 23)
    x1 = torch.from_numpy(np.ascontiguousarray(Xa[:ntr])).to(dev)
    z1 = torch.from_numpy(zp).to(dev)
    n1 = torch.from_numpy(nn).to(dev)
    Ka = torch.empty((5, ntr, ntr), dtype=torch.float64, device=dev)
    aws = torch.empty(lib.fmlb_arad_workspace_bytes(ntr, ntr, 23, 1), dtype=torch.uint8, device=dev)
    for prec, name in ((1, "fp32"), (0, "fp64")):
        ms = _time(torch, lambda: _lib.call(
            "fmlb_arad_kernels", P(x1), P(z1), P(n1), ntr, None, None, None, ntr, 23, asp, 5, 0.2,
            6.0, 1.0, 0.5, 1, prec, P(Ka), P(aws), aws.numel(), st), reps=1)
        d = {"stage": "arad_symmetric_" + name, "config": "%d molecules (size 23, cut 1e6), 5 "
             "sigmas" % ntr, "ms": ms, "kernel_entries_per_s": ntr * ntr * 5 / (ms * 1e-3),
             "neighbour_pair_evals": evals_sym, "evals_per_s": evals_sym / (ms * 1e-3),
             "bound": "fp32 / mufu issue" if prec else "fp64 issue",
             "mufu_frac": evals_sym / (ms * 1e-3) / MUFU_PEAK_PER_S, "stage_of": "fml_b200 hot path"}
        out.append(d)
        print(json.dumps(d), flush=True)
    del akeep
    return out


# ---------------------------------------------------------------------------
# batched uneven KRR (256 problems, one persistent launch, CUDA graph)
# ---------------------------------------------------------------------------
def batched_problems(nprob, nt=500, arad_fraction=0.5):
    """Uneven KRR problems: problem p draws from seed 1000+p its descriptor kind
    (ARAD with probability ``arad_fraction``, else the sorted CM, nmax 23), its
    training size (log-uniform 100..4000), sigma and lambda (log-uniform
    1e-10..1e-6). CM problems take sigma log-uniform in [50, 2000]; ARAD
    problems take the same quantile of [0.1, 5] (ARAD kernel entries are sums of
    exp(-l2/sigma^2) with l2 of order one, so sigma >= 50 makes every term ~1
    and K numerically rank one). ARAD descriptors use the Molecule default
    cut 5.0 (fml/fml.py:80-86)."""
    import torch

    import fml_b200
    from fml_b200 import synthetic
    from fml_b200.batched import AradProblem, GaussianProblem

    probs, kinds, ytest = [], [], []
    for p in range(nprob):
        rng = np.random.default_rng(1000 + p)
        is_arad = rng.random() < arad_fraction
        n = int(round(np.exp(rng.uniform(np.log(100), np.log(4000)))))
        u = rng.random()
        lam = float(np.exp(rng.uniform(np.log(1e-10), np.log(1e-6))))
        b = synthetic.generate(n + nt, nmax=23, seed=1000 + p)
        y = b.energies[:n]
        if is_arad:
            sigma = float(0.1 * 50.0 ** u)
            X = fml_b200.generate_arad_descriptors(torch.from_numpy(b.charges).cuda(),
                                                   torch.from_numpy(b.coords).cuda(),
                                                   torch.from_numpy(b.offsets).cuda(), size=23)
            Z = [b.charges[b.offsets[i]:b.offsets[i + 1]] for i in range(n + nt)]
            probs.append(AradProblem(X[:n], Z[:n], y, X[n:], Z[n:], sigma, lam))
        else:
            sigma = float(50.0 * 40.0 ** u)
            X = fml_b200.generate_coulomb_matrices(b.charges, b.coords, b.offsets, size=23)
            probs.append(GaussianProblem(X[:n], y, X[n:], sigma, lam))
        kinds.append("arad" if is_arad else "cm")
        ytest.append(b.energies[n:])
    return probs, kinds, ytest, nt


class PlainLoop:
    """The plain FP64 GPU path looped over the problems: FP64 kernel build,
    K + lambda I, blocked Cholesky, solve, prediction, one problem at a time."""

    def __init__(self, probs):
        import ctypes

        import torch

        from fml_b200 import _lib
        from fml_b200.batched import AradProblem
        from fml_b200.kernels import _ptp_arrays
        self.lib = _lib.load()
        self.probs = probs
        nmax = max(len(p.y) for p in probs)
        ntmax = max(len(p.Z_test) if isinstance(p, AradProblem) else p.X_test.shape[0]
                    for p in probs)
        dev = torch.device("cuda")
        self.K = torch.empty(nmax * nmax, dtype=torch.float64, device=dev)
        self.Kt = torch.empty(max(ntmax * nmax, 1), dtype=torch.float64, device=dev)
        self.work = torch.empty(self.lib.fmlb_potrf_workspace_bytes(nmax), dtype=torch.uint8,
                                device=dev)
        self.pwork = torch.empty(self.lib.fmlb_kernel_predict_workspace_bytes(ntmax, nmax, 1),
                                 dtype=torch.uint8, device=dev)
        self.info = torch.zeros(len(probs), dtype=torch.int32, device=dev)
        self.pred, self.staged = [], []
        wsb = 256
        for p in probs:
            n = len(p.y)
            st = {"y": torch.from_numpy(np.asarray(p.y, np.float64)).to(dev),
                  "alpha": torch.empty(n, dtype=torch.float64, device=dev),
                  "sig": (ctypes.c_double * 1)(p.sigma)}
            if isinstance(p, AradProblem):
                amax = p.X_train.shape[1]
                z1, n1 = _ptp_arrays(p.Z_train, amax)
                z2, n2 = _ptp_arrays(p.Z_test, amax)
                st.update(X1=p.X_train.contiguous(), X2=p.X_test.contiguous(),
                          Z1=torch.from_numpy(z1).to(dev), N1=torch.from_numpy(n1).to(dev),
                          Z2=torch.from_numpy(z2).to(dev), N2=torch.from_numpy(n2).to(dev),
                          nt=len(p.Z_test), amax=amax)
                wsb = max(wsb, self.lib.fmlb_arad_workspace_bytes(n, n, amax, 1),
                          self.lib.fmlb_arad_workspace_bytes(len(p.Z_test), n, amax, 0))
            else:
                st.update(Xtr=torch.from_numpy(np.ascontiguousarray(p.X_train)).to(dev),
                          Xte=torch.from_numpy(np.ascontiguousarray(p.X_test)).to(dev),
                          nt=p.X_test.shape[0], d=p.X_train.shape[1])
            self.pred.append(torch.empty(max(st["nt"], 1), dtype=torch.float64, device=dev))
            self.staged.append(st)
        self.ws = torch.empty(wsb, dtype=torch.uint8, device=dev)

    def launches(self):
        from fml_b200.kernels import arad_launches
        from fml_b200.krr import potrf_launches
        c = 0
        for st, p in zip(self.staged, self.probs):
            n = len(p.y)
            if "X1" in st:
                c += arad_launches(True, "fp64", st["amax"], 1) + \
                    arad_launches(False, "fp64", st["amax"], 1) + 1
            else:
                c += 1 + 2
            c += 1 + potrf_launches(n) + 2 * -(-n // 128)
        return c

    def run(self):
        import ctypes

        import torch

        from fml_b200 import _lib
        P = _lib.ptr
        s = _lib.stream_handle()
        for k, (st, p) in enumerate(zip(self.staged, self.probs)):
            n, nt = len(p.y), st["nt"]
            sp = ctypes.cast(st["sig"], ctypes.POINTER(ctypes.c_double))
            if "X1" in st:
                _lib.call("fmlb_arad_kernels", P(st["X1"]), P(st["Z1"]), P(st["N1"]), n, None,
                          None, None, n, st["amax"], sp, 1, 0.2, 6.0, 1.0, 0.5, 1, 0, P(self.K),
                          P(self.ws), self.ws.numel(), s)
            else:
                d = st["d"]
                _lib.call("fmlb_gaussian_kernel_f64", P(st["Xtr"]), n, d, P(st["Xtr"]), n, d, d,
                          sp, 1, P(self.K), n, n * n, 1, s)
            _lib.call("fmlb_add_diagonal_f64", P(self.K), n, n, p.lam, s)
            _lib.call("fmlb_potrf_f64", P(self.K), n, n, P(self.work), P(self.info[k:k + 1]), s)
            st["alpha"].copy_(st["y"])
            _lib.call("fmlb_potrs_f64", P(self.K), n, n, P(self.work), P(st["alpha"]), s)
            if "X1" in st:
                _lib.call("fmlb_arad_kernels", P(st["X2"]), P(st["Z2"]), P(st["N2"]), nt,
                          P(st["X1"]), P(st["Z1"]), P(st["N1"]), n, st["amax"], sp, 1, 0.2, 6.0,
                          1.0, 0.5, 0, 0, P(self.Kt), P(self.ws), self.ws.numel(), s)
                _lib.call("fmlb_gemv_f64", P(self.Kt), n, nt, n, P(st["alpha"]),
                          P(self.pred[k]), s)
            else:
                d = st["d"]
                _lib.call("fmlb_kernel_predict_f64", 0, P(st["Xte"]), nt, d, P(st["Xtr"]), n, d,
                          d, sp, 1, P(st["alpha"]), n, P(self.pred[k]), nt, P(self.pwork),
                          self.pwork.numel(), s)
        return torch.cuda.current_stream()


def run_batched(a):
    """256 uneven KRR problems (CM Gaussian and ARAD) in one pass: ARAD kernel
    builds on side streams, then one persistent launch that builds the Gaussian
    kernels and factors / solves / predicts every problem up to the autotuned
    split (larger ones on the multi-CTA path), all captured in one CUDA graph.
    Compared with the plain FP64 path looped over the problems."""
    import torch

    from fml_b200 import autotune
    from fml_b200.batched import BatchedKRR

    torch.cuda.set_device(0)
    probs, kinds, ytest, nt = batched_problems(a.nprob)
    bk = BatchedKRR(probs, split_threshold=autotune.DEFAULT["split_threshold"],
                    grid=autotune.DEFAULT["grid"])
    cfg = autotune.batched_config(probs, tune=True, batch=bk)
    bk.configure(cfg["split_threshold"], cfg["grid"])
    g = bk.capture()
    for _ in range(max(a.warmup - 1, 0)):
        g.replay()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / a.steps
    preds = bk.predictions()
    info_b = bk.infos()
    # the solve pass alone (ARAD kernels restored, not rebuilt)
    bk.keep_kernels()
    gs = bk.capture(builds=False)
    gs.replay()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        gs.replay()
    e1.record()
    torch.cuda.synchronize()
    ms_solve = e0.elapsed_time(e1) / a.steps
    del gs, g
    # the plain FP64 path looped per problem (timed once, after one warm-up pass)
    loop = PlainLoop(probs)
    loop.run()
    torch.cuda.synchronize()
    e0.record()
    loop.run()
    e1.record()
    torch.cuda.synchronize()
    ms_loop = e0.elapsed_time(e1)
    info_l = loop.info.cpu().numpy()
    rel_mae, max_diff = {"cm": [], "arad": []}, {"cm": 0.0, "arad": 0.0}
    ok = (info_b == 0) & (info_l == 0)
    for k, (pr, pl, kind, yt) in enumerate(zip(preds, loop.pred, kinds, ytest)):
        if not ok[k]:
            continue
        pl = pl.cpu().numpy()[:len(pr)]
        max_diff[kind] = max(max_diff[kind], float(np.max(np.abs(pr - pl))))
        mae_b, mae_l = np.mean(np.abs(pr - yt)), np.mean(np.abs(pl - yt))
        rel_mae[kind].append(abs(mae_b - mae_l) / mae_l)
    mae_stats = {k: {"median": float(np.median(v)), "max": float(np.max(v)), "n": len(v)}
                 for k, v in rel_mae.items() if v}
    ns = np.array([len(p.y) for p in probs])
    entries = float(np.sum(ns.astype(np.float64) ** 2 + nt * ns))
    narad = sum(k == "arad" for k in kinds)
    print(json.dumps({
        "metric": METRIC,
        "workload": "batched uneven KRR: %d problems (%d ARAD, %d CM Gaussian), n_train "
                    "log-uniform 100..4000, n_test %d, nmax 23, lambda log-uniform 1e-10..1e-6; "
                    "CM kernels FP64 inside the persistent launch, ARAD kernels FP32; FP64 "
                    "Cholesky / solve / prediction" % (a.nprob, narad, a.nprob - narad, nt),
        "value": a.nprob / (ms * 1e-3), "unit": "KRR solves/s", "ms_per_step": ms,
        "ms_solve_pass_without_arad_builds": ms_solve,
        "looped_plain_fp64_ms": ms_loop, "speedup_vs_looped": ms_loop / ms,
        "kernel_entries_per_s": entries / (ms * 1e-3),
        "autotune": {k: cfg[k] for k in ("split_threshold", "grid") if k in cfg},
        "n_multi_cta": len(bk.big), "cholesky_failures": {"batched": int((info_b != 0).sum()),
                                                          "looped": int((info_l != 0).sum())},
        "max_abs_pred_diff_vs_looped_fp64": max_diff,
        "rel_mae_diff_vs_looped_fp64": mae_stats, "clocks": clocks,
        "gpu_launches_per_step": bk.launches_per_run(),
        "gpu_launches_looped": loop.launches(), "cuda_graph": True}))


def serving_models(max_train, size=29):
    """16 models: 8 CM-Gaussian and 8 ARAD, training sizes log-spaced
    2000..max_train, model m seeded 400+m."""
    from fml_b200 import synthetic
    ns = np.unique(np.round(np.geomspace(2000, max_train, 8)).astype(int))
    ns = np.resize(ns, 8)
    specs = []
    for m in range(16):
        kind = "cm" if m < 8 else "arad"
        n = int(ns[m % 8])
        b = synthetic.generate(n, nmax=size, seed=400 + m)
        if kind == "cm":
            sigma, lam = (100.0, 400.0, 1600.0)[m % 3], 1e-8
        else:
            sigma, lam = (0.5, 1.0, 2.0)[m % 3], 1e-6
        specs.append((m, kind, b, sigma, lam))
    return specs


def serving_requests(nreq, rate, pool, nmodels, seed, train_sizes, retrain_frac=0.02):
    """Poisson arrivals at ``rate``; each request names a model uniformly, holds
    1..512 query molecules (a slice of the pool); ``retrain_frac`` of them append
    10% of the model's training size."""
    from fml_b200.serving import Request
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, nreq))
    out = []
    for i in range(nreq):
        m = int(rng.integers(0, nmodels))
        retrain = rng.random() < retrain_frac
        cnt = max(1, train_sizes[m] // 10) if retrain else int(rng.integers(1, 513))
        lo = int(rng.integers(0, pool.nmol - cnt))
        sub = pool.subset(np.arange(lo, lo + cnt))
        out.append(Request(m, sub.charges, sub.coords, sub.offsets.astype(np.int64),
                           float(t[i]), y=sub.energies if retrain else None, retrain=retrain))
        out[-1].truth = sub.energies
    return out


def run_serving(a):
    """Served KRR: resident models, Poisson request streams, continuous batching,
    HBM-budget admission, retrains; p50/p99 latency and molecules/s, beside the
    sequential plain FP64 prediction path."""
    import ctypes

    import torch

    from fml_b200 import _lib, synthetic
    from fml_b200.kernels import _ptp_arrays
    from fml_b200.serving import ARAD_CUT, ARAD_PARAMS, KRRServer, latency_summary

    torch.cuda.set_device(0)
    size = 29
    t_setup = time.perf_counter()
    srv = KRRServer(hbm_budget=150e9, max_inflight=8, max_batch_molecules=1024)
    specs = serving_models(a.serve_max_train, size)
    for m, kind, b, sigma, lam in specs:
        srv.add_model(m, kind, b.charges, b.coords, b.offsets, b.energies, sigma, lam, size=size)
    srv.reserve()
    setup_s = time.perf_counter() - t_setup
    train_sizes = [b.nmol for _, _, b, _, _ in specs]
    pool = synthetic.generate(20000, nmax=size, seed=4000)
    # warm-up: one request per model
    warm = serving_requests(16, 1e6, pool, 16, 3999, train_sizes, retrain_frac=0.0)
    for k, r in enumerate(warm):
        r.model = k
    srv.serve(warm, realtime=False)
    results = {}
    launches0 = srv.launches
    sampler = ClockSampler(0)
    sampler.start()
    all_reqs = []
    for rate in [float(x) for x in a.serve_rates.split(",")]:
        srv.stats.clear()
        srv.batch_log.clear()
        srv.retrain_host_s.clear()
        srv.phase_max.clear()
        retries0 = torch.cuda.memory_stats().get("num_alloc_retries", 0)
        reqs = serving_requests(a.serve_requests, rate, pool, 16, 4000, train_sizes,
                                retrain_frac=a.serve_retrain_frac)
        wall = srv.serve(reqs, realtime=True)
        preds = [r for r in reqs if not r.retrain]
        mols = sum(r.nmol for r in preds)
        rt = [r.done - r.arrival for r in reqs if r.retrain]
        res = latency_summary(reqs)
        res.update({"offered_req_per_s": rate, "molecules_per_s": mols / wall,
                    "requests_per_s": len(preds) / wall, "wall_s": wall,
                    "arrival_span_s": reqs[-1].arrival,
                    "batches": srv.stats["batches"], "retrains": len(rt),
                    "retrain_latency_ms_max": float(max(rt) * 1e3) if rt else None,
                    "budget_waits": srv.stats["budget_waits"],
                    "batch_device_ms_p50": {k: float(np.median([b[2] for b in srv.batch_log
                                                                  if b[0] == k]) * 1e3)
                                            for k in ("cm", "arad")
                                            if any(b[0] == k for b in srv.batch_log)},
                    "batch_host_launch_ms_max": float(max(b[1] for b in srv.batch_log) * 1e3)
                    if srv.batch_log else None,
                    "retrain_host_launch_ms_max": float(max(srv.retrain_host_s) * 1e3)
                    if srv.retrain_host_s else None,
                    "loop_max_ms": {k: v * 1e3 for k, v in srv.phase_max.items()},
                    "allocator_retries": int(torch.cuda.memory_stats().get("num_alloc_retries", 0)
                                             - retries0),
                    "cm": latency_summary([r for r in preds if r.model < 8]),
                    "arad": latency_summary([r for r in preds if r.model >= 8])})
        res["stats"] = dict(srv.stats)
        results["%g" % rate] = res
        all_reqs += preds
        if a.serve_trace:
            with open("%s.%g.json" % (a.serve_trace, rate), "w") as f:
                json.dump({"requests": [[r.model, r.nmol, r.retrain, r.arrival, r.admitted,
                                          r.done] for r in reqs],
                           "batches": srv.batch_log}, f)
    clocks = sampler.stop()
    launches = srv.launches - launches0
    # sequential plain FP64 prediction, one request at a time, on a bounded sample
    # of the same requests (fresh FP64 copies of each model's alpha / descriptors)
    lib = _lib.load()
    P = _lib.ptr
    st = _lib.stream_handle()
    sample = serving_requests(64, 200.0, pool, 16, 4001, train_sizes, retrain_frac=0.0)
    seq_mols, seq_t, mae_srv, mae_seq = 0, 0.0, [], []
    srv_preds = {}
    srv.serve([r for r in sample], realtime=False)
    for r in sample:
        srv_preds[id(r)] = r.result
    t_start = time.perf_counter()
    done = 0
    for r in sample:
        if time.perf_counter() - t_start > a.serve_baseline_seconds and done >= 4:
            break
        mdl = srv.models[r.model]
        v = mdl.version
        nq = r.nmol
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        z = torch.from_numpy(r.charges).cuda()
        c = torch.from_numpy(np.ascontiguousarray(r.coords)).cuda()
        o = torch.from_numpy(r.offsets.astype(np.int32)).cuda()
        out = torch.empty(nq, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        e0.record()
        if mdl.kind == "cm":
            X = torch.empty((nq, mdl.d), dtype=torch.float64, device="cuda")
            _lib.call("fmlb_coulomb_matrices", P(z), P(c), P(o), nq, size, P(X), mdl.d, None, 0,
                      None, None, st)
            pw = torch.empty(lib.fmlb_kernel_predict_workspace_bytes(nq, v.n, 1),
                             dtype=torch.uint8, device="cuda")
            _lib.call("fmlb_kernel_predict_f64", 0, P(X), nq, mdl.d, P(v.X), v.n, mdl.d, mdl.d,
                      mdl.sig_ptr, 1, P(v.alpha), v.n, P(out), nq, P(pw), pw.numel(), st)
        else:
            X = torch.empty((nq, size, 5, size), dtype=torch.float64, device="cuda")
            _lib.call("fmlb_arad_descriptors", P(z), P(c), P(o), nq, size, ARAD_CUT, P(X), None,
                      st)
            Zs = [r.charges[r.offsets[i]:r.offsets[i + 1]] for i in range(nq)]
            zp, n1 = _ptp_arrays(Zs, size)
            Zd = torch.from_numpy(zp).cuda()
            Nd = torch.from_numpy(n1).cuda()
            Kt = torch.empty((nq, v.n), dtype=torch.float64, device="cuda")
            ws = torch.empty(lib.fmlb_arad_workspace_bytes(nq, v.n, size, 0), dtype=torch.uint8,
                             device="cuda")
            _lib.call("fmlb_arad_kernels", P(X), P(Zd), P(Nd), nq, P(v.X), P(v.Z), P(v.N), v.n,
                      size, mdl.sig_ptr, 1, *ARAD_PARAMS, 0, 0, P(Kt), P(ws), ws.numel(), st)
            _lib.call("fmlb_gemv_f64", P(Kt), v.n, nq, v.n, P(v.alpha), P(out), st)
        e1.record()
        torch.cuda.synchronize()
        seq_t += e0.elapsed_time(e1) * 1e-3
        seq_mols += nq
        done += 1
        ref = out.cpu().numpy()
        mae_seq.append(float(np.mean(np.abs(ref - r.truth))))
        mae_srv.append(float(np.mean(np.abs(srv_preds[id(r)] - r.truth))))
    rel = [abs(x - y) / y for x, y in zip(mae_srv, mae_seq)]
    best = max(results.values(), key=lambda x: x["molecules_per_s"])
    print(json.dumps({
        "metric": METRIC,
        "workload": "KRR serving: 16 resident models (8 CM-Gaussian, 8 ARAD, FP32 ARAD kernels), "
                    "n_train log-spaced 2000..%d, molecules of 4..29 atoms, Poisson arrivals, "
                    "1..512 query molecules per request, 2%% retrains (+10%% data), HBM budget "
                    "150 GB, %d requests per rate" % (a.serve_max_train, a.serve_requests),
        "value": best["molecules_per_s"], "unit": "molecules/s", "per_rate": results,
        "setup_s": setup_s, "resident_gb": srv.resident_bytes() / 1e9,
        "sequential_plain_fp64": {"molecules_per_s": seq_mols / seq_t if seq_t else None,
                                  "requests": done, "device_s": seq_t},
        "speedup_vs_sequential_fp64": best["molecules_per_s"] / (seq_mols / seq_t)
        if seq_t else None,
        "rel_mae_diff_vs_sequential_fp64": {"median": float(np.median(rel)),
                                            "max": float(np.max(rel))} if rel else None,
        "gpu_launches": launches, "clocks": clocks}))


def run_small(a):
    """The reference's CPU-runnable configuration, end to end: 2000 molecules
    (n <= 23, seed 0), sorted CM, 1000 train / 1000 test, sigma 724, lambda
    1e-8, FP64; the oracle port runs the same configuration in full beside it."""
    import torch

    import fml_b200
    import oracle
    from fml_b200 import synthetic

    torch.cuda.set_device(0)
    b = synthetic.generate(2000, nmax=23, seed=0)
    ytr, yte = b.energies[:1000], b.energies[1000:]

    def ours():
        X = fml_b200.generate_coulomb_matrices(b.charges, b.coords, b.offsets, size=23)
        K = fml_b200.gaussian_kernel(X[:1000].T, X[:1000].T, 724.0)
        K[np.diag_indices_from(K)] += 1e-8
        alpha = fml_b200.cho_solve(K, ytr)
        return fml_b200.gaussian_kernel(X[1000:].T, X[:1000].T, 724.0) @ alpha

    def cpu():
        X = oracle.coulomb_matrices(b.charges, b.coords, b.offsets, 23)
        K = oracle.gaussian_kernel(X[:1000].T, X[:1000].T, 724.0)
        K[np.diag_indices_from(K)] += 1e-8
        alpha, _ = oracle.cho_solve(K, ytr)
        return oracle.gaussian_kernel(X[1000:].T, X[:1000].T, 724.0) @ alpha

    for _ in range(max(a.warmup, 1)):
        p_ours = ours()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        p_ours = ours()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / a.steps * 1e3
    oracle.build()
    p_cpu = cpu()
    t0 = time.perf_counter()
    p_cpu = cpu()
    ms_cpu = (time.perf_counter() - t0) * 1e3
    entries = 1000 * 1000 + 1000 * 1000
    print(json.dumps({
        "metric": METRIC, "workload": "plain FP64 Gaussian KRR on sorted CMs: 2000 molecules "
        "(n <= 23, seed 0), 1000 train / 1000 test, sigma 724, lambda 1e-8, through the "
        "drop-in API (numpy in, numpy out)", "value": entries / (ms * 1e-3), "unit": UNIT,
        "ms_per_step": ms, "mae": float(np.abs(p_ours - yte).mean()),
        "cpu_baseline": {"value": entries / (ms_cpu * 1e-3), "unit": UNIT, "cores": _CORES,
                         "kind": "port", "sample": "the full configuration, one run",
                         "ms": ms_cpu, "mae": float(np.abs(p_cpu - yte).mean())},
        "max_rel_pred_diff_vs_cpu_port": float(np.max(np.abs(p_ours - p_cpu) /
                                                      np.maximum(np.abs(p_cpu), 1e-300))),
        "note": "wall-clock per call including host<->device copies of the numpy API"}))


def run_arad(a):
    """ARAD KRR, plain FP64 against FP32 kernels: 4000 molecules (n <= 23, seed 1),
    ARAD descriptors (size 23, cut 1e6), 3000 train / 1000 test, sigmas {0.1, 0.5,
    1, 2, 5}, lambda 1e-9; FP64 Cholesky and prediction in both cases."""
    import torch

    import fml_b200
    from fml_b200 import _lib, synthetic

    torch.cuda.set_device(0)
    b = synthetic.generate(4000, nmax=23, seed=1)
    X = fml_b200.generate_arad_descriptors(torch.from_numpy(b.charges).cuda(),
                                           torch.from_numpy(b.coords).cuda(),
                                           torch.from_numpy(b.offsets).cuda(), size=23, cut=1e6)
    Z = [b.charges[b.offsets[i]:b.offsets[i + 1]] for i in range(4000)]
    sig = [0.1, 0.5, 1.0, 2.0, 5.0]
    ytr = torch.from_numpy(b.energies[:3000]).cuda()
    yte = b.energies[3000:]
    out = {}
    for prec in ("fp64", "fp32"):
        def step():
            Ktr = fml_b200.get_atomic_symmetric_kernels_arad(X[:3000], Z[:3000], sig,
                                                             precision=prec)
            Kte = fml_b200.get_atomic_kernels_arad(X[3000:], X[:3000], Z[3000:], Z[:3000], sig,
                                                   precision=prec)
            preds = torch.empty((len(sig), 1000), dtype=torch.float64, device="cuda")
            for k in range(len(sig)):
                K = Ktr[k].clone()
                _lib.call("fmlb_add_diagonal_f64", _lib.ptr(K), 3000, 3000, 1e-9,
                          _lib.stream_handle())
                alpha = fml_b200.cho_solve(K, ytr)
                _lib.call("fmlb_gemv_f64", _lib.ptr(Kte[k]), 3000, 1000, 3000, _lib.ptr(alpha),
                          _lib.ptr(preds[k]), _lib.stream_handle())
            return Ktr, Kte, preds
        step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Ktr, Kte, P = step()
        torch.cuda.synchronize()
        out[prec] = (time.perf_counter() - t0, Ktr, Kte, P.cpu().numpy())
    t64, K64, T64, P64 = out["fp64"]
    t32, K32, T32, P32 = out["fp32"]
    mae64 = np.abs(P64 - yte).mean(axis=1)
    mae32 = np.abs(P32 - yte).mean(axis=1)
    print(json.dumps({
        "metric": METRIC, "workload": "ARAD KRR: 4000 molecules (n <= 23, seed 1), ARAD size 23 "
        "cut 1e6, 3000 train / 1000 test, sigmas 0.1,0.5,1,2,5, lambda 1e-9; FP64 against FP32 "
        "ARAD kernels, FP64 Cholesky and prediction",
        "value": 3000 * 3000 * 5 / t32, "unit": "kernel entries/s (train kernel, FP32 step)",
        "step_s": {"fp64": t64, "fp32": t32}, "speedup_fp32_vs_fp64": t64 / t32,
        "max_abs_kernel_err_fp32": {"train": float((K32 - K64).abs().max()),
                                    "test": float((T32 - T64).abs().max())},
        "max_rel_kernel_err_fp32_where_K_gt_1e-8_max": float(max(
            ((K32[k] - K64[k]).abs() / K64[k].abs())[K64[k].abs() > 1e-8 * K64[k].abs().max()]
            .max() for k in range(len(sig)))),
        "mae": {"fp64": dict(zip(map(str, sig), map(float, mae64))),
                "fp32": dict(zip(map(str, sig), map(float, mae32)))},
        "note": "wall-clock per step through the drop-in API (device tensors in and out)"}))


def main():
    a = parse()
    if a.workload == "small":
        return run_small(a)
    if a.workload == "arad":
        return run_arad(a)
    if a.workload == "batched":
        return run_batched(a)
    if a.workload == "serving":
        return run_serving(a)
    if a.stages:
        run_stages(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
