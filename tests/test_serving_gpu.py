"""KRR serving loop: resident models, continuous batching, retraining.

Checks:
* every request's predictions are the same served alone and in a concurrent
  mix of requests for several models (tolerance 0: the kernels compute each
  query row in the same order whatever the batch);
* CM-Gaussian predictions match the oracle (FP64 kernel, Cholesky, K_test @
  alpha) to 1e-8 relative; ARAD predictions with FP64 kernels match the oracle
  to 1e-8 relative;
* a retrain (+10% molecules, ARAD kernel rows appended to the kept K) gives
  the model trained from scratch on the union (1e-8 relative);
* a budget that cannot hold a request raises MemoryError instead of waiting.
"""

import numpy as np
import pytest
import torch

from fml_b200 import synthetic
from fml_b200.serving import KRRServer, Request, latency_summary

pytestmark = pytest.mark.gpu

SIZE = 16


def _mols(n, seed):
    return synthetic.generate(n, nmax=SIZE, seed=seed)


def _request(model, b, lo, hi, arrival=0.0):
    sub = b.subset(np.arange(lo, hi))
    return Request(model, sub.charges, sub.coords, sub.offsets.astype(np.int64), arrival)


@pytest.fixture(scope="module")
def server():
    srv = KRRServer(hbm_budget=8e9, max_inflight=4, max_batch_molecules=64)
    specs = [(0, "cm", 300, 500.0, 1e-6, "fp64"), (1, "cm", 180, 900.0, 1e-5, "fp64"),
             (2, "arad", 120, 1.0, 1e-4, "fp32"), (3, "arad", 90, 2.0, 1e-3, "fp64")]
    train = {}
    for mid, kind, n, sig, lam, prec in specs:
        b = _mols(n, 500 + mid)
        srv.add_model(mid, kind, b.charges, b.coords, b.offsets, b.energies, sig, lam,
                      size=SIZE, precision=prec)
        train[mid] = (b, sig, lam)
    srv.reserve()
    assert srv.arena_bytes() > 0
    return srv, train


@pytest.fixture(scope="module")
def queries():
    return _mols(400, 77)


def _mix(queries, seed=5, nreq=40):
    rng = np.random.default_rng(seed)
    out, lo = [], 0
    for i in range(nreq):
        cnt = int(rng.integers(1, 20))
        if lo + cnt > queries.nmol:
            lo = 0
        out.append(_request(int(rng.integers(0, 4)), queries, lo, lo + cnt,
                            arrival=float(i) * 1e-4))
        lo += cnt
    return out


def test_same_alone_and_in_the_mix(server, queries):
    srv, _ = server
    mix = _mix(queries)
    srv.serve(mix, realtime=True)
    assert all(r.done is not None for r in mix)
    assert srv.stats["batches"] < len(mix)  # requests were merged into batches
    for r in mix:
        alone = srv.predict(r.model, r.charges, r.coords, r.offsets)
        np.testing.assert_array_equal(alone, r.result)
    lat = latency_summary(mix)
    assert lat["n"] == len(mix) and lat["p99_ms"] >= lat["p50_ms"] > 0


def test_predictions_match_oracle(server, queries, oracle_mod):
    srv, train = server
    sub = queries.subset(np.arange(0, 25))
    for mid in (0, 1, 3):
        b, sig, lam = train[mid]
        got = srv.predict(mid, sub.charges, sub.coords, sub.offsets)
        if srv.models[mid].kind == "cm":
            Xtr = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, SIZE)
            Xq = oracle_mod.coulomb_matrices(sub.charges, sub.coords, sub.offsets, SIZE)
            K = oracle_mod.gaussian_kernel(Xtr.T, Xtr.T, sig)
            Kq = oracle_mod.gaussian_kernel(Xq.T, Xtr.T, sig)
        else:
            Xtr = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, SIZE, 5.0)
            Xq = oracle_mod.arad_descriptors(sub.charges, sub.coords, sub.offsets, SIZE, 5.0)
            Ztr = [b.molecule(i)[0] for i in range(b.nmol)]
            Zq = [sub.molecule(i)[0] for i in range(sub.nmol)]
            K = oracle_mod.get_atomic_symmetric_kernels_arad(Xtr, Ztr, [sig])[0]
            Kq = oracle_mod.get_atomic_kernels_arad(Xq, Xtr, Zq, Ztr, [sig])[0]
        alpha, info = oracle_mod.cho_solve(K + lam * np.eye(len(K)), b.energies)
        assert info == 0
        ref = Kq @ alpha
        np.testing.assert_allclose(got, ref, rtol=1e-8, atol=1e-8 * np.abs(ref).max())


@pytest.mark.parametrize("mid", [1, 3])
def test_retrain_appends_and_matches_from_scratch(server, mid):
    srv, train = server
    m = srv.models[mid]
    n0 = m.version.n
    add = _mols(n0 // 10, 900 + mid)
    q = _mols(12, 901 + mid)
    rt = Request(mid, add.charges, add.coords, add.offsets.astype(np.int64), 0.0, y=add.energies,
                 retrain=True)
    pq = Request(mid, q.charges, q.coords, q.offsets.astype(np.int64), 0.0)
    srv.serve([rt, pq], realtime=False)
    assert rt.result[0] == 0 and m.version.n == n0 + add.nmol
    after = srv.predict(mid, q.charges, q.coords, q.offsets)
    # from scratch on the union
    b, sig, lam = train[mid]
    zs = np.concatenate([b.charges, add.charges])
    rs = np.concatenate([b.coords, add.coords])
    offs = np.concatenate([b.offsets, add.offsets[1:] + b.offsets[-1]])
    ys = np.concatenate([b.energies, add.energies])
    ref_srv = KRRServer(hbm_budget=4e9, max_inflight=2)
    ref_srv.add_model(mid, m.kind, zs, rs, offs, ys, sig, lam, size=SIZE, precision=m.precision)
    ref = ref_srv.predict(mid, q.charges, q.coords, q.offsets)
    np.testing.assert_allclose(after, ref, rtol=1e-8, atol=1e-8 * np.abs(ref).max())
    # the prediction served with the retrain used one of the two versions
    assert pq.result.shape == (q.nmol,)


def test_budget_too_small_raises(queries):
    b = _mols(200, 3)
    srv = KRRServer(hbm_budget=2e9, max_inflight=2)
    srv.add_model(0, "arad", b.charges, b.coords, b.offsets, b.energies, 1.0, 1e-3, size=SIZE)
    srv.budget = srv.resident_bytes() + 1000
    with pytest.raises(MemoryError):
        srv.serve([_request(0, queries, 0, 10)], realtime=False)
    torch.cuda.synchronize()
