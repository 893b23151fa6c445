"""Batched uneven KRR (one persistent launch + multi-CTA path for large
problems) against the oracle solved problem by problem.

Tolerance: predictions to 1e-8 relative (well-conditioned problems, lambda
>= 1e-4)."""

import numpy as np
import pytest
import torch

from fml_b200 import synthetic
from fml_b200.batched import BatchedKRR, GaussianProblem, PrecomputedProblem

pytestmark = pytest.mark.gpu


def _oracle_predict(oracle_mod, Xtr, y, Xte, sigma, lam):
    K = oracle_mod.gaussian_kernel(Xtr.T, Xtr.T, sigma)
    K[np.diag_indices_from(K)] += lam
    alpha, info = oracle_mod.cho_solve(K, y)
    return oracle_mod.gaussian_kernel(Xte.T, Xtr.T, sigma) @ alpha, info


@pytest.fixture(scope="module")
def problems(oracle_mod):
    rng = np.random.default_rng(3)
    sizes = [70, 130, 257, 64, 1, 500, 900, 33, 200, 1300]
    out = []
    for i, n in enumerate(sizes):
        b = synthetic.generate(n + 40, nmax=23, seed=100 + i)
        X = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 23)
        out.append(GaussianProblem(X[:n], b.energies[:n], X[n:], float(rng.uniform(200, 1000)),
                                   float(10 ** rng.uniform(-4, -2))))
    return out


def test_batched_matches_per_problem_oracle(oracle_mod, problems):
    bk = BatchedKRR(problems, split_threshold=600, grid=0)
    assert bk.big and bk.small  # both paths exercised
    bk.run()
    torch.cuda.synchronize()
    assert (bk.infos() == 0).all()
    for p, pred in zip(problems, bk.predictions()):
        ref, info = _oracle_predict(oracle_mod, p.X_train, p.y, p.X_test, p.sigma, p.lam)
        assert info == 0
        np.testing.assert_allclose(pred, ref, rtol=1e-8, atol=1e-8 * np.abs(ref).max())


def test_batched_graph_replay_is_identical(problems):
    bk = BatchedKRR(problems, split_threshold=600, grid=0)
    bk.run()
    torch.cuda.synchronize()
    first = [p.copy() for p in bk.predictions()]
    g = bk.capture()
    bk.pred.zero_()
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(first, bk.predictions()):
        np.testing.assert_array_equal(a, b)


def test_batched_precomputed_kernels_and_failure_isolation(oracle_mod, problems):
    # two ARAD problems (precomputed kernels) and one indefinite problem
    b = synthetic.generate(60, nmax=12, seed=9)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 12, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    Ktr = oracle_mod.get_atomic_symmetric_kernels_arad(X[:45], Z[:45], [2.0])[0]
    Kte = oracle_mod.get_atomic_kernels_arad(X[45:], X[:45], Z[45:], Z[:45], [2.0])[0]
    arad = PrecomputedProblem(Ktr, Kte, b.energies[:45], 1e-3)
    bad = PrecomputedProblem(-np.eye(20), np.ones((3, 20)), np.ones(20), 0.0)
    probs = problems[:4] + [arad, bad]
    bk = BatchedKRR(probs, split_threshold=10000, grid=0)
    bk.run()
    torch.cuda.synchronize()
    info = bk.infos()
    assert info[5] == 1 and (info[:5] == 0).all()
    Ka = Ktr + 1e-3 * np.eye(45)
    alpha, _ = oracle_mod.cho_solve(Ka, b.energies[:45])
    np.testing.assert_allclose(bk.predictions()[4], Kte @ alpha, rtol=1e-8)
    for p, pred in zip(problems[:4], bk.predictions()[:4]):
        ref, _ = _oracle_predict(oracle_mod, p.X_train, p.y, p.X_test, p.sigma, p.lam)
        np.testing.assert_allclose(pred, ref, rtol=1e-8, atol=1e-8 * np.abs(ref).max())


@pytest.fixture(scope="module")
def arad_set(oracle_mod):
    b = synthetic.generate(110, nmax=12, seed=21)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 12, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    return b, X, Z


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-8), ("fp32", 1e-3)])
def test_batched_arad_builds_in_pass(oracle_mod, problems, arad_set, precision, rtol):
    """ARAD kernels built by the pass itself (side streams), one ARAD problem on
    the multi-CTA path (stored test kernel, GEMV prediction), graph replay."""
    from fml_b200.batched import AradProblem
    b, X, Z = arad_set
    splits = [(slice(0, 30), slice(30, 40), 0.7, 1e-3), (slice(40, 100), slice(100, 110), 2.0,
                                                         1e-2)]
    aps, refs = [], []
    for tr, te, sig, lam in splits:
        aps.append(AradProblem(X[tr], Z[tr], b.energies[tr], X[te], Z[te], sig, lam,
                               precision=precision))
        Ktr = oracle_mod.get_atomic_symmetric_kernels_arad(X[tr], Z[tr], [sig])[0]
        Kte = oracle_mod.get_atomic_kernels_arad(X[te], X[tr], Z[te], Z[tr], [sig])[0]
        alpha, info = oracle_mod.cho_solve(Ktr + lam * np.eye(len(Ktr)), b.energies[tr])
        assert info == 0
        refs.append(Kte @ alpha)
    probs = [problems[0], aps[0], problems[2], aps[1]]
    bk = BatchedKRR(probs, split_threshold=50, grid=0)
    assert 3 in bk.big and 1 in bk.small
    g = bk.capture()
    bk.pred.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert (bk.infos() == 0).all()
    preds = bk.predictions()
    for k, ref in zip((1, 3), refs):
        np.testing.assert_allclose(preds[k], ref, rtol=rtol, atol=rtol * np.abs(ref).max())
    for k in (0, 2):
        p = probs[k]
        ref, _ = _oracle_predict(oracle_mod, p.X_train, p.y, p.X_test, p.sigma, p.lam)
        np.testing.assert_allclose(preds[k], ref, rtol=1e-8, atol=1e-8 * np.abs(ref).max())
    assert bk.launches_per_run() > 1


def test_autotuner_times_candidates_and_caches(tmp_path, monkeypatch, problems, arad_set):
    """The tuner times every (split threshold, grid) candidate on the solve pass
    (ARAD kernels restored, not rebuilt), keeps the fastest, caches it, and the
    tuned batch gives the same predictions as an untuned one."""
    from fml_b200 import autotune
    from fml_b200.batched import AradProblem
    monkeypatch.setenv("FMLB_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b, X, Z = arad_set
    probs = problems[:5] + [AradProblem(X[:40], Z[:40], b.energies[:40], X[40:50], Z[40:50],
                                        1.0, 1e-3)]
    bk = BatchedKRR(probs, split_threshold=autotune.DEFAULT["split_threshold"],
                    grid=autotune.DEFAULT["grid"])
    bk.run()
    torch.cuda.synchronize()
    ref = [p.copy() for p in bk.predictions()]
    cfg = autotune.batched_config(probs, tune=True, batch=bk)
    n_cand = len(autotune.CANDIDATE_THRESHOLDS) * len(autotune.CANDIDATE_GRID_MULT)
    assert len(cfg["candidates"]) == n_cand
    assert cfg["ms"] == min(c[2] for c in cfg["candidates"])
    assert autotune.batched_config(probs) == cfg  # served from the cache now
    tuned = BatchedKRR(probs)
    assert (tuned.split_threshold, tuned.grid) == (cfg["split_threshold"], cfg["grid"])
    tuned.run()
    torch.cuda.synchronize()
    for a, c in zip(ref, tuned.predictions()):
        np.testing.assert_allclose(c, a, rtol=1e-9, atol=1e-9 * np.abs(a).max())
