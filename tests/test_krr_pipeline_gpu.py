"""The headline KRR path (krr_fit_predict / KRRPipeline) against the oracle.

The pipeline is the one the large-N benchmark times: sorted Coulomb matrices
(nmax 29) -> FP64 kernel for three sigmas in one pass -> K + lambda I ->
three Cholesky factorisations issued on three streams at once -> solves ->
fused prediction. n_train = 16500 is above 16384, where the factorisation's
outer panels are 1024 columns wide, so the bulk/strip lookahead of the
large-N case runs, three factorisations deep, sharing the per-thread table
of lookahead streams.

Oracle: oracle.c Coulomb matrices (frepresentations.f90:23-110) and kernels
(fkernels.f90:317-377), LAPACK dpotrf/dpotrs through scipy
(fcho_solve.f90:35-42), prediction K_test @ alpha in numpy.

Tolerances: the systems have condition numbers up to ~1e11 at lambda = 1e-8,
so individual weights of two FP64 solvers agree less well than the
predictions they produce. Predictions are compared relative to max
|prediction| per sigma: 3e-8 for the unrefined FP64 factorisation (its panel
solves multiply by the explicit inverse of each 128 x 128 diagonal block,
which loses a small factor of accuracy against LAPACK's triangular solves;
1.1e-8 measured at sigma = 100), 1e-8 for the refined int8 factorisation.
LAPACK info equal. Runs on two caller streams at once are bit-identical to a
run alone.
"""

import numpy as np
import pytest
import torch

import fml_b200
from fml_b200 import synthetic
from fml_b200.krr import KRRPipeline

pytestmark = pytest.mark.gpu

N_TRAIN, N_TEST, NMAX = 16500, 500, 29
SIGMAS = (100.0, 400.0, 1600.0)
LAM = 1e-8


@pytest.fixture(scope="module")
def batch():
    return synthetic.generate(N_TRAIN + N_TEST, nmax=NMAX, seed=2)


_ORACLE = {}


def _oracle_predictions(oracle_mod, b, kind):
    if kind in _ORACLE:
        return _ORACLE[kind]
    X = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, NMAX)
    Xtr, Xte = X[:N_TRAIN], X[N_TRAIN:]
    y = b.energies[:N_TRAIN]
    Kt = oracle_mod.kernels_multi(kind, Xte.T, Xtr.T, SIGMAS)
    preds, infos = [], []
    for q, s in enumerate(SIGMAS):
        K = oracle_mod.kernels_multi(kind, Xtr.T, Xtr.T, [s])[0]
        K[np.diag_indices_from(K)] += LAM
        alpha, info = oracle_mod.cho_solve(K, y)
        del K
        preds.append(Kt[q] @ alpha)
        infos.append(info)
    _ORACLE[kind] = (np.array(preds), infos)
    return _ORACLE[kind]


@pytest.mark.parametrize("kind", ["gaussian", "laplacian"])
def test_krr_fit_predict_matches_oracle(oracle_mod, batch, kind):
    b = batch
    pred, info = fml_b200.krr_fit_predict(b.charges, b.coords, b.offsets, b.energies[:N_TRAIN],
                                          N_TRAIN, SIGMAS, LAM, size=NMAX, kind=kind,
                                          return_info=True)
    ref, ref_info = _oracle_predictions(oracle_mod, b, kind)
    assert list(info) == list(ref_info) == [0, 0, 0]
    assert pred.shape == (len(SIGMAS), N_TEST)
    for q in range(len(SIGMAS)):
        scale = np.abs(ref[q]).max()
        err = np.abs(pred[q] - ref[q]).max()
        assert err <= 3e-8 * scale, (kind, SIGMAS[q], err / scale)


@pytest.mark.parametrize("kind", ["gaussian", "laplacian"])
def test_pipeline_runs_on_two_caller_streams_bit_identical(batch, kind):
    b = batch
    dev = torch.device("cuda")
    z = torch.from_numpy(b.charges).to(dev)
    r = torch.from_numpy(b.coords).to(dev)
    o = torch.from_numpy(b.offsets).to(dev)
    y = torch.from_numpy(b.energies[:N_TRAIN]).to(dev)
    p1 = KRRPipeline(b.nmol, N_TRAIN, NMAX, SIGMAS, LAM, kind)
    solo = p1.run(z, r, o, y).clone()
    torch.cuda.synchronize()
    p2 = KRRPipeline(b.nmol, N_TRAIN, NMAX, SIGMAS, LAM, kind)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(s1):
        out1 = p1.run(z, r, o, y, stream=s1)
    with torch.cuda.stream(s2):
        out2 = p2.run(z, r, o, y, stream=s2)
    torch.cuda.synchronize()
    assert (p1.info.cpu() == 0).all() and (p2.info.cpu() == 0).all()
    assert torch.equal(out1, solo)
    assert torch.equal(out2, solo)


@pytest.mark.parametrize("kind", ["gaussian", "laplacian"])
def test_krr_ozaki_factor_refined_matches_oracle(oracle_mod, batch, kind):
    """The int8 tensor-core factorisation followed by two double-double
    refinement steps: predictions to the FP64 oracle's at 1e-8 relative,
    refined relative residual below 1e-10."""
    b = batch
    dev = torch.device("cuda")
    pipe = KRRPipeline(b.nmol, N_TRAIN, NMAX, SIGMAS, LAM, kind, factor="ozaki", slices=7,
                       refine=2)
    pred = pipe.run(torch.from_numpy(b.charges).to(dev), torch.from_numpy(b.coords).to(dev),
                    torch.from_numpy(b.offsets).to(dev),
                    torch.from_numpy(b.energies[:N_TRAIN]).to(dev)).cpu().numpy()
    assert (pipe.info.cpu() == 0).all()
    res = pipe.relative_residuals()
    assert (res[:, -1] < 1e-10).all(), res
    ref, _ = _oracle_predictions(oracle_mod, b, kind)
    for q in range(len(SIGMAS)):
        scale = np.abs(ref[q]).max()
        err = np.abs(pred[q] - ref[q]).max()
        assert err <= 1e-8 * scale, (kind, SIGMAS[q], err / scale)
