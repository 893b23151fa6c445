"""Atomic Laplacian KRR of fml.kernels: get_alpha / get_prediction
(fkernels.f90:380-539) and their from-distance forms (:541-702). The
reference ships no test: on CPU the oracle's molecule kernel is pinned
against the vector-kernel oracle (same sum, another loop order) and a numpy
statement, and alpha against a numpy solve; the GPU drop-ins are compared
with the oracle."""

import numpy as np
import pytest

from fml_b200 import synthetic


def _atoms(oracle_mod, nmol, nmax, seed):
    b = synthetic.generate(nmol, nmax=nmax, seed=seed, nmin=1)
    cm = oracle_mod.local_coulomb_matrices(b.charges, b.coords, b.offsets, nmax, "local")
    return cm.T.copy(), np.diff(b.offsets).astype(np.int32)  # Q (d, na), N


def _padded(Q, N, amax):
    x = np.zeros((len(N), amax, Q.shape[0]))
    off = np.concatenate([[0], np.cumsum(N)])
    for m in range(len(N)):
        x[m, :N[m]] = Q[:, off[m]:off[m + 1]].T
    return x


def test_oracle_kernel_matches_vector_kernel_and_alpha_solve(oracle_mod):
    Q, N = _atoms(oracle_mod, 15, 7, 81)
    y = np.random.default_rng(1).standard_normal(len(N))
    sigma, lam = 400.0, 1e-3
    alpha, info, info2 = oracle_mod.get_alpha(Q, N, y, sigma, lam)
    assert info == info2 == 0 and alpha.shape == (N.sum(),)
    x = _padded(Q, N, 7)
    K = oracle_mod.vector_kernels("laplacian", x, x, N, N, [sigma])[0]
    mol = np.linalg.solve(K + lam * np.eye(len(N)), y)
    np.testing.assert_allclose(alpha, np.repeat(mol, N), rtol=1e-8, atol=1e-10 * abs(mol).max())
    # the from-distance route with the L1 atom distances gives the same weights
    D = np.abs(Q.T[:, None, :] - Q.T[None, :, :]).sum(-1)
    a2, _, _ = oracle_mod.get_alpha_from_distance(D, N, y, sigma, lam)
    np.testing.assert_allclose(a2, alpha, rtol=1e-8, atol=1e-10 * abs(mol).max())
    # predictions: the direct and from-distance forms agree with numpy
    Q2, N2 = _atoms(oracle_mod, 6, 7, 82)
    Yp = oracle_mod.get_prediction(Q, Q2, N2, alpha, sigma)
    D2 = np.abs(Q.T[:, None, :] - Q2.T[None, :, :]).sum(-1)  # (na, na2)
    csa = (np.exp(-D2 / sigma) * alpha[:, None]).sum(0)
    off2 = np.concatenate([[0], np.cumsum(N2)])
    ref = np.array([csa[off2[j]:off2[j + 1]].sum() for j in range(len(N2))])
    np.testing.assert_allclose(Yp, ref, rtol=1e-10)
    np.testing.assert_allclose(oracle_mod.get_prediction_from_distance(D2, N2, alpha, sigma),
                               ref, rtol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("nmol,nmax,seed", [(40, 12, 83), (200, 23, 84), (1, 3, 85)])
def test_atomic_krr_vs_oracle(oracle_mod, nmol, nmax, seed):
    import fml_b200
    Q, N = _atoms(oracle_mod, nmol, nmax, seed)
    y = np.random.default_rng(seed).standard_normal(nmol)
    sigma, lam = 400.0, 1e-3
    ref, info, _ = oracle_mod.get_alpha(Q, N, y, sigma, lam)
    assert info == 0
    alpha = fml_b200.get_alpha(Q, N, y, sigma, lam)
    np.testing.assert_allclose(alpha, ref, rtol=1e-8, atol=1e-10 * np.abs(ref).max())
    Q2, N2 = _atoms(oracle_mod, 17, nmax, seed + 100)
    # the per-molecule sums cancel (alpha has both signs): the absolute
    # tolerance scales with the sum of |terms|, bounded by N2.max() * sum|alpha|
    scale = N2.max() * np.abs(alpha).sum()
    Y = fml_b200.get_prediction(Q, Q2, N2, alpha, sigma)
    np.testing.assert_allclose(Y, oracle_mod.get_prediction(Q, Q2, N2, alpha, sigma), rtol=1e-10,
                               atol=1e-14 * scale)
    D = np.abs(Q.T[:, None, :] - Q.T[None, :, :]).sum(-1)
    ad = fml_b200.get_alpha_from_distance(D, N, y, sigma, lam)
    rd, _, _ = oracle_mod.get_alpha_from_distance(D, N, y, sigma, lam)
    np.testing.assert_allclose(ad, rd, rtol=1e-8, atol=1e-10 * np.abs(rd).max())
    D2 = np.abs(Q.T[:, None, :] - Q2.T[None, :, :]).sum(-1)
    Yd = fml_b200.get_prediction_from_distance(D2, N2, alpha, sigma)
    np.testing.assert_allclose(Yd, oracle_mod.get_prediction_from_distance(D2, N2, alpha, sigma),
                               rtol=1e-10, atol=1e-14 * scale)


@pytest.mark.gpu
def test_atomic_krr_errors():
    import fml_b200
    Q = np.random.default_rng(0).standard_normal((5, 6))
    with pytest.raises(ValueError):
        fml_b200.get_alpha(Q, [3, 4], np.ones(2), 1.0, 1e-3)   # sum(N) > atoms
    with pytest.raises(ValueError):
        fml_b200.get_alpha(Q, [3, 3], np.ones(3), 1.0, 1e-3)   # len(Y) != nm
    with pytest.warns(fml_b200.CholeskyWarning):
        a = fml_b200.get_alpha(Q, [3, 3], np.ones(2), 1.0, -1e6)
    assert np.isnan(a).all()
