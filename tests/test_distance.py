"""Generic distance matrices (fml/math/distance.py:58-117 -> fdistance.f90).
The reference ships no test for them: the oracle is pinned against scipy's
independent cdist (cityblock, euclidean, minkowski) on CPU; the GPU drop-ins
are compared with the oracle, including the reference's signed p-th powers
(no abs) for odd and real p."""

import numpy as np
import pytest
from scipy.spatial.distance import cdist


def _sets(seed, d=40, na=33, nb=71):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((d, na)), rng.standard_normal((d, nb))


def test_oracle_matches_scipy(oracle_mod):
    A, B = _sets(1)
    np.testing.assert_allclose(oracle_mod.distance_matrix("manhattan", A, B),
                               cdist(A.T, B.T, "cityblock"), rtol=1e-13)
    np.testing.assert_allclose(oracle_mod.distance_matrix("l2", A, B),
                               cdist(A.T, B.T, "euclidean"), rtol=1e-13)
    np.testing.assert_allclose(oracle_mod.distance_matrix("p_int", np.abs(A), -np.abs(B), 4),
                               cdist(np.abs(A).T, -np.abs(B).T, "minkowski", p=4), rtol=1e-12)
    # real p on non-negative differences equals the Minkowski distance
    np.testing.assert_allclose(oracle_mod.distance_matrix("p_real", np.abs(A) + 5, -np.abs(B), 2.5),
                               cdist((np.abs(A) + 5).T, -np.abs(B).T, "minkowski", p=2.5),
                               rtol=1e-12)
    # the signed form: odd p keeps the sign of each difference
    D3 = oracle_mod.distance_matrix("p_int", A, B, 3)
    ref = np.cbrt(((A[:, :, None] - B[:, None, :]) ** 3).sum(0))
    ok = ref > 0
    np.testing.assert_allclose(D3[ok], ref[ok], rtol=1e-10)
    assert np.isnan(D3[~ok]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("d,na,nb", [(40, 33, 71), (276, 130, 65), (1, 1, 1), (17, 64, 128)])
def test_distances_vs_oracle(oracle_mod, d, na, nb):
    import fml_b200
    A, B = _sets(d + na, d, na, nb)
    D = fml_b200.manhattan_distance(A, B)
    assert D.flags["F_CONTIGUOUS"] and D.shape == (na, nb)
    np.testing.assert_allclose(D, oracle_mod.distance_matrix("manhattan", A, B), rtol=1e-13)
    np.testing.assert_allclose(fml_b200.l2_distance(A, B),
                               oracle_mod.distance_matrix("l2", A, B), rtol=1e-13)
    np.testing.assert_allclose(fml_b200.p_distance(A, B), oracle_mod.distance_matrix("l2", A, B),
                               rtol=1e-13)
    for p in (1, 3, 4):
        np.testing.assert_allclose(fml_b200.p_distance(A, B, p),
                                   oracle_mod.distance_matrix("p_int", A, B, p), rtol=1e-12)
    for p in (1.5, 2.0):
        np.testing.assert_allclose(fml_b200.p_distance(A, B, p),
                                   oracle_mod.distance_matrix("p_real", A, B, p), rtol=1e-12)


def test_distance_argument_errors():
    """The reference's argument checks (distance.py:60-64, :92-117) run on the
    host before any device work."""
    import fml_b200
    A, B = _sets(3)
    with pytest.raises(ValueError):
        fml_b200.manhattan_distance(A, B[:-1])
    with pytest.raises(ValueError):
        fml_b200.l2_distance(A[0], B)
    with pytest.raises(ValueError):
        fml_b200.p_distance(A, B, np.int64(3))  # the reference tests type(p) exactly
