"""Pins the CPU oracle against the reference's own outputs (tests/golden/).

The fixtures were produced by tests/golden/make_golden.py from the
reference's Python-3-runnable code: ARAD.describe (fml/arad.py), the
pure-Python sorted Coulomb matrix (fml/representations/representations.py:63-113)
and the ARAD distance/kernel restatement of tests/test_arad.py:172-310,
evaluated as tests/test_arad.py:319-400 does.
"""

import json
import os

import numpy as np
import pytest

from fml_b200.data import NUCLEAR_CHARGE, PTP

HERE = os.path.dirname(os.path.abspath(__file__))


def _mols(g, prefix):
    off = g[prefix + "offsets"]
    return [(g[prefix + "charges"][off[i]:off[i + 1]], g[prefix + "coords"][off[i]:off[i + 1]])
            for i in range(len(off) - 1)]


def test_tables_match_reference():
    t = json.load(open(os.path.join(HERE, "golden", "reference_tables.json")))
    assert {int(k): v for k, v in t["PTP"].items()} == PTP
    assert t["NUCLEAR_CHARGE"] == NUCLEAR_CHARGE


@pytest.mark.parametrize("size", [23, 30])
def test_cm_oracle_matches_reference_python(golden, oracle_mod, size):
    g = golden
    cm = oracle_mod.coulomb_matrices(g["xyz_charges"], g["xyz_coords"], g["xyz_offsets"], size)
    ref = g["cm_xyz_s%d" % size]
    np.testing.assert_allclose(cm, ref, rtol=1e-14, atol=1e-13)


def test_cm_oracle_matches_reference_python_synthetic(golden, oracle_mod):
    g = golden
    cm = oracle_mod.coulomb_matrices(g["syn12_charges"], g["syn12_coords"], g["syn12_offsets"], 23)
    np.testing.assert_allclose(cm, g["cm_syn_s23"], rtol=1e-14, atol=1e-13)


@pytest.mark.parametrize("key,size,cut", [("xyz_s30_c5", 30, 5.0), ("xyz_s20_c5", 20, 5.0),
                                          ("xyz_s23_c1e+06", 23, 1e6), ("xyz_s23_c5", 23, 5.0)])
def test_arad_describe_oracle_matches_reference(golden, oracle_mod, key, size, cut):
    g = golden
    d = oracle_mod.arad_descriptors(g["xyz_charges"], g["xyz_coords"], g["xyz_offsets"], size, cut)
    np.testing.assert_allclose(d, g["arad_" + key], rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("cut", [5.0, 1e6])
def test_arad_describe_oracle_matches_reference_synthetic(golden, oracle_mod, cut):
    g = golden
    d = oracle_mod.arad_descriptors(g["syn11_charges"], g["syn11_coords"], g["syn11_offsets"],
                                    23, cut)
    np.testing.assert_allclose(d, g["arad_syn_s23_c%g" % cut], rtol=1e-13, atol=1e-14)


def test_arad_kernel_oracle_matches_reference_test_restatement(golden, oracle_mod):
    """tests/test_arad.py:358-399: 5 vs 5 fixture molecules, sigmas {0.1, 1, 10, 100}."""
    g = golden
    x = g["arad_xyz_s30_c5"]
    Z = [z for z, _ in _mols(g, "xyz_")]
    K = oracle_mod.get_atomic_kernels_arad(x[:5], x[5:], Z[:5], Z[5:], g["testarad_sigmas"])
    np.testing.assert_allclose(K, g["testarad_K_5v5"], rtol=1e-11)


def test_arad_l2_distance_oracle_matches_reference_test_restatement(golden, oracle_mod):
    """get_l2_distance_arad (atomic_arad_l2_distance_all, farad.f90:452-600)
    against the distance matrix Da of tests/test_arad.py:358 (condense with
    molecular=False), which is what the reference test compares it with. Da
    holds NaN past each molecule's atoms; the Fortran routine holds 0."""
    g = golden
    x = g["arad_xyz_s30_c5"]
    Z = [z for z, _ in _mols(g, "xyz_")]
    D = oracle_mod.get_l2_distance_arad(x[:5], x[5:], Z[:5], Z[5:])
    Da = g["testarad_D_5v5"]
    assert D.shape == Da.shape
    ok = ~np.isnan(Da)
    np.testing.assert_allclose(D[ok], Da[ok], rtol=1e-12, atol=1e-13)
    assert (D[~ok] == 0).all()


def test_arad_symmetric_kernel_oracle_matches_reference_test_restatement(golden, oracle_mod):
    # the test restatement has no |l2| < 5e-12 clamp (farad_kernels.f90:735); on the
    # diagonal (identical atoms, l2 ~ 1e-15) that changes exp(-l2/0.1**2) by ~1e-10
    g = golden
    x = g["arad_xyz_s30_c5"]
    Z = [z for z, _ in _mols(g, "xyz_")]
    K = oracle_mod.get_atomic_symmetric_kernels_arad(x, Z, g["testarad_sigmas"])
    np.testing.assert_allclose(K, g["testarad_K_10v10"], rtol=1e-9)


def test_arad_kernel_oracle_synthetic_far_cut(golden, oracle_mod):
    """Descriptor cut 1e6 (neighbours beyond the kernel cut of 6.0 are dropped)."""
    g = golden
    x = g["arad_syn_s23_c1e+06"][:12]
    Z = [z for z, _ in _mols(g, "syn11_")][:12]
    K = oracle_mod.get_atomic_kernels_arad(x[:6], x[6:], Z[:6], Z[6:], g["testarad_syn_sigmas"])
    np.testing.assert_allclose(K, g["testarad_syn_K_6v6"], rtol=1e-11)


def test_oracle_cho_solve_restatement_matches_lapack(oracle_mod):
    rng = np.random.default_rng(3)
    M = rng.standard_normal((120, 120))
    A = M @ M.T + 120 * np.eye(120)
    y = rng.standard_normal(120)
    x1, i1 = oracle_mod.cho_solve(A, y)
    x2, i2 = oracle_mod.cho_solve_restated(A, y)
    assert i1 == i2 == 0
    np.testing.assert_allclose(x1, x2, rtol=1e-12)
    B = A.copy()
    B[37, 37] = -1.0
    assert oracle_mod.cho_solve(B, y)[1] == oracle_mod.cho_solve_restated(B, y)[1] == 38


def test_oracle_symmetric_equals_general(golden, oracle_mod):
    g = golden
    x = g["arad_xyz_s23_c5"]
    Z = [z for z, _ in _mols(g, "xyz_")]
    s = [0.5, 2.0]
    np.testing.assert_allclose(oracle_mod.get_atomic_symmetric_kernels_arad(x, Z, s),
                               oracle_mod.get_atomic_kernels_arad(x, x, Z, Z, s), rtol=1e-13)


def test_gaussian_laplacian_oracle_cross_checked_by_scipy(golden, oracle_mod):
    """fgaussian_kernel / flaplacian_kernel (fkernels.f90:317-377) have no test
    or golden vector in the reference; the oracle's restatement is checked
    against an independent distance code (scipy cdist) on the reference's own
    sorted CMs."""
    from scipy.spatial.distance import cdist
    g = golden
    X = g["cm_syn_s23"]
    A, B = X[:40].T, X[40:].T  # reference layout (d, n)
    for sigma in (50.0, 724.0):
        np.testing.assert_allclose(oracle_mod.gaussian_kernel(A, B, sigma),
                                   np.exp(-cdist(A.T, B.T, "sqeuclidean") / (2 * sigma ** 2)),
                                   rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(oracle_mod.laplacian_kernel(A, B, sigma),
                                   np.exp(-cdist(A.T, B.T, "cityblock") / sigma),
                                   rtol=1e-12, atol=1e-300)


def test_multi_sigma_oracle_bit_identical_to_single_sigma(golden, oracle_mod):
    """kernels_multi (used by the headline-pipeline parity test) forms each
    pair sum once and must give, bit for bit, the single-sigma restatements."""
    X = golden["cm_syn_s23"]
    A, B = X[:33].T, X[33:].T
    sig = [50.0, 724.0, 3000.0]
    for kind, single in (("gaussian", oracle_mod.gaussian_kernel),
                         ("laplacian", oracle_mod.laplacian_kernel)):
        K = oracle_mod.kernels_multi(kind, A, B, sig)
        for q, s in enumerate(sig):
            np.testing.assert_array_equal(K[q], single(A, B, s))


@pytest.mark.parametrize("cut", [5.0, 1e6])
def test_arad_describe_oracle_keeps_reference_tie_order(golden, oracle_mod, cut):
    """Exactly equidistant neighbours of different elements (25 atoms, ties of
    up to 24): arad.py:110 sorts with numpy's default (non-stable above 16
    entries) argsort, and the oracle reproduces its order. Channels 0-2
    (distances, neighbour PTP row/column) are bit-equal; channels 3-4 agree to
    rounding."""
    g = golden
    d = oracle_mod.arad_descriptors(g["ties_charges"], g["ties_coords"], g["ties_offsets"], 30,
                                    cut)
    ref = g["arad_ties_s30_c%g" % cut]
    np.testing.assert_array_equal(d[:, :, :3, :], ref[:, :, :3, :])
    np.testing.assert_allclose(d, ref, rtol=0, atol=1e-14)
