"""Atom-level ARAD kernel (fget_atomic_kernels_arad, farad_kernels.f90:757-899),
oracle side. The reference ships no test for it; the oracle's atom-pair core
(atomic_distl2) is the one pinned through the molecular ARAD kernels, and the
atom-level kernel is pinned against them here: for per-atom descriptors cut
out of molecular ones (neighbour count = the molecule's atom count), the sum
of the atom-level kernel over the atoms of two molecules is the molecular
symmetric kernel (fget_symmetric_kernels_arad, unconditional sine factors as
in the atom-level routine), to 1e-12 relative."""

import numpy as np

from fml_b200 import synthetic
from fml_b200.data import ptp_of


def atoms_of(X, Z):
    """Per-atom descriptors (na, 5, amax), PTP (na, 2), counts (na,), molecule id."""
    q, z, n, mol = [], [], [], []
    for m, zm in enumerate(Z):
        for a in range(len(zm)):
            q.append(X[m, a])
            n.append(len(zm))
            mol.append(m)
        z.append(ptp_of(zm))
    return np.array(q), np.concatenate(z), np.array(n, np.int32), np.array(mol)


def test_atomic_kernel_sums_to_molecular_symmetric_kernel(oracle_mod):
    b = synthetic.generate(9, nmax=10, seed=4)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 10, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    q, z, n, mol = atoms_of(X, Z)
    sig = [0.5, 2.0]
    Ka = oracle_mod.fget_atomic_kernels_arad(q, q, z, z, n, n, sig, len(q), len(q), len(sig),
                                             0.2, 6.0, 1.0, 0.5)
    Km = oracle_mod.get_atomic_symmetric_kernels_arad(X, Z, sig)
    for k in range(len(sig)):
        summed = np.zeros((b.nmol, b.nmol))
        np.add.at(summed, (mol[:, None], mol[None, :]), Ka[k])
        np.testing.assert_allclose(summed, Km[k], rtol=1e-12)
    # self pairs: l2 = 0 exactly, so the diagonal of every sigma is 1
    for k in range(len(sig)):
        np.testing.assert_array_equal(np.diag(Ka[k]), 1.0)


def test_atomic_distances_are_the_kernel_exponents(oracle_mod):
    """fget_atomic_distance_arad's l2 and fget_atomic_kernels_arad's exp(-l2/s^2)
    come from the same l2 (farad_kernels.f90:873-891 and :1005-1019)."""
    b = synthetic.generate(6, nmax=9, seed=5)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 9, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    q, z, n, _ = atoms_of(X, Z)
    D = oracle_mod.atomic_distances_arad(q, q[:20], z, z[:20], n, n[:20], 0.2, 6.0, 1.0, 0.5)
    K = oracle_mod.fget_atomic_kernels_arad(q, q[:20], z, z[:20], n, n[:20], [1.3], len(q), 20,
                                            1, 0.2, 6.0, 1.0, 0.5)
    np.testing.assert_allclose(K[0], np.exp(D * (-1.0 / 1.3 ** 2)), rtol=1e-15, atol=0)


def test_alpha_kernel_is_symmetric_kernel_plus_lambda(oracle_mod):
    """fget_alpha_arad's matrix (farad_kernels.f90:231-389) is the symmetric
    ARAD kernel with the routine's fixed parameters plus lambda I; only its eps
    differs (1e-11 vs 5e-12), which moves no entry by more than 1e-12
    relative. The weights are inv(K + lambda I) y, spread over each
    molecule's atoms."""
    b = synthetic.generate(12, nmax=9, seed=14)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 9, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    n = np.array([len(z) for z in Z], np.int32)
    zp = np.zeros((b.nmol, 9, 2))
    for i, z in enumerate(Z):
        zp[i, :len(z)] = ptp_of(z)
    y = np.random.default_rng(0).standard_normal(b.nmol)
    sigma, lam = 2.0, 1e-2
    alpha, info, info2 = oracle_mod.fget_alpha_arad(X, zp, n, y, sigma, lam)
    assert info == info2 == 0 and alpha.shape == (n.sum(),)
    K = oracle_mod.get_atomic_symmetric_kernels_arad(X, Z, [sigma])[0] + lam * np.eye(b.nmol)
    mol_alpha = np.linalg.solve(K, y)
    np.testing.assert_allclose(alpha, np.repeat(mol_alpha, n), rtol=1e-9,
                               atol=1e-12 * np.abs(mol_alpha).max())
