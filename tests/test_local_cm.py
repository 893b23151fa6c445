"""Per-atom Coulomb matrices (fgenerate_local_coulomb_matrix /
fgenerate_atomic_coulomb_matrix, frepresentations.f90:204-390) and the atomic
vector kernels over them (fget_vector_kernels_gaussian / _laplacian,
fkernels.f90:23-162).

CPU tests pin the oracle: the per-atom matrices against the reference's own
Python versions (representations.py:117-217 and :219-251, run by
tests/golden/make_golden.py), the vector kernels against a direct numpy
statement of the Fortran loops (the reference ships no test and no Python
version of them). GPU tests compare libfmlb with the oracle."""

import numpy as np
import pytest

from fml_b200 import synthetic

KINDS = ("local", "atomic")


def _numpy_vector_kernels(kind, x1, x2, n1, n2, sigmas):
    K = np.zeros((len(sigmas), len(n1), len(n2)))
    for i in range(len(n1)):
        for j in range(len(n2)):
            a = x1[i, :n1[i]][:, None, :]
            b = x2[j, :n2[j]][None, :, :]
            if kind == "gaussian":
                d = ((a - b) ** 2).sum(-1)
                c = [-0.5 / s ** 2 for s in sigmas]
            else:
                d = np.abs(a - b).sum(-1)
                c = [-1.0 / s for s in sigmas]
            for k in range(len(sigmas)):
                K[k, i, j] = np.exp(d * c[k]).sum()
    return K


def _per_molecule(cm, offsets, amax):
    off = np.asarray(offsets)
    x = np.zeros((len(off) - 1, amax, cm.shape[1]))
    for m in range(len(off) - 1):
        x[m, :off[m + 1] - off[m]] = cm[off[m]:off[m + 1]]
    return x, np.diff(off).astype(np.int32)


# ---------------------------------------------------------------- oracle pins
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("src,pre", [("xyz", "xyz_"), ("syn", "syn12_")])
def test_local_cm_oracle_matches_reference_python(golden, oracle_mod, kind, src, pre):
    g = golden
    cm = oracle_mod.local_coulomb_matrices(g[pre + "charges"], g[pre + "coords"],
                                           g[pre + "offsets"], 23, kind)
    np.testing.assert_allclose(cm, g["lcm_%s_%s_s23" % (kind, src)], rtol=1e-14, atol=1e-13)


def test_local_cm_oracle_orders(oracle_mod):
    # C at the origin, H at 1.0 and 2.0 on x, O at 1.5 on y
    z = np.array([6.0, 1.0, 1.0, 8.0])
    r = np.array([[0, 0, 0], [1.0, 0, 0], [2.0, 0, 0], [0, 1.5, 0]])
    loc = oracle_mod.local_coulomb_matrices(z, r, [0, 4], 4, "local")
    atm = oracle_mod.local_coulomb_matrices(z, r, [0, 4], 4, "atomic")
    # first diagonal entry is always the central atom
    for k in range(4):
        assert loc[k, 0] == atm[k, 0] == 0.5 * z[k] ** 2.4
    # atomic, centre H2 (index 2): H1 at 1.0, C at 2.0, O at 2.5
    diag = [atm[2, m * (m + 1) // 2 + m] for m in range(4)]
    np.testing.assert_allclose(diag, 0.5 * z[[2, 1, 0, 3]] ** 2.4)


def test_local_cm_oracle_ties(oracle_mod):
    # two H mirrored through C: equal row norms (higher index first) and
    # equal distances from C (lower index first)
    z = np.array([6.0, 1.0, 1.0])
    r = np.array([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0], [-1.1, 0.0, 0.0]])
    loc = oracle_mod.local_coulomb_matrices(z, r, [0, 3], 3, "local")
    atm = oracle_mod.local_coulomb_matrices(z, r, [0, 3], 3, "atomic")
    assert np.isfinite(loc).all() and np.isfinite(atm).all()
    # centre H1: local order is H1, C, H2; atomic order is H1, C, H2 too
    np.testing.assert_allclose(loc[1], atm[1])


@pytest.mark.parametrize("kind", ["gaussian", "laplacian"])
def test_vector_kernels_oracle_matches_numpy(oracle_mod, kind):
    b = synthetic.generate(14, nmax=9, seed=21, nmin=2)
    cm = oracle_mod.local_coulomb_matrices(b.charges, b.coords, b.offsets, 9, "local")
    x, n = _per_molecule(cm, b.offsets, 9)
    sig = [3.0, 30.0, 300.0] if kind == "gaussian" else [10.0, 100.0, 1000.0]
    K = oracle_mod.vector_kernels(kind, x[:6], x[6:], n[:6], n[6:], sig)
    np.testing.assert_allclose(K, _numpy_vector_kernels(kind, x[:6], x[6:], n[:6], n[6:], sig),
                               rtol=1e-13)


# ---------------------------------------------------------------- GPU parity
@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("src,pre", [("xyz", "xyz_"), ("syn", "syn12_")])
def test_local_cm_vs_reference_python(golden, kind, src, pre):
    import fml_b200
    g = golden
    cm = fml_b200.generate_local_coulomb_matrices(g[pre + "charges"], g[pre + "coords"],
                                                  g[pre + "offsets"], size=23, kind=kind)
    np.testing.assert_allclose(cm, g["lcm_%s_%s_s23" % (kind, src)], rtol=1e-14, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("nmax,seed,nmol", [(23, 3, 500), (40, 4, 60), (5, 5, 33), (1, 6, 7)])
def test_local_cm_vs_oracle(oracle_mod, kind, nmax, seed, nmol):
    import fml_b200
    b = synthetic.generate(nmol, nmax=nmax, seed=seed, nmin=1)
    cm = fml_b200.generate_local_coulomb_matrices(b.charges, b.coords, b.offsets, size=nmax,
                                                  kind=kind)
    ref = oracle_mod.local_coulomb_matrices(b.charges, b.coords, b.offsets, nmax, kind)
    np.testing.assert_allclose(cm, ref, rtol=1e-14, atol=0)


@pytest.mark.gpu
def test_local_cm_ties_and_molecule_dropin(oracle_mod, golden):
    import fml_b200
    z = np.array([6.0, 1.0, 1.0])
    r = np.array([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0], [-1.1, 0.0, 0.0]])
    for kind in KINDS:
        cm = fml_b200.generate_local_coulomb_matrices(z, r, [0, 3], size=4, kind=kind)
        np.testing.assert_array_equal(cm, oracle_mod.local_coulomb_matrices(z, r, [0, 3], 4,
                                                                            kind))
    g = golden
    off = g["xyz_offsets"]
    for i in range(len(off) - 1):
        m = fml_b200.Molecule()
        m.nuclear_charges = list(g["xyz_charges"][off[i]:off[i + 1]])
        m.coordinates = g["xyz_coords"][off[i]:off[i + 1]]
        m.natoms = len(m.nuclear_charges)
        m.generate_local_coulomb_matrix(size=23)
        m.generate_atomic_coulomb_matrix(size=23)
        np.testing.assert_allclose(m.local_coulomb_matrix,
                                   g["lcm_local_xyz_s23"][off[i]:off[i + 1]], rtol=1e-14,
                                   atol=1e-13)
        np.testing.assert_allclose(m.atomic_coulomb_matrix,
                                   g["lcm_atomic_xyz_s23"][off[i]:off[i + 1]], rtol=1e-14,
                                   atol=1e-13)
    with pytest.raises(ValueError):
        fml_b200.generate_local_coulomb_matrices(np.ones(5), np.random.rand(5, 3), [0, 5],
                                                 size=4)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gaussian", "laplacian"])
@pytest.mark.parametrize("nmax,nm1,nm2,seed", [(23, 40, 70, 7), (9, 17, 5, 8), (3, 4, 4, 9),
                                               (64, 6, 9, 10)])
def test_vector_kernels_vs_oracle(oracle_mod, kind, nmax, nm1, nm2, seed):
    import torch

    from fml_b200 import _lib
    from fml_b200.kernels import _vector_kernels
    b = synthetic.generate(nm1 + nm2, nmax=nmax, seed=seed, nmin=1)
    cm = oracle_mod.local_coulomb_matrices(b.charges, b.coords, b.offsets, nmax, "local")
    x, n = _per_molecule(cm, b.offsets, nmax)
    sig = [5.0, 50.0, 500.0] if kind == "gaussian" else [20.0, 200.0, 2000.0]
    ref = oracle_mod.vector_kernels(kind, x[:nm1], x[nm1:], n[:nm1], n[nm1:], sig)
    dev = torch.device("cuda", 0)
    x1 = torch.from_numpy(np.ascontiguousarray(x[:nm1])).to(dev)
    x2 = torch.from_numpy(np.ascontiguousarray(x[nm1:])).to(dev)
    K = _vector_kernels(0 if kind == "gaussian" else 1, x1, x2, n[:nm1], n[nm1:], sig)
    np.testing.assert_allclose(K.cpu().numpy(), ref, rtol=1e-13, atol=1e-300)
    assert _lib.load() is not None


@pytest.mark.gpu
def test_atomic_kernels_dropins(oracle_mod, golden):
    import fml_b200
    g = golden
    off = g["xyz_offsets"]
    mols = []
    for i in range(len(off) - 1):
        m = fml_b200.Molecule()
        m.nuclear_charges = list(g["xyz_charges"][off[i]:off[i + 1]])
        m.coordinates = g["xyz_coords"][off[i]:off[i + 1]]
        m.natoms = len(m.nuclear_charges)
        m.generate_local_coulomb_matrix(size=23)
        mols.append(m)
    sig = [10.0, 100.0]
    K = fml_b200.get_atomic_kernels_gaussian(mols[:4], mols[4:], sig)
    x, n = _per_molecule(g["lcm_local_xyz_s23"], off, int(np.diff(off).max()))
    ref = oracle_mod.vector_kernels("gaussian", x[:4], x[4:], n[:4], n[4:], sig)
    np.testing.assert_allclose(K, ref, rtol=1e-13)
    # laplacian drop-in takes the reference's (d, amax, nm) Fortran argument layout
    xf = np.asfortranarray(x.transpose(2, 1, 0))
    Kl = fml_b200.get_atomic_kernels_laplacian(xf[:, :, :4], xf[:, :, 4:], n[:4], n[4:], sig)
    refl = oracle_mod.vector_kernels("laplacian", x[:4], x[4:], n[:4], n[4:], sig)
    np.testing.assert_allclose(Kl, refl, rtol=1e-13)
    with pytest.raises(ValueError):
        fml_b200.get_atomic_kernels_laplacian(xf, xf, n, n, [-1.0])
    # the f2py routine exported as is: same arrays, explicit sizes
    Kf = fml_b200.fget_vector_kernels_gaussian(xf[:, :, :4], xf[:, :, 4:], n[:4], n[4:], sig, 4,
                                               len(n) - 4, 2)
    np.testing.assert_allclose(Kf, ref, rtol=1e-13)


# ------------------------------------------------------- unsorted Coulomb matrix
def _sorted_order_batch(oracle_mod, z, r, off, size):
    """Atoms of every molecule permuted into the sorted-CM order (the oracle's
    order, bit-exact against the reference's row-norm sort)."""
    _, order = oracle_mod.coulomb_matrices(z, r, off, size, return_order=True)
    idx = np.concatenate([off[m] + order[m][:off[m + 1] - off[m]] for m in range(len(off) - 1)])
    return z[idx], r[idx]


def test_unsorted_cm_oracle_pinned_by_permutation(golden, oracle_mod):
    """The unsorted CM of atoms already in sorted order is the sorted CM: the
    oracle against the reference's sorted matrices (representations.py:63-113),
    which pins it (the reference has no Python unsorted version)."""
    g = golden
    for pre, key in (("xyz_", "cm_xyz_s23"), ("syn12_", "cm_syn_s23")):
        z, r, off = g[pre + "charges"], g[pre + "coords"], g[pre + "offsets"]
        zs, rs = _sorted_order_batch(oracle_mod, z, r, off, 23)
        np.testing.assert_allclose(oracle_mod.unsorted_coulomb_matrices(zs, rs, off, 23), g[key],
                                   rtol=1e-14, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("nmax,seed,nmol", [(23, 13, 300), (40, 14, 50), (1, 15, 9)])
def test_unsorted_cm_vs_oracle(oracle_mod, golden, nmax, seed, nmol):
    import fml_b200
    b = synthetic.generate(nmol, nmax=nmax, seed=seed, nmin=1)
    cm = fml_b200.generate_unsorted_coulomb_matrices(b.charges, b.coords, b.offsets, size=nmax)
    np.testing.assert_allclose(cm, oracle_mod.unsorted_coulomb_matrices(b.charges, b.coords,
                                                                        b.offsets, nmax),
                               rtol=1e-14, atol=0)
    g = golden
    z, r, off = g["xyz_charges"], g["xyz_coords"], g["xyz_offsets"]
    zs, rs = _sorted_order_batch(oracle_mod, z, r, off, 23)
    m = fml_b200.Molecule()
    m.nuclear_charges = list(zs[off[2]:off[3]])
    m.coordinates = rs[off[2]:off[3]]
    m.natoms = len(m.nuclear_charges)
    m.generate_unsorted_coulomb_matrix(size=23)
    np.testing.assert_allclose(m.unsorted_coulomb_matrix, g["cm_xyz_s23"][2], rtol=1e-14,
                               atol=1e-13)
