"""GPU parity: every hot-path entry point against the CPU oracle and the
reference's golden fixtures, through the C ABI (libfmlb.so).

Tolerances (stated per test):
* Coulomb matrices: sort order bit-exact; values to 1e-14 relative.
* ARAD descriptors: 1e-12 relative / 1e-13 absolute (padding 1e100 exact).
* Gaussian / Laplacian FP64: 1e-12 relative.
* ARAD kernels FP64: 1e-12 relative against the oracle.
* cho_solve FP64: 1e-10 relative on well-conditioned systems; LAPACK info equal.
"""

import numpy as np
import pytest
import torch

import fml_b200
from fml_b200 import synthetic
from fml_b200.data import ptp_of

pytestmark = pytest.mark.gpu


def _mols(g, prefix):
    off = g[prefix + "offsets"]
    return [(g[prefix + "charges"][off[i]:off[i + 1]], g[prefix + "coords"][off[i]:off[i + 1]])
            for i in range(len(off) - 1)]


# ---------------------------------------------------------------------------
# descriptors
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("nmax,seed,nmol", [(23, 0, 700), (29, 2, 500), (5, 3, 64), (40, 4, 64)])
def test_coulomb_matrices_vs_oracle(oracle_mod, nmax, seed, nmol):
    b = synthetic.generate(nmol, nmax=nmax, seed=seed, nmin=1 if nmax < 6 else 4)
    cm, order = fml_b200.generate_coulomb_matrices(b.charges, b.coords, b.offsets, size=nmax,
                                                   return_order=True)
    ref, ref_order = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, nmax,
                                                 return_order=True)
    np.testing.assert_array_equal(order, ref_order)          # bit-exact permutation
    np.testing.assert_allclose(cm, ref, rtol=1e-14, atol=0)


def test_coulomb_matrix_ties_go_to_higher_index(oracle_mod):
    # two identical H atoms mirrored through the C: equal row norms
    z = np.array([6.0, 1.0, 1.0])
    r = np.array([[0.0, 0.0, 0.0], [1.1, 0.0, 0.0], [-1.1, 0.0, 0.0]])
    cm, order = fml_b200.generate_coulomb_matrices(z, r, [0, 3], size=4, return_order=True)
    _, ref_order = oracle_mod.generate_coulomb_matrix(z, r, 4, return_order=True)
    assert list(order[0, :3]) == list(ref_order) == [0, 2, 1]


@pytest.mark.parametrize("size", [23, 30])
def test_coulomb_matrices_vs_reference_python(golden, size):
    g = golden
    cm = fml_b200.generate_coulomb_matrices(g["xyz_charges"], g["xyz_coords"], g["xyz_offsets"],
                                            size=size)
    np.testing.assert_allclose(cm, g["cm_xyz_s%d" % size], rtol=1e-14, atol=1e-13)


def test_molecule_dropin(golden):
    g = golden
    for i, (z, r) in enumerate(_mols(g, "xyz_")):
        m = fml_b200.Molecule()
        m.nuclear_charges = list(z)
        m.coordinates = r
        m.natoms = len(z)
        m.generate_coulomb_matrix(size=23)
        np.testing.assert_allclose(m.coulomb_matrix, g["cm_xyz_s23"][i], rtol=1e-14, atol=1e-13)
        m.generate_arad_descriptor(size=30)
        np.testing.assert_allclose(m.arad_descriptor, g["arad_xyz_s30_c5"][i], rtol=1e-12,
                                   atol=1e-13)


def test_coulomb_oversize_raises():
    with pytest.raises(ValueError):
        fml_b200.generate_coulomb_matrices(np.ones(5), np.random.rand(5, 3), [0, 5], size=4)


@pytest.mark.parametrize("key,size,cut", [("xyz_s30_c5", 30, 5.0), ("xyz_s20_c5", 20, 5.0),
                                          ("xyz_s23_c1e+06", 23, 1e6)])
def test_arad_descriptors_vs_reference(golden, key, size, cut):
    g = golden
    d = fml_b200.generate_arad_descriptors(g["xyz_charges"], g["xyz_coords"], g["xyz_offsets"],
                                           size=size, cut=cut)
    np.testing.assert_allclose(d, g["arad_" + key], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("cut,nmax", [(5.0, 23), (1e6, 23), (5.0, 29), (3.0, 64)])
def test_arad_descriptors_vs_oracle(oracle_mod, cut, nmax):
    b = synthetic.generate(150, nmax=nmax, seed=21)
    d = fml_b200.generate_arad_descriptors(b.charges, b.coords, b.offsets, size=nmax, cut=cut)
    ref = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, nmax, cut)
    np.testing.assert_allclose(d, ref, rtol=1e-12, atol=1e-13)


def _canonical_neighbours(D):
    """Neighbour columns of every atom's (5, size) block sorted by all five
    channels: equal for two descriptors that differ only in the order of
    exactly equidistant neighbours."""
    out = np.empty_like(D)
    for m in range(D.shape[0]):
        for a in range(D.shape[1]):
            blk = D[m, a]
            order = np.lexsort(np.round(blk[::-1], 12))
            out[m, a] = blk[:, order]
    return out


@pytest.mark.parametrize("cut", [5.0, 1e6])
def test_arad_descriptors_exact_ties_vs_reference(golden, cut):
    """Molecules with exactly equidistant neighbours of different elements.
    The reference orders such ties by numpy's default argsort (arad.py:110,
    not stable above 16 entries); the kernel orders them by atom index. The
    descriptors agree as sets of neighbour records (1e-13), and the ARAD
    kernels built from them agree to 1e-12, since the kernel sums over all
    neighbour pairs."""
    g = golden
    d = fml_b200.generate_arad_descriptors(g["ties_charges"], g["ties_coords"], g["ties_offsets"],
                                           size=30, cut=cut)
    ref = g["arad_ties_s30_c%g" % cut]
    np.testing.assert_array_equal(d[:, :, 0, :], ref[:, :, 0, :])   # sorted distances
    np.testing.assert_allclose(_canonical_neighbours(d), _canonical_neighbours(ref), rtol=0,
                               atol=1e-13)
    off = g["ties_offsets"]
    Z = [list(g["ties_charges"][off[i]:off[i + 1]]) for i in range(len(off) - 1)]
    sig = [0.1, 1.0, 5.0]
    K = fml_b200.get_atomic_symmetric_kernels_arad(d, Z, sig)
    Kref = fml_b200.get_atomic_symmetric_kernels_arad(ref, Z, sig)
    np.testing.assert_allclose(K, Kref, rtol=1e-12, atol=0)


def test_arad_unknown_element_raises():
    with pytest.raises(KeyError):
        fml_b200.generate_arad_descriptors(np.array([1.0, 0.0]), np.random.rand(2, 3), [0, 2])


# ---------------------------------------------------------------------------
# Gaussian / Laplacian
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def cm_small(oracle_mod):
    b = synthetic.generate(523, nmax=23, seed=5)
    return oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 23)


@pytest.mark.parametrize("fn", ["gaussian_kernel", "laplacian_kernel"])
@pytest.mark.parametrize("sigma", [724.0, 50.0])
def test_pairwise_kernel_vs_oracle(oracle_mod, cm_small, fn, sigma):
    A = cm_small[:317].T  # reference layout (d, na)
    B = cm_small[317:].T
    K = getattr(fml_b200, fn)(A, B, sigma)
    ref = getattr(oracle_mod, fn)(A, B, sigma)
    assert K.shape == (317, 206)
    np.testing.assert_allclose(K, ref, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("fn", ["gaussian_kernel", "laplacian_kernel"])
def test_pairwise_kernel_symmetric_and_multi_sigma(oracle_mod, cm_small, fn):
    A = cm_small[:263].T
    sig = [100.0, 400.0, 1600.0]
    Ks = getattr(fml_b200, fn)(A, A, sig)              # A is A -> symmetric build
    Kf = getattr(fml_b200, fn)(A, A.copy(), sig)       # full build
    assert Ks.shape == (3, 263, 263)
    np.testing.assert_array_equal(Ks, Kf)
    for k, s in enumerate(sig):
        np.testing.assert_array_equal(Ks[k], Ks[k].T)
        np.testing.assert_allclose(Ks[k], getattr(oracle_mod, fn)(A, A, s), rtol=1e-12)


def test_pairwise_kernel_torch_in_torch_out(oracle_mod, cm_small):
    A = torch.from_numpy(cm_small[:64].T.copy()).cuda()
    K = fml_b200.gaussian_kernel(A, A, 300.0)
    assert isinstance(K, torch.Tensor) and K.is_cuda
    np.testing.assert_allclose(K.cpu().numpy(),
                               oracle_mod.gaussian_kernel(cm_small[:64].T, cm_small[:64].T, 300.0),
                               rtol=1e-12)


def test_pairwise_kernel_edge_sizes(oracle_mod):
    rng = np.random.default_rng(0)
    for na, nb, d in [(1, 1, 1), (1, 70, 3), (65, 1, 17), (129, 130, 33)]:
        A = rng.standard_normal((d, na))
        B = rng.standard_normal((d, nb))
        np.testing.assert_allclose(fml_b200.gaussian_kernel(A, B, 2.0),
                                   oracle_mod.gaussian_kernel(A, B, 2.0), rtol=1e-12)
        np.testing.assert_allclose(fml_b200.laplacian_kernel(A, B, 2.0),
                                   oracle_mod.laplacian_kernel(A, B, 2.0), rtol=1e-12)


# ---------------------------------------------------------------------------
# ARAD kernels
# ---------------------------------------------------------------------------
def test_arad_kernels_vs_reference_test(golden):
    """tests/test_arad.py:358-399 fixture comparison, now with an assertion."""
    g = golden
    x = g["arad_xyz_s30_c5"]
    Z = [list(z) for z, _ in _mols(g, "xyz_")]
    K = fml_b200.get_atomic_kernels_arad(x[:5], x[5:], Z[:5], Z[5:], list(g["testarad_sigmas"]))
    np.testing.assert_allclose(K, g["testarad_K_5v5"], rtol=1e-11)


@pytest.mark.parametrize("cut_desc", [5.0, 1e6])
def test_arad_kernels_vs_oracle(oracle_mod, cut_desc):
    b = synthetic.generate(40, nmax=23, seed=31)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 23, cut_desc)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    sig = [0.1, 0.5, 1.0, 2.0, 5.0]
    K = fml_b200.get_atomic_kernels_arad(X[:25], X[25:], Z[:25], Z[25:], sig)
    ref = oracle_mod.get_atomic_kernels_arad(X[:25], X[25:], Z[:25], Z[25:], sig)
    np.testing.assert_allclose(K, ref, rtol=1e-12, atol=1e-300)
    Ks = fml_b200.get_atomic_symmetric_kernels_arad(X, Z, sig)
    refs = oracle_mod.get_atomic_symmetric_kernels_arad(X, Z, sig)
    np.testing.assert_allclose(Ks, refs, rtol=1e-12, atol=1e-300)


def test_arad_kernels_fp32_error_bound(oracle_mod):
    b = synthetic.generate(40, nmax=23, seed=32)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 23, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    sig = [0.5, 1.0, 2.0, 5.0]
    K32 = fml_b200.get_atomic_symmetric_kernels_arad(X, Z, sig, precision="fp32")
    K64 = oracle_mod.get_atomic_symmetric_kernels_arad(X, Z, sig)
    rel = np.abs(K32 - K64) / np.maximum(np.abs(K64), 1e-300)
    assert rel.max() < 2e-3, rel.max()


# ---------------------------------------------------------------------------
# Cholesky
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [1, 63, 64, 65, 200, 700])
def test_cho_solve_vs_lapack(oracle_mod, cm_small, n):
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, n))
    A = M @ M.T / n + np.eye(n)
    y = rng.standard_normal(n)
    x = fml_b200.cho_solve(A, y)
    ref, info = oracle_mod.cho_solve(A, y)
    assert info == 0
    np.testing.assert_allclose(x, ref, rtol=1e-10, atol=1e-12)


def test_cho_solve_kernel_matrix(oracle_mod, cm_small):
    X = cm_small[:500]
    K = oracle_mod.gaussian_kernel(X.T, X.T, 724.0) + 1e-2 * np.eye(500)
    y = np.random.default_rng(1).standard_normal(500)
    x = fml_b200.cho_solve(K, y)
    ref, _ = oracle_mod.cho_solve(K, y)
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_cho_solve_reads_upper_triangle_only(oracle_mod):
    rng = np.random.default_rng(2)
    M = rng.standard_normal((90, 90))
    A = M @ M.T + 90 * np.eye(90)
    y = rng.standard_normal(90)
    B = A.copy()
    B[np.tril_indices(90, -1)] = 1e6  # garbage below the diagonal
    np.testing.assert_allclose(fml_b200.cho_solve(B, y), oracle_mod.cho_solve(A, y)[0],
                               rtol=1e-10)


def test_cho_solve_not_positive_definite_warns(oracle_mod):
    A = np.eye(150) * 2.0
    A[100, 100] = -1.0
    y = np.ones(150)
    with pytest.warns(fml_b200.CholeskyWarning, match="error code: 101"):
        fml_b200.cho_solve(A, y)
    assert oracle_mod.cho_solve(A, y)[1] == 101
    with pytest.raises(np.linalg.LinAlgError):
        fml_b200.cho_solve(A, y, strict=True)


@pytest.mark.parametrize("n", [1, 2, 5, 127, 128, 129, 300, 1031, 2304, 4099])
def test_cho_invert_vs_lapack(oracle_mod, n):
    rng = np.random.default_rng(100 + n)
    M = rng.standard_normal((n, n))
    A = M @ M.T / n + np.eye(n)
    A[np.tril_indices(n, -1)] += 3.0  # not symmetric: only the upper triangle is read
    out = fml_b200.cho_invert(A)
    ref, info, info2 = oracle_mod.cho_invert(A)
    assert info == info2 == 0
    assert out.flags["F_CONTIGUOUS"] and out.shape == (n, n)
    iu, il = np.triu_indices(n), np.tril_indices(n, -1)
    np.testing.assert_allclose(out[iu], ref[iu], rtol=1e-10, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_array_equal(out[il], A[il])  # untouched, as LAPACK leaves it


def test_cho_invert_kernel_matrix_and_torch(oracle_mod):
    import torch
    b = synthetic.generate(1500, nmax=23, seed=55)
    X = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 23)
    K = oracle_mod.gaussian_kernel(X.T, X.T, 724.0) + 1e-3 * np.eye(1500)
    ref, _, _ = oracle_mod.cho_invert(K)
    Kt = torch.from_numpy(K).cuda()
    out = fml_b200.cho_invert(Kt)
    assert out.is_cuda
    iu = np.triu_indices(1500)
    o = out.cpu().numpy()
    np.testing.assert_allclose(o[iu], ref[iu], rtol=1e-8, atol=1e-9 * np.abs(ref).max())
    # alpha = inv(K) y through the symmetric inverse equals the solve
    y = np.random.default_rng(3).standard_normal(1500)
    full = np.triu(o) + np.triu(o, 1).T
    np.testing.assert_allclose(full @ y, oracle_mod.cho_solve(K, y)[0], rtol=1e-7,
                               atol=1e-8 * np.abs(full @ y).max())


def test_cho_invert_not_positive_definite(oracle_mod):
    A = np.eye(300) * 2.0
    A[200, 200] = -1.0
    with pytest.warns(fml_b200.CholeskyWarning, match="error code: 201"):
        out = fml_b200.cho_invert(A)
    assert np.isnan(out[np.triu_indices(300)]).all()
    assert oracle_mod.cho_invert(A)[1] == 201
    with pytest.raises(np.linalg.LinAlgError):
        fml_b200.cho_invert(A, strict=True)
    with pytest.raises(ValueError):
        fml_b200.cho_invert(np.ones((3, 4)))


# ---------------------------------------------------------------------------
# end to end: plain FP64 KRR on sorted Coulomb matrices (2000 molecules)
# ---------------------------------------------------------------------------
def test_krr_plain_fp64_end_to_end(oracle_mod):
    b = synthetic.generate(2000, nmax=23, seed=0)
    X = fml_b200.generate_coulomb_matrices(b.charges, b.coords, b.offsets, size=23)
    Xr = oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 23)
    np.testing.assert_allclose(X, Xr, rtol=1e-14)
    tr, te = slice(0, 1000), slice(1000, 2000)
    sigma, lam = 724.0, 1e-8
    K = fml_b200.gaussian_kernel(X[tr].T, X[tr].T, sigma)
    K[np.diag_indices_from(K)] += lam
    alpha = fml_b200.cho_solve(K, b.energies[tr])
    Ks = fml_b200.gaussian_kernel(X[te].T, X[tr].T, sigma)
    mae = np.abs(Ks @ alpha - b.energies[te]).mean()
    Kr = oracle_mod.gaussian_kernel(Xr[tr].T, Xr[tr].T, sigma)
    Kr[np.diag_indices_from(Kr)] += lam
    ar, _ = oracle_mod.cho_solve(Kr, b.energies[tr])
    mae_r = np.abs(oracle_mod.gaussian_kernel(Xr[te].T, Xr[tr].T, sigma) @ ar
                   - b.energies[te]).mean()
    assert abs(mae - mae_r) <= 1e-6 * mae_r, (mae, mae_r)


@pytest.mark.parametrize("m,k,ld_pad", [(1, 1, 0), (130, 128, 0), (257, 128, 1), (300, 37, 3)])
def test_syrk_lower_update(m, k, ld_pad):
    """C -= P P^T on the lower triangle only (FP64 tensor-core kernel), aligned
    (even stride) and unaligned (odd stride) operand paths, 1e-13 relative."""
    from fml_b200 import _lib
    rng = np.random.default_rng(m + k)
    ld = max(m, k) + ld_pad
    buf = rng.standard_normal((m, ld))
    P = rng.standard_normal((m, k))
    Pbuf = np.zeros((m, ld))
    Pbuf[:, :k] = P
    C = torch.from_numpy(buf.copy()).cuda()
    Pd = torch.from_numpy(Pbuf).cuda()
    _lib.call("fmlb_syrk_lower_f64", _lib.ptr(C), ld, m, _lib.ptr(Pd), ld, k, 0, None,
              _lib.stream_handle())
    out = C.cpu().numpy()
    ref = buf[:, :m] - P @ P.T
    low = np.tril_indices(m)
    np.testing.assert_allclose(out[:, :m][low], ref[low], rtol=1e-13, atol=1e-12)
    up = np.triu_indices(m, 1)
    np.testing.assert_array_equal(out[:, :m][up], buf[:, :m][up])


@pytest.mark.parametrize("n", [1031, 2304])
def test_cho_solve_multi_panel(oracle_mod, n):
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, n // 2))
    A = M @ M.T / n + 0.5 * np.eye(n)
    y = rng.standard_normal(n)
    x = fml_b200.cho_solve(A, y)
    ref, info = oracle_mod.cho_solve(A, y)
    assert info == 0
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-10 * np.abs(ref).max())


def test_cho_solve_wide_outer_panels(oracle_mod):
    """n >= 16384 factors with 1024-column outer panels (16 full panels and a
    partial one here)."""
    n = 16500
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, 64))
    A = M @ M.T / 64 + 0.5 * np.eye(n)
    y = rng.standard_normal(n)
    x = fml_b200.cho_solve(A, y)
    ref, info = oracle_mod.cho_solve(A, y)
    assert info == 0
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("bad", [1, 33, 300, 1000])
def test_cho_solve_failure_column_matches_lapack(oracle_mod, bad):
    n = 1031
    A = np.eye(n) * 3.0 + 0.01
    A[bad - 1, bad - 1] = -5.0
    y = np.ones(n)
    with pytest.warns(fml_b200.CholeskyWarning, match="error code: %d$" % bad):
        fml_b200.cho_solve(A, y)
    assert oracle_mod.cho_solve(A, y)[1] == bad


# ---------------------------------------------------------------------------
# tensor-core (tcgen05) Gaussian, BF16 hi/lo x3, FP32 output
# Stated error bound: |K_tc - K_fp64| <= 2e-4 absolute for sigma >= 100 on
# Coulomb matrices (6e-5 measured at sigma = 100 in a numpy emulation).
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def cm_large(oracle_mod):
    b = synthetic.generate(700, nmax=29, seed=41)
    return oracle_mod.coulomb_matrices(b.charges, b.coords, b.offsets, 29)


@pytest.mark.parametrize("na,nb", [(300, 300), (130, 257), (1, 129), (600, 1), (333, 64),
                                   (129, 516)])
def test_gaussian_tc_vs_fp64(oracle_mod, cm_large, na, nb):
    A = cm_large[:na].T
    B = cm_large[-nb:].T
    sig = [100.0, 400.0, 1600.0]
    K = fml_b200.gaussian_kernel(A, B, sig, precision="bf16x3")
    assert K.dtype == np.float32 and K.shape == (3, na, nb)
    for k, s in enumerate(sig):
        ref = oracle_mod.gaussian_kernel(A, B, s)
        assert np.abs(K[k] - ref).max() <= 2e-4, (s, np.abs(K[k] - ref).max())


@pytest.mark.parametrize("n", [517, 300, 640])
def test_gaussian_tc_symmetric_exact(oracle_mod, cm_large, n):
    """n = 517: per-element stores (rows not 16-byte aligned); 300 and 640:
    TMA bulk-tensor stores of the off-diagonal tiles, partial and whole."""
    A = cm_large[:n].T
    sig = [100.0, 1600.0]
    K = fml_b200.gaussian_kernel(A, A, sig, precision="bf16x3")
    for k, s in enumerate(sig):
        np.testing.assert_array_equal(K[k], K[k].T)
        np.testing.assert_array_equal(np.diag(K[k]), 1.0)
        ref = oracle_mod.gaussian_kernel(A, A, s)
        assert np.abs(K[k] - ref).max() <= 2e-4


def test_gaussian_tc_wait_timeout_reports_and_recovers(oracle_mod, cm_large):
    """Every mbarrier wait of the tcgen05 kernel is bounded. With the test hook
    set (waits of 20000 cycles, the TMA producer issues no copies) the MMA and
    epilogue waits run out with nothing in flight: the call raises FmlbError
    (FMLB_ETIMEDOUT) and the context stays usable, so the next call matches
    the oracle."""
    from fml_b200 import _lib
    A = cm_large[:300].T
    try:
        _lib.call("fmlb_tc_test_hooks", 20000, 1)
        with pytest.raises(_lib.FmlbError) as err:
            fml_b200.gaussian_kernel(A, A, [400.0], precision="bf16x3")
    finally:
        _lib.call("fmlb_tc_test_hooks", 0, 0)
    assert err.value.code == _lib.FMLB_ETIMEDOUT
    K = fml_b200.gaussian_kernel(A, A, [400.0], precision="bf16x3")
    assert np.abs(K[0] - oracle_mod.gaussian_kernel(A, A, 400.0)).max() <= 2e-4


@pytest.mark.parametrize("m,strip", [(300, 128), (100, 128), (257, 64)])
def test_syrk_lower_strip(m, strip):
    """strip_cols > 0 updates only the first strip_cols columns of the lower triangle."""
    from fml_b200 import _lib
    rng = np.random.default_rng(m)
    k = 128
    buf = rng.standard_normal((m, m))
    P = rng.standard_normal((m, k))
    C = torch.from_numpy(buf.copy()).cuda()
    Pd = torch.from_numpy(P).cuda()
    _lib.call("fmlb_syrk_lower_f64", _lib.ptr(C), m, m, _lib.ptr(Pd), k, k, strip, None,
              _lib.stream_handle())
    out = C.cpu().numpy()
    ref = buf - P @ P.T
    r, c = np.indices((m, m))
    upd = (c <= r) & (c < strip)
    np.testing.assert_allclose(out[upd], ref[upd], rtol=1e-13, atol=1e-12)
    np.testing.assert_array_equal(out[~upd], buf[~upd])


def test_cho_solve_512_outer_panels(oracle_mod):
    """n >= 8192 takes 512-column outer panels; n = 8300 ends in a partial one."""
    n = 8300
    rng = np.random.default_rng(7)
    M = rng.standard_normal((n, 600))
    A = M @ M.T / 600 + 0.25 * np.eye(n)
    y = rng.standard_normal(n)
    x = fml_b200.cho_solve(A, y)
    ref, info = oracle_mod.cho_solve(A, y)
    assert info == 0
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-10 * np.abs(ref).max())
    B = A.copy()
    B[5001, 5001] = -1.0
    with pytest.warns(fml_b200.CholeskyWarning, match="error code: 5002$"):
        fml_b200.cho_solve(B, y)


def _arad_set(oracle_mod, nmol, nmax, seed, cut, zpool=None):
    b = synthetic.generate(nmol, nmax=nmax, seed=seed)
    charges = b.charges.copy()
    if zpool is not None:
        rng = np.random.default_rng(seed)
        charges = rng.choice(np.asarray(zpool, dtype=np.float64), size=len(charges))
    X = oracle_mod.arad_descriptors(charges, b.coords, b.offsets, nmax, cut)
    Z = [charges[b.offsets[i]:b.offsets[i + 1]] for i in range(nmol)]
    return X, Z


@pytest.mark.parametrize("nmol,nmax,seed", [(40, 23, 61), (301, 12, 62), (1, 5, 63)])
def test_fget_alpha_arad_vs_oracle(oracle_mod, nmol, nmax, seed):
    X, Z = _arad_set(oracle_mod, nmol, nmax, seed, 1e6)
    n = np.array([len(z) for z in Z], np.int32)
    zp = np.zeros((nmol, nmax, 2))
    for i, z in enumerate(Z):
        zp[i, :len(z)] = ptp_of(z)
    y = np.random.default_rng(seed).standard_normal(nmol)
    ref, info, info2 = oracle_mod.fget_alpha_arad(X, zp, n, y, 2.0, 1e-2)
    assert info == info2 == 0
    alpha = np.zeros(n.sum() + 3)  # f2py intent(inout): filled in place, the rest zeroed
    alpha[-1] = 7.0
    assert fml_b200.fget_alpha_arad(X, zp, n, y, 2.0, 1e-2, alpha) is None
    np.testing.assert_allclose(alpha[:n.sum()], ref, rtol=1e-8, atol=1e-10 * np.abs(ref).max())
    assert (alpha[n.sum():] == 0).all()
    np.testing.assert_array_equal(fml_b200.fget_alpha_arad(X, zp, n, y, 2.0, 1e-2),
                                  alpha[:n.sum()])


def test_l2_distance_arad_vs_reference_test_and_oracle(golden, oracle_mod):
    """get_l2_distance_arad against the reference test's own distance matrix
    (tests/test_arad.py:358-363 compares the two) and the oracle; exp-sums of
    it reproduce the molecular kernel (tests/test_arad.py:379-387)."""
    g = golden
    x = g["arad_xyz_s30_c5"]
    off = g["xyz_offsets"]
    Z = [g["xyz_charges"][off[i]:off[i + 1]] for i in range(len(off) - 1)]
    D = fml_b200.get_l2_distance_arad(x[:5], x[5:], Z[:5], Z[5:])
    Da = g["testarad_D_5v5"]
    ok = ~np.isnan(Da)
    np.testing.assert_allclose(D[ok], Da[ok], rtol=1e-12, atol=1e-13)
    assert (D[~ok] == 0).all()
    np.testing.assert_allclose(D, oracle_mod.get_l2_distance_arad(x[:5], x[5:], Z[:5], Z[5:]),
                               rtol=1e-12, atol=1e-13)
    Ka = np.zeros((4, 5, 5))
    for s, sigma in enumerate(g["testarad_sigmas"]):
        Ka[s] = np.nansum(np.exp(np.where(ok, D, np.nan) * (-1.0 / sigma ** 2)), axis=(-2, -1))
    np.testing.assert_allclose(Ka, g["testarad_K_5v5"], rtol=1e-11)


@pytest.mark.parametrize("nm1,nm2,nmax,seed", [(37, 21, 23, 71), (3, 50, 9, 72)])
def test_l2_distance_arad_synthetic(oracle_mod, nm1, nm2, nmax, seed):
    X, Z = _arad_set(oracle_mod, nm1 + nm2, nmax, seed, 1e6)
    D = fml_b200.get_l2_distance_arad(X[:nm1], X[nm1:], Z[:nm1], Z[nm1:])
    ref = oracle_mod.get_l2_distance_arad(X[:nm1], X[nm1:], Z[:nm1], Z[nm1:])
    np.testing.assert_allclose(D, ref, rtol=1e-12, atol=1e-12)


def test_fget_kernel_arad_vs_oracle(oracle_mod):
    X, Z = _arad_set(oracle_mod, 30, 12, 65, 1e6)
    n = np.array([len(z) for z in Z], np.int32)
    zp = np.zeros((30, 12, 2))
    for i, z in enumerate(Z):
        zp[i, :len(z)] = ptp_of(z)
    K = fml_b200.fget_kernel_arad(X, zp, n, 1.5, 25)  # the first 25 molecules
    assert K.shape == (25, 25)
    np.testing.assert_allclose(K, oracle_mod.fget_kernel_arad(X, zp, n, 1.5, 25), rtol=1e-12)


def test_fget_alpha_arad_not_positive_definite(oracle_mod):
    X, Z = _arad_set(oracle_mod, 6, 8, 64, 1e6)
    n = np.array([len(z) for z in Z], np.int32)
    zp = np.zeros((6, 8, 2))
    for i, z in enumerate(Z):
        zp[i, :len(z)] = ptp_of(z)
    with pytest.warns(fml_b200.CholeskyWarning, match="DPOTRF"):
        out = fml_b200.fget_alpha_arad(X, zp, n, np.ones(6), 2.0, -1e6)
    assert np.isnan(out).all()


@pytest.mark.parametrize("zpool,nmax", [(None, 23), ([1, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 14, 15,
                                                      16, 17, 19, 20, 35], 23), (None, 40)])
def test_arad_fp32_paths_vs_fp64(oracle_mod, zpool, nmax):
    """FP32 ARAD kernels (the fast path for <= 16 element classes and amax <= 32,
    the generic path otherwise) against the FP64 oracle: relative error <= 2e-3
    for sigma >= 0.5 (FP32 cancellation in l2 = s1 + s2 - 2 S stoch)."""
    X, Z = _arad_set(oracle_mod, 30, nmax, 77, 1e6, zpool)
    sig = [0.5, 1.0, 2.0, 5.0]
    K32 = fml_b200.get_atomic_kernels_arad(X[:17], X[17:], Z[:17], Z[17:], sig, precision="fp32")
    K64 = oracle_mod.get_atomic_kernels_arad(X[:17], X[17:], Z[:17], Z[17:], sig)
    rel = np.abs(K32 - K64) / np.maximum(np.abs(K64), 1e-300)
    assert rel.max() < 2e-3, rel.max()
    S32 = fml_b200.get_atomic_symmetric_kernels_arad(X, Z, sig, precision="fp32")
    S64 = oracle_mod.get_atomic_symmetric_kernels_arad(X, Z, sig)
    rel = np.abs(S32 - S64) / np.maximum(np.abs(S64), 1e-300)
    assert rel.max() < 2e-3, rel.max()
    np.testing.assert_array_equal(S32, np.swapaxes(S32, 1, 2))


@pytest.mark.parametrize("cut", [1e6, 5.0])
def test_arad_fp32_sigma_01_tolerance(oracle_mod, cut):
    """sigma = 0.1 (the smallest sigma of the ARAD configuration): every FP32
    kernel entry above 1e-30 of the largest within 1e-3 relative of the FP64
    one (3.3e-4 measured on 400-molecule sets). Smaller entries (exp(-100 l2)
    of distant environments, down to 1e-40 and below) lie under FP32's
    normal range and flush to zero. The exponent -l2/sigma^2 is 100 l2 here,
    so the FP32 cancellation error of l2 is magnified 25x against
    sigma = 0.5."""
    X, Z = _arad_set(oracle_mod, 120, 23, 1, cut)
    sig = [0.1]
    K32 = fml_b200.get_atomic_symmetric_kernels_arad(X, Z, sig, precision="fp32")
    K64 = fml_b200.get_atomic_symmetric_kernels_arad(X, Z, sig)
    big = np.abs(K64) > 1e-30 * np.abs(K64).max()
    rel = np.abs(K32 - K64)[big] / np.abs(K64)[big]
    assert rel.max() < 1e-3, rel.max()
    A32 = fml_b200.get_atomic_kernels_arad(X[:60], X[60:], Z[:60], Z[60:], sig, precision="fp32")
    A64 = fml_b200.get_atomic_kernels_arad(X[:60], X[60:], Z[:60], Z[60:], sig)
    big = np.abs(A64) > 1e-30 * np.abs(A64).max()
    rel = np.abs(A32 - A64)[big] / np.abs(A64)[big]
    assert rel.max() < 1e-3, rel.max()


def test_arad_fp32_fixtures_sigma_sweep(golden):
    """Reference fixtures (tests/test_arad.py sigmas): FP32 max-abs error stated per sigma."""
    g = golden
    x = g["arad_xyz_s30_c5"]
    Z = [list(z) for z, _ in _mols(g, "xyz_")]
    K32 = fml_b200.get_atomic_kernels_arad(x[:5], x[5:], Z[:5], Z[5:], list(g["testarad_sigmas"]),
                                           precision="fp32")
    ref = g["testarad_K_5v5"]
    for k in range(len(g["testarad_sigmas"])):
        assert np.abs(K32[k] - ref[k]).max() <= 2e-3 * np.abs(ref[k]).max() + 1e-6


@pytest.mark.parametrize("na,nb", [(300, 300), (130, 257), (1, 129)])
def test_laplacian_fp32_vs_fp64(oracle_mod, cm_large, na, nb):
    """FP32 Laplacian: relative error <= 1e-4 where K > 1e-30 (FP32 L1 sums)."""
    A = cm_large[:na].T
    B = cm_large[-nb:].T
    sig = [100.0, 400.0, 1600.0]
    K = fml_b200.laplacian_kernel(A, B, sig, precision="fp32")
    assert K.dtype == np.float32
    for k, s in enumerate(sig):
        ref = oracle_mod.laplacian_kernel(A, B, s)
        big = ref > 1e-30
        assert (np.abs(K[k][big] - ref[big]) / ref[big]).max() <= 1e-4
        assert np.abs(K[k][~big]).max(initial=0.0) <= 1e-30


def test_laplacian_fp32_symmetric(cm_large):
    A = cm_large[:333].T
    K = fml_b200.laplacian_kernel(A, A, [200.0, 800.0], precision="fp32")
    for k in range(2):
        np.testing.assert_array_equal(K[k], K[k].T)
        np.testing.assert_array_equal(np.diag(K[k]), 1.0)


# ---------------------------------------------------------------------------
# FP64 residual and iterative refinement (extension; the reference solves once)
# Tolerances: the residual itself 1e-12 relative to numpy when it is far from
# the rounding floor; refined x against LAPACK to 1e-5 relative at cond 1e9.
# ---------------------------------------------------------------------------
def test_residual_kernel_matches_numpy():
    from fml_b200 import _lib
    rng = np.random.default_rng(21)
    n, lam = 777, 0.37
    M = rng.standard_normal((n, n))
    K = M + M.T
    y = rng.standard_normal(n)
    x = rng.standard_normal(n)
    dev = torch.device("cuda")
    Kd = torch.from_numpy(K).to(dev)
    yd, xd = torch.from_numpy(y).to(dev), torch.from_numpy(x).to(dev)
    lib = _lib.load()
    scratch = torch.empty(lib.fmlb_krr_refine_scratch_doubles(n), dtype=torch.float64, device=dev)
    resid = torch.empty(1, dtype=torch.float64, device=dev)
    work = torch.empty(256, dtype=torch.uint8, device=dev)
    _lib.call("fmlb_krr_refine_f64", _lib.ptr(Kd), n, n, lam, _lib.ptr(Kd), n, _lib.ptr(work),
              _lib.ptr(yd), _lib.ptr(xd), 0, _lib.ptr(resid), _lib.ptr(scratch),
              _lib.stream_handle())
    r = y - K @ x - lam * x
    np.testing.assert_allclose(scratch[:n].cpu().numpy(), r, rtol=1e-12, atol=1e-12 * np.abs(r).max())
    np.testing.assert_allclose(resid.item(), np.linalg.norm(r), rtol=1e-12)
    np.testing.assert_array_equal(xd.cpu().numpy(), x)  # iters = 0 leaves x alone


def test_symmetrize_lower():
    from fml_b200 import _lib
    rng = np.random.default_rng(22)
    n = 130
    A = rng.standard_normal((n, n))
    Ad = torch.from_numpy(A).cuda()
    _lib.call("fmlb_symmetrize_lower_f64", _lib.ptr(Ad), n, n, _lib.stream_handle())
    L = np.tril(A)
    np.testing.assert_array_equal(Ad.cpu().numpy(), L + np.tril(A, -1).T)


def test_cho_solve_refinement(oracle_mod):
    n = 600
    rng = np.random.default_rng(11)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q * np.logspace(0, -9, n)) @ Q.T  # condition number 1e9
    A = (A + A.T) / 2
    y = rng.standard_normal(n)
    B = A.copy()
    B[np.tril_indices(n, -1)] = 7.0  # only the upper triangle is read, refinement included
    x0, r0 = fml_b200.cho_solve(B, y, return_residuals=True)
    x2, r2 = fml_b200.cho_solve(B, y, refine=2, return_residuals=True)
    assert r0.shape == (1,) and r2.shape == (3,)
    np.testing.assert_array_equal(x0, fml_b200.cho_solve(B, y))
    assert r2[-1] <= 1.5 * r2[0]
    ref, info = oracle_mod.cho_solve(A, y)
    assert info == 0
    np.testing.assert_allclose(x2, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


# ---------------------------------------------------------------------------
# atom-level ARAD kernel (fget_atomic_kernels_arad) against the oracle, FP64,
# 1e-12 relative; different descriptor widths for the two sets, a cut that
# ends some neighbour lists early
# ---------------------------------------------------------------------------
def test_atomic_kernels_arad_vs_oracle(oracle_mod):
    from tests.test_arad_atomic_cpu import atoms_of
    b = synthetic.generate(14, nmax=12, seed=12)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 12, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    q, z, n, _ = atoms_of(X, Z)
    q1, z1, n1 = q[:70], z[:70], n[:70]
    q2, z2, n2 = q[50:, :, :10], z[50:], np.minimum(n[50:], 10)
    sig = [0.3, 1.0, 4.0]
    for cut in (6.0, 3.0):
        got = fml_b200.fget_atomic_kernels_arad(q1, q2, z1, z2, n1, n2, sig, len(q1), len(q2),
                                                len(sig), 0.2, cut, 1.0, 0.5)
        ref = oracle_mod.fget_atomic_kernels_arad(q1, q2, z1, z2, n1, n2, sig, len(q1), len(q2),
                                                  len(sig), 0.2, cut, 1.0, 0.5)
        assert got.shape == (3, 70, len(q2))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-300)
    same = fml_b200.fget_atomic_kernels_arad(q1, q1, z1, z1, n1, n1, sig, 70, 70, 3, 0.2, 6.0,
                                             1.0, 0.5)
    for k in range(3):
        np.testing.assert_array_equal(np.diag(same[k]), 1.0)


def test_atomic_distance_arad_vs_oracle(oracle_mod):
    from tests.test_arad_atomic_cpu import atoms_of
    b = synthetic.generate(10, nmax=11, seed=13)
    X = oracle_mod.arad_descriptors(b.charges, b.coords, b.offsets, 11, 1e6)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    q, z, n, _ = atoms_of(X, Z)
    q1, q2 = q[:40], q[-40:]
    z1, z2, n1, n2 = z[:40], z[-40:], n[:40], n[-40:]
    got = fml_b200.fget_atomic_distance_arad(q1, q2, z1, z2, n1, n2, 40, 40, 0.2, 6.0, 1.0, 0.5)
    D = oracle_mod.atomic_distances_arad(q1, q2, z1, z2, n1, n2, 0.2, 6.0, 1.0, 0.5)
    np.testing.assert_allclose(got, D.T, rtol=1e-12, atol=1e-12 * np.abs(D).max())
    with pytest.raises(ValueError):
        fml_b200.fget_atomic_distance_arad(q1, q2[:5], z1, z2[:5], n1, n2[:5], 40, 5, 0.2, 6.0,
                                           1.0, 0.5)
