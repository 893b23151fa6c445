"""Host-side logic that needs no GPU: tables, marshalling, generators, errors."""

import os

import numpy as np
import pytest
import torch

import fml_b200
from fml_b200 import data, synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_ptp_of_matches_table():
    z = np.array([1, 6, 7, 8, 16, 101, 102])
    np.testing.assert_array_equal(data.ptp_of(z), [[1, 1], [2, 4], [2, 5], [2, 6], [3, 6],
                                                   [7, 32], [7, 14]])
    with pytest.raises(KeyError):
        data.ptp_of([0])
    with pytest.raises(KeyError):
        data.ptp_of([119])


def test_synthetic_generator_is_seeded_and_valid():
    a = synthetic.generate(50, nmax=23, seed=7)
    b = synthetic.generate(50, nmax=23, seed=7)
    np.testing.assert_array_equal(a.coords, b.coords)
    np.testing.assert_array_equal(a.energies, b.energies)
    n = a.natoms
    assert n.min() >= 4 and n.max() <= 23
    assert set(np.unique(a.charges)) <= {1.0, 6.0, 7.0, 8.0, 16.0}
    for i in range(a.nmol):
        z, r = a.molecule(i)
        d = np.sqrt(((r[:, None] - r[None]) ** 2).sum(-1))
        assert (d[np.triu_indices(len(z), 1)] >= synthetic.MIN_PAIR_DIST).all()
        assert (np.linalg.norm(r, axis=1) <= 1.5 * len(z) ** (1 / 3) + 1e-12).all()
    sub = a.subset([3, 1])
    assert sub.nmol == 2 and sub.natoms[0] == a.natoms[3]


def test_read_xyz(tmp_path):
    p = tmp_path / "m.xyz"
    p.write_text("3\ncomment\n O 0.0 0.0 0.1\n H 0.7 0.0 -0.4\n H -0.7 0.0 -0.4\n")
    m = fml_b200.Molecule()
    m.read_xyz(str(p))
    assert m.natoms == 3
    assert m.nuclear_charges == [8, 1, 1]
    assert m.coordinates.shape == (3, 3)


def test_no_cpu_fallback_without_gpu():
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        fml_b200.gaussian_kernel(np.ones((4, 3)), np.ones((4, 2)), 1.0)


def test_cho_solve_shape_errors():
    with pytest.raises(ValueError, match="expected square matrix"):
        fml_b200.cho_solve(np.ones((3, 4)), np.ones(3))
    with pytest.raises(ValueError, match="same stride size"):
        fml_b200.cho_solve(np.eye(3), np.ones(4))


def test_arad_size_asserts():
    X = np.zeros((2, 5, 5, 5))
    with pytest.raises(AssertionError, match="code = 2"):
        fml_b200.get_atomic_kernels_arad(X, np.zeros((2, 4, 5, 4)), [[1], [1]], [[1], [1]], [1.0])
    with pytest.raises(AssertionError, match="code = 4"):
        fml_b200.get_atomic_symmetric_kernels_arad(X, [[1]], [1.0])


def test_autotune_cache_roundtrip(tmp_path, monkeypatch):
    from fml_b200 import autotune
    from fml_b200.batched import GaussianProblem
    monkeypatch.setenv("FMLB_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    monkeypatch.setenv("FMLB_AUTOTUNE", "0")
    probs = [GaussianProblem(np.zeros((n, 3)), np.zeros(n), np.zeros((2, 3)), 1.0, 1e-3)
             for n in (100, 300, 3000)]
    assert autotune.batched_config(probs) == autotune.DEFAULT
    key = "batched_krr|%s|%s" % (autotune.shape_class(probs), autotune.gpu_key())
    autotune._store({key: {"split_threshold": 2048, "grid": 296}})
    assert autotune.batched_config(probs)["split_threshold"] == 2048


def test_serving_ptp_packing_matches_reference_marshalling():
    from fml_b200 import synthetic
    from fml_b200.kernels import _ptp_arrays
    from fml_b200.serving import _ptp_packed
    b = synthetic.generate(40, nmax=17, seed=8)
    Z = [b.molecule(i)[0] for i in range(b.nmol)]
    ref, nref = _ptp_arrays(Z, 17)
    got, n = _ptp_packed(b.charges, b.offsets, 17)
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal(n, nref)
    with pytest.raises(KeyError):
        _ptp_packed(np.array([1.0, 200.0]), np.array([0, 2]), 4)


@pytest.mark.parametrize("fn", ["generate_coulomb_matrices", "generate_local_coulomb_matrices",
                                "generate_arad_descriptors"])
def test_descriptor_offsets_checked_before_launch(fn):
    """Offsets past the charge / coordinate buffers are rejected on the host."""
    import fml_b200
    z, r = np.ones(4), np.zeros((4, 3))
    with pytest.raises(ValueError):
        getattr(fml_b200, fn)(z, r, [0, 2, 6], size=8)
    with pytest.raises(ValueError):
        getattr(fml_b200, fn)(z, r, [-1, 2], size=8)


def test_segment_sums_and_counts():
    """Per-molecule sums of per-atom values (fkernels.f90:532-535, :696-698),
    including empty molecules, and the atom-count checks."""
    from fml_b200.kernels import _counts, _segment_sums
    n, off = _counts([2, 0, 3, 0], "t")
    assert n.tolist() == [2, 0, 3, 0] and off.tolist() == [0, 2, 2, 5, 5]
    v = np.arange(1.0, 7.0)  # one extra value past the last molecule is ignored
    np.testing.assert_array_equal(_segment_sums(v, off), [3.0, 0.0, 12.0, 0.0])
    np.testing.assert_array_equal(_segment_sums(v, _counts([0, 0], "t")[1]), [0.0, 0.0])
    with pytest.raises(ValueError):
        _counts([1, -1], "t")


def test_vector_kernel_dropin_checks_sizes():
    with pytest.raises(ValueError):
        fml_b200.fget_vector_kernels_gaussian(np.zeros((3, 2, 4)), np.zeros((3, 2, 5)),
                                              [1] * 4, [1] * 5, [1.0], 4, 4, 1)


def _reference_ptp_marshalling(Z, amax):
    """The loops of kernels.py:261-292 (get_atomic_kernels_arad), restated
    with the reference's PTP dict, for comparison with the vectorised form."""
    from fml_b200.data import PTP
    N = np.array([len(z) for z in Z], dtype=np.int32)
    c = [np.array([PTP[int(q)] for q in z], dtype=np.int32) for z in Z]
    out = np.zeros((len(Z), amax, 2))
    for i in range(len(Z)):
        for j, p in enumerate(c[i]):
            out[i, j] = p
    return out, N


def _outcome(fn, *args):
    try:
        return fn(*args)
    except (KeyError, IndexError, ValueError, OverflowError) as e:
        return type(e), e.args[:1] if isinstance(e, KeyError) else ()


from hypothesis import given, settings  # noqa: E402
from hypothesis import strategies as hst  # noqa: E402

_CHARGE = hst.one_of(hst.sampled_from([1.0, 6.0, 7.0, 8.0, 16.0, 9.0, 17.0, 35.0, 53.0]),
                     hst.floats(-3.0, 130.0), hst.sampled_from([0.0, -0.5, 118.0, 6.99,
                                                                float("nan"), float("inf")]))


@settings(max_examples=300, deadline=None)
@given(hst.lists(hst.lists(_CHARGE, max_size=7), max_size=5), hst.integers(1, 6))
def test_ptp_marshalling_matches_reference_loops(Z, amax):
    """Same arrays, or the same exception (type and KeyError key) in the same
    order of checks, as the reference's per-molecule loops."""
    from fml_b200.kernels import _ptp_arrays
    got = _outcome(_ptp_arrays, Z, amax)
    ref = _outcome(_reference_ptp_marshalling, Z, amax)
    if isinstance(ref, tuple) and isinstance(ref[0], type):
        assert got == ref, (Z, amax, got, ref)
        return
    np.testing.assert_array_equal(got[0], ref[0])
    np.testing.assert_array_equal(got[1], ref[1])
