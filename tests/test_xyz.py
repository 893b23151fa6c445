"""Batched XYZ ingestion (fmlb_xyz_scan / fmlb_xyz_parse, host code): the
rules of Molecule.read_xyz (fml/fml.py:109-132), checked against the golden
molecules parsed from the reference's tests/xyz fixtures and against the
Python reader on edge cases. Runs without a GPU."""

import numpy as np
import pytest

import fml_b200
from fml_b200 import synthetic
from fml_b200.data import NUCLEAR_CHARGE


def _write(path, text, newline="\n"):
    with open(path, "w", newline="") as f:
        f.write(text.replace("\n", newline))
    return str(path)


def _xyz_text(symbols, coords, comment="", declared=None):
    lines = [str(len(symbols) if declared is None else declared), comment]
    lines += ["%s %r %r %r" % (s, *map(float, c)) for s, c in zip(symbols, coords)]
    return "\n".join(lines) + "\n"


def _python_read(path):
    m = fml_b200.Molecule()
    m.read_xyz(path)
    return m


def test_golden_molecules_round_trip(golden, tmp_path):
    g = golden
    off, sym = g["xyz_offsets"], g["xyz_symbols"]
    paths = []
    for i in range(len(off) - 1):
        a, b = off[i], off[i + 1]
        paths.append(_write(tmp_path / ("m%d.xyz" % i),
                            _xyz_text(sym[a:b], g["xyz_coords"][a:b], "golden %d" % i)))
    batch = fml_b200.read_xyz_batch(paths)
    np.testing.assert_array_equal(batch.offsets, off)
    np.testing.assert_array_equal(batch.charges.numpy(), g["xyz_charges"])
    np.testing.assert_array_equal(batch.coords.numpy(), g["xyz_coords"])
    np.testing.assert_array_equal(batch.natoms_declared, g["xyz_natoms"])
    assert sum((batch.atomtypes(i) for i in range(len(paths))), []) == list(sym)


def test_many_files_threads_agree(tmp_path):
    b = synthetic.generate(300, nmax=23, seed=5)
    inv = {float(v): k for k, v in NUCLEAR_CHARGE.items()}
    paths = []
    for i in range(b.nmol):
        z, r = b.molecule(i)
        paths.append(_write(tmp_path / ("s%d.xyz" % i), _xyz_text([inv[q] for q in z], r)))
    one = fml_b200.read_xyz_batch(paths, nthreads=1)
    many = fml_b200.read_xyz_batch(paths, nthreads=8)
    np.testing.assert_array_equal(one.offsets, b.offsets)
    np.testing.assert_array_equal(one.charges.numpy(), b.charges)
    np.testing.assert_array_equal(one.coords.numpy(), b.coords)
    for f in ("charges", "coords", "symbol_index"):
        np.testing.assert_array_equal(getattr(one, f).numpy(), getattr(many, f).numpy())


@pytest.mark.parametrize("newline", ["\n", "\r\n", "\r"])
def test_edge_cases_match_python_reader(tmp_path, newline):
    text = ("  5 \n"                          # declared 5, only 3 atom lines follow
            "comment with four tokens here\n"
            "C\t0.0  1.5e-3\t-2\n"
            "H 1.25 -0.5 3.0 extra tokens\n"
            "O   +7 .5 -1E2\n"
            "N 1.0 2.0\n"                     # fewer than 4 tokens: the list ends
            "H 9 9 9\n")
    p = _write(tmp_path / "edge.xyz", text, newline)
    batch = fml_b200.read_xyz_batch([p])
    m = _python_read(p)
    assert batch.natoms_declared[0] == m.natoms == 5
    assert list(batch.offsets) == [0, 3]
    assert batch.atomtypes(0) == m.atomtypes
    np.testing.assert_array_equal(batch.charges.numpy(), np.array(m.nuclear_charges, float))
    np.testing.assert_array_equal(batch.coords.numpy(), m.coordinates)


def test_molecules_match_python_reader(golden, tmp_path):
    g = golden
    off, sym = g["xyz_offsets"], g["xyz_symbols"]
    paths = [_write(tmp_path / ("m%d.xyz" % i),
                    _xyz_text(sym[off[i]:off[i + 1]], g["xyz_coords"][off[i]:off[i + 1]],
                              declared=off[i + 1] - off[i] + (i % 2)))
             for i in range(len(off) - 1)]
    for p, m in zip(paths, fml_b200.read_xyz_molecules(paths)):
        r = _python_read(p)
        assert m.natoms == r.natoms and m.atomtypes == r.atomtypes
        assert m.nuclear_charges == r.nuclear_charges
        np.testing.assert_array_equal(m.coordinates, r.coordinates)


def test_blank_line_ends_atoms_and_empty_molecule(tmp_path):
    p1 = _write(tmp_path / "a.xyz", "2\n\nH 0 0 0\n\nH 0 0 1\n")
    p2 = _write(tmp_path / "b.xyz", "0\ncomment\n")
    batch = fml_b200.read_xyz_batch([p1, p2])
    assert list(batch.offsets) == [0, 1, 1]
    assert _python_read(p1).coordinates.shape == (1, 3)


def test_errors(tmp_path):
    bad_el = _write(tmp_path / "el.xyz", "1\n\nXx 0 0 0\n")
    with pytest.raises(KeyError):
        fml_b200.read_xyz_batch([bad_el])
    with pytest.raises(KeyError):
        _python_read(bad_el)
    bad_num = _write(tmp_path / "num.xyz", "1\n\nH 0 abc 0\n")
    with pytest.raises(ValueError):
        fml_b200.read_xyz_batch([bad_num])
    bad_count = _write(tmp_path / "count.xyz", "two\n\nH 0 0 0\n")
    with pytest.raises(ValueError):
        fml_b200.read_xyz_batch([bad_count])
    empty = _write(tmp_path / "empty.xyz", "")
    with pytest.raises(ValueError):
        fml_b200.read_xyz_batch([empty])
    with pytest.raises(ValueError):
        fml_b200.read_xyz_batch([str(tmp_path / "missing.xyz")])
    assert fml_b200.read_xyz_batch([]).offsets.tolist() == [0]


@pytest.mark.gpu
def test_batch_to_device_feeds_descriptors(golden, tmp_path):
    g = golden
    off, sym = g["xyz_offsets"], g["xyz_symbols"]
    paths = [_write(tmp_path / ("m%d.xyz" % i),
                    _xyz_text(sym[off[i]:off[i + 1]], g["xyz_coords"][off[i]:off[i + 1]]))
             for i in range(len(off) - 1)]
    batch = fml_b200.read_xyz_batch(paths, to_device=True)
    assert batch.charges.is_pinned() and batch.device_coords.is_cuda
    cm = fml_b200.generate_coulomb_matrices(batch.device_charges, batch.device_coords,
                                            batch.device_offsets, size=23)
    np.testing.assert_allclose(cm.cpu().numpy(), g["cm_xyz_s23"], rtol=1e-14, atol=1e-13)
