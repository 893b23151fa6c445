"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run where the reference tree is available, naming its root in
``FML_REFERENCE``::

    FML_REFERENCE=<path to the andersx/fml checkout> python tests/golden/make_golden.py

The reference is Python 2 + f2py Fortran, and no Fortran compiler is
available, so only its Python-3-runnable parts are executed here:

* ``fml/arad.py`` (ARAD.describe) and ``fml/data.py`` (NUCLEAR_CHARGE) import
  unmodified;
* ``fml/representations/representations.py``: the pure-Python sorted Coulomb
  matrix ``generate_coulomb_matrix`` and ``triangular_to_vector`` (their
  module fails to parse under Python 3 only because of a Python-2 ``print``
  statement, which is rewritten as a call before the two functions are run),
  and the per-atom ``generate_local_coulomb_matrix`` /
  ``generate_atomic_coulomb_matrix`` (the latter's Python-2 debug line
  ``print distances`` is dropped: it only prints);
* ``tests/test_arad.py``: the reference test's own ARAD distance / kernel
  restatement (``calcNorm``, ``calcProd``, ``_MDist``, ``_dist``,
  ``_StochDist``, the ``PTP`` table), evaluated serially the way
  ``condense(..., molecular=False)`` and tests/test_arad.py:377-387 use them.

The XYZ fixtures tests/xyz/*.xyz are parsed with the same rules as
``Molecule.read_xyz`` (fml/fml.py:109-132) and stored as arrays, so nothing
at test time reads the reference tree.
"""

import importlib.util
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fml_b200.synthetic import generate  # noqa: E402

REF = os.environ.get("FML_REFERENCE")
if not REF:
    sys.exit("make_golden.py: set FML_REFERENCE to the root of the andersx/fml checkout")


def _load_module(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _extract(path, names):
    """Return the source text of top-level defs / assignments ``names``."""
    text = open(path).read()
    lines = text.split("\n")
    out = []
    for name in names:
        pat = re.compile(r"^(def %s\(|%s\s*=)" % (re.escape(name), re.escape(name)))
        start = next(i for i, l in enumerate(lines) if pat.match(l))
        end = start + 1
        while end < len(lines) and not re.match(r"^(def |class |if __name__|[A-Za-z_]\w*\s*=)",
                                                 lines[end]):
            end += 1
        out.append("\n".join(lines[start:end]))
    src = "\n\n".join(out)
    # Python-2 print statements -> calls (only inside error branches)
    src = re.sub(r'print ("[^"\n]*")', r"print(\1)", src)
    return src


def read_xyz(path, charge_table):
    """fml/fml.py:109-132 reading rules."""
    lines = open(path).read().split("\n")
    natoms = int(lines[0])
    symbols, coords = [], []
    for line in lines[2:]:
        tok = line.split()
        if len(tok) < 4:
            break
        symbols.append(tok[0])
        coords.append([float(tok[1]), float(tok[2]), float(tok[3])])
    return natoms, symbols, np.array(coords)


def tie_molecules():
    """Molecules whose atoms have exactly equidistant neighbours of different
    elements: a centre atom plus the 24 signed permutations of (a, b, c) with
    an even number of minus signs. The squares of a, b, c and their sums are
    exact in binary, so the 24 centre distances are bit-equal; no vertex has
    its antipode in the set, so no three atoms are collinear (collinear atoms
    send arad.py's arccos slightly past +-1, to NaN)."""
    from itertools import permutations
    cyc = np.array([1.0, 6.0, 7.0, 8.0, 16.0])
    mols = []
    for abc, zc in (((0.75, 1.25, 1.5), 6.0), ((0.5, 1.25, 2.0), 7.0)):
        pts = [(0.0, 0.0, 0.0)]
        for perm in permutations(abc):
            for signs in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1)):
                pts.append(tuple(s * v for s, v in zip(signs, perm)))
        r = np.array(pts)
        z = np.concatenate([[zc], cyc[np.arange(len(r) - 1) % 5]])
        mols.append((z, r))
    return mols


def main():
    arad_mod = _load_module("ref_arad", os.path.join(REF, "fml/arad.py"))
    data_mod = _load_module("ref_data", os.path.join(REF, "fml/data.py"))
    charge_table = data_mod.NUCLEAR_CHARGE

    # ---- tables -----------------------------------------------------------
    ptp = arad_mod.ARAD().PTP
    with open(os.path.join(HERE, "reference_tables.json"), "w") as f:
        json.dump({"PTP": {str(k): v for k, v in sorted(ptp.items())},
                   "NUCLEAR_CHARGE": charge_table}, f, indent=0, sort_keys=True)

    # ---- XYZ fixtures ------------------------------------------------------
    xyz_dir = os.path.join(REF, "tests/xyz")
    names = sorted(os.listdir(xyz_dir))
    mols = [read_xyz(os.path.join(xyz_dir, n), charge_table) for n in names]
    charges = [np.array([charge_table[s] for s in m[1]], dtype=np.float64) for m in mols]
    coords = [m[2] for m in mols]
    offsets = np.zeros(len(mols) + 1, dtype=np.int32)
    np.cumsum([len(c) for c in charges], out=offsets[1:])
    xyz = dict(names=np.array(names), natoms=np.array([m[0] for m in mols]),
               symbols=np.array(sum([m[1] for m in mols], [])),
               charges=np.concatenate(charges), coords=np.concatenate(coords), offsets=offsets)

    # ---- ARAD descriptors from the reference's ARAD.describe --------------
    arad = {}
    for size, cut in ((30, 5.0), (20, 5.0), (23, 1e6), (23, 5.0)):
        a = arad_mod.ARAD(maxMolSize=size, maxAts=size, cut=cut)
        arad["xyz_s%d_c%g" % (size, cut)] = np.stack(
            [a.describe(c, z) for c, z in zip(coords, charges)])
    syn = generate(48, nmax=23, seed=11)
    for cut in (5.0, 1e6):
        a = arad_mod.ARAD(maxMolSize=23, maxAts=23, cut=cut)
        arad["syn_s23_c%g" % cut] = np.stack(
            [a.describe(syn.molecule(i)[1], syn.molecule(i)[0]) for i in range(syn.nmol)])

    # ---- exact ties: equidistant neighbours of different elements ---------
    # arad.py:110 sorts neighbour distances with numpy's default argsort, which
    # is not stable above 16 elements; these molecules have many exact ties.
    ties = tie_molecules()
    for size, cut in ((30, 5.0), (30, 1e6)):
        a = arad_mod.ARAD(maxMolSize=size, maxAts=size, cut=cut)
        arad["ties_s%d_c%g" % (size, cut)] = np.stack([a.describe(r, z) for z, r in ties])
    tie_off = np.zeros(len(ties) + 1, dtype=np.int32)
    np.cumsum([len(z) for z, _ in ties], out=tie_off[1:])

    # ---- sorted Coulomb matrices from representations.py ------------------
    rep_path = os.path.join(REF, "fml/representations/representations.py")
    ns = {"np": np}
    exec(_extract(rep_path, ["NUCLEAR_CHARGE", "triangular_to_vector",
                             "generate_coulomb_matrix"]), ns)
    # representations.py's table holds H C N O F Si P S Ge: fill the rest from data.py
    for s, z in charge_table.items():
        ns["NUCLEAR_CHARGE"].setdefault(s, float(z))
    cm = {}
    cm["xyz_s23"] = np.stack([ns["generate_coulomb_matrix"](m[1], m[2], size=23) for m in mols])
    cm["xyz_s30"] = np.stack([ns["generate_coulomb_matrix"](m[1], m[2], size=30) for m in mols])
    inv = {1.0: "H", 6.0: "C", 7.0: "N", 8.0: "O", 16.0: "S"}
    syn_cm = generate(64, nmax=23, seed=12)
    cm["syn_s23"] = np.stack([
        ns["generate_coulomb_matrix"]([inv[z] for z in syn_cm.molecule(i)[0]],
                                      syn_cm.molecule(i)[1], size=23)
        for i in range(syn_cm.nmol)])

    # ---- per-atom (local / atomic) Coulomb matrices from representations.py
    src = _extract(rep_path, ["generate_local_coulomb_matrix", "generate_atomic_coulomb_matrix"])
    assert src.count("print distances") == 1
    exec(src.replace("print distances", "pass"), ns)
    lcm = {}
    for kind in ("local", "atomic"):
        fn = ns["generate_%s_coulomb_matrix" % kind]
        lcm[kind + "_xyz_s23"] = np.concatenate(
            [np.array(fn(m[1], m[2], size=23)) for m in mols])
        lcm[kind + "_syn_s23"] = np.concatenate([
            np.array(fn([inv[z] for z in syn_cm.molecule(i)[0]], syn_cm.molecule(i)[1],
                        size=23)) for i in range(syn_cm.nmol)])

    # ---- ARAD kernels from tests/test_arad.py's restatement ----------------
    ta_path = os.path.join(REF, "tests/test_arad.py")
    tns = {"np": np}
    exec(_extract(ta_path, ["PTP", "calcNorm", "calcProd", "_MDist", "_dist",
                            "_StochDist"]), tns)

    def create_zinp(Z, l):  # tests/test_arad.py:46-51
        z_inp = -1 * np.ones((len(Z), l, 2)).astype(int)
        for i in range(len(Z)):
            z_inp[i, :len(Z[i])] = np.asarray([tns["PTP"][int(z)] for z in Z[i]])
        return z_inp

    def test_arad_distance(x1, x2, z1, z2, width=0.2, cut=6.0, rw=1.0, cw=0.5):
        """condense(..., molecular=False) evaluated serially (test_arad.py:45-150)."""
        Z1, Z2 = create_zinp(z1, len(x1[0])), create_zinp(z2, len(x2[0]))
        D1 = np.asarray([tns["calcNorm"](x, z, width, cut, rw, cw) for x, z in zip(x1, Z1)])
        D2 = np.asarray([tns["calcNorm"](x, z, width, cut, rw, cw) for x, z in zip(x2, Z2)])
        rows = [tns["calcProd"](x1[i], np.asarray(x2), Z1[i], Z2, D1[i], D2, width, cut, rw,
                                cw, np.nan) for i in range(len(x1))]
        return np.asarray(rows)  # (nm1, nm2, amax, amax)

    def kernel_from_distance(Da, sigmas):  # tests/test_arad.py:379-387
        Ka = np.zeros((len(sigmas), Da.shape[0], Da.shape[1]))
        for s, sigma in enumerate(sigmas):
            for i in range(Da.shape[0]):
                for j in range(Da.shape[1]):
                    Ka[s, i, j] = np.nansum(np.exp(Da[i, j] * (-1.0 / sigma ** 2)))
        return Ka

    sigmas = [0.1, 1.0, 10.0, 100.0]  # tests/test_arad.py:377
    x30 = arad["xyz_s30_c5"]
    z_lists = [list(c) for c in charges]
    Da = test_arad_distance(list(x30[:5]), list(x30[5:]), z_lists[:5], z_lists[5:])
    Ka = kernel_from_distance(Da, sigmas)
    Ds = test_arad_distance(list(x30), list(x30), z_lists, z_lists)
    Ks = kernel_from_distance(Ds, sigmas)

    # same restatement on synthetic molecules with the descriptor cut of 1e6
    xs = arad["syn_s23_c1e+06"][:12]
    zs = [list(syn.molecule(i)[0]) for i in range(12)]
    Dsyn = test_arad_distance(list(xs[:6]), list(xs[6:]), zs[:6], zs[6:])
    sig_syn = [0.1, 0.5, 1.0, 2.0, 5.0]
    Ksyn = kernel_from_distance(Dsyn, sig_syn)

    np.savez_compressed(
        os.path.join(HERE, "reference_golden.npz"),
        **{"xyz_" + k: v for k, v in xyz.items()},
        **{"arad_" + k: v for k, v in arad.items()},
        **{"cm_" + k: v for k, v in cm.items()},
        **{"lcm_" + k: v for k, v in lcm.items()},
        ties_charges=np.concatenate([z for z, _ in ties]),
        ties_coords=np.concatenate([r for _, r in ties]), ties_offsets=tie_off,
        syn11_charges=syn.charges, syn11_coords=syn.coords, syn11_offsets=syn.offsets,
        syn12_charges=syn_cm.charges, syn12_coords=syn_cm.coords,
        syn12_offsets=syn_cm.offsets,
        testarad_sigmas=np.array(sigmas), testarad_K_5v5=Ka, testarad_D_5v5=Da,
        testarad_K_10v10=Ks, testarad_syn_sigmas=np.array(sig_syn),
        testarad_syn_K_6v6=Ksyn)
    print("wrote", os.path.join(HERE, "reference_golden.npz"))


if __name__ == "__main__":
    main()
