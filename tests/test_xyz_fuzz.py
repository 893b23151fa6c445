"""Property test of the native XYZ reader (fmlb_xyz_scan / fmlb_xyz_parse)
against the Python reader that restates Molecule.read_xyz (fml/fml.py:109-132):
on random ASCII files — valid and malformed numbers (signs, fractions,
exponents, inf / nan spellings, PEP 515 underscores, stray characters), the
separators Python's str.split() knows, unknown elements, short lines ending the
atom list, and the three newline styles — both give the same molecule or raise
the same exception type. Runs without a GPU."""

import os
import tempfile

import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import fml_b200

SEPARATORS = [" ", "  ", "\t", "\x0b", "\x0c", "\x1c", "\x1f", " \t "]
ELEMENTS = ["H", "C", "N", "O", "S", "Cl", "Xx", "h"]


def _underscored(s, draw):
    """Insert underscores at random places (valid only between two digits)."""
    out = []
    for ch in s:
        out.append(ch)
        if draw(st.integers(0, 9)) == 0:
            out.append("_" * draw(st.integers(1, 2)))
    return "".join(out)


@st.composite
def number_token(draw):
    kind = draw(st.integers(0, 5))
    if kind == 0:  # Python's own spelling of a double
        x = draw(st.floats(allow_nan=True, allow_infinity=True, width=64))
        return repr(x)
    if kind == 1:  # printf forms
        x = draw(st.floats(-1e6, 1e6))
        fmt = draw(st.sampled_from(["%e", "%.3f", "%g", "%.0f", "%+.2E", "%.1f"]))
        return fmt % x
    if kind == 2:  # hand-built decimal forms
        sign = draw(st.sampled_from(["", "+", "-"]))
        ip = draw(st.text("0123456789", max_size=4))
        fp = draw(st.sampled_from(["", "."])) + draw(st.text("0123456789", max_size=3))
        ex = draw(st.sampled_from(["", "e", "E", "e+", "e-", "E-"]))
        ed = draw(st.text("0123456789", max_size=3)) if ex else ""
        return sign + ip + fp + ex + ed or "0"
    if kind == 3:  # inf / nan spellings
        word = draw(st.sampled_from(["inf", "Infinity", "NAN", "nan", "iNf", "infinit",
                                     "nan(1)", "na", "infinity"]))
        return draw(st.sampled_from(["", "+", "-"])) + word
    if kind == 4:  # digit-group underscores, valid or not
        x = draw(st.floats(-1e4, 1e4))
        return _underscored(draw(st.sampled_from(["%.4f", "%e", "%g"])) % x, draw)
    return draw(st.text("0123456789+-._eEinfatyINFATYx()d", min_size=1, max_size=6))


@st.composite
def count_line(draw):
    kind = draw(st.integers(0, 3))
    n = draw(st.integers(0, 40))
    if kind == 0:
        s = str(n)
    elif kind == 1:
        s = draw(st.sampled_from(["+", "-", "", "00"])) + str(n)
    elif kind == 2:
        s = _underscored(str(n * 1001), draw)
    else:
        s = draw(st.text("0123456789+-_. x", min_size=0, max_size=4))
    pad = st.text(" \t\x0b\x0c", max_size=2)
    return draw(pad) + s + draw(pad)


@st.composite
def xyz_file(draw):
    lines = [draw(count_line()), draw(st.text(st.characters(min_codepoint=32, max_codepoint=126),
                                              max_size=12))]
    for _ in range(draw(st.integers(0, 6))):
        ntok = draw(st.sampled_from([4, 4, 4, 4, 5, 3, 0]))
        toks = [draw(st.sampled_from(ELEMENTS))] + [draw(number_token()) for _ in range(4)]
        toks = toks[:ntok]
        seps = [draw(st.sampled_from(SEPARATORS)) for _ in range(len(toks) + 1)]
        lead = seps[0] if draw(st.booleans()) else ""
        lines.append(lead + "".join(t + s for t, s in zip(toks, seps[1:])))
    newline = draw(st.sampled_from(["\n", "\r\n", "\r"]))
    return newline.join(lines) + (newline if draw(st.booleans()) else "")


def _native(path):
    try:
        b = fml_b200.read_xyz_batch([path], nthreads=1)
    except (ValueError, KeyError) as e:
        return type(e)
    return (int(b.natoms_declared[0]), b.atomtypes(0), b.charges.numpy().copy(),
            b.coords.numpy().reshape(-1, 3).copy())


def _python(path):
    m = fml_b200.Molecule()
    try:
        m.read_xyz(path)
    except (ValueError, KeyError) as e:
        return type(e)
    return (m.natoms, m.atomtypes, np.array(m.nuclear_charges, dtype=np.float64),
            np.asarray(m.coordinates, dtype=np.float64).reshape(-1, 3))


@settings(max_examples=400, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(xyz_file())
def test_native_reader_matches_python_reader(text):
    fd, path = tempfile.mkstemp(suffix=".xyz")
    try:
        with os.fdopen(fd, "w", newline="") as f:
            f.write(text)
        a, b = _native(path), _python(path)
    finally:
        os.unlink(path)
    if isinstance(a, type) or isinstance(b, type):
        assert a == b, (text, a, b)
        return
    assert a[0] == b[0] and a[1] == b[1], (text, a, b)
    np.testing.assert_array_equal(a[2], b[2])
    # bit-identical coordinates: same doubles, same NaN and signed-zero signs
    assert a[3].shape == b[3].shape
    np.testing.assert_array_equal(np.isnan(a[3]), np.isnan(b[3]))
    np.testing.assert_array_equal(np.signbit(a[3]), np.signbit(b[3]))
    ok = ~np.isnan(a[3])
    np.testing.assert_array_equal(a[3][ok].view(np.uint64), b[3][ok].view(np.uint64))
