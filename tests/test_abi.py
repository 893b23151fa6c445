"""The C-ABI library builds, loads without a GPU and exports every symbol
that include/fmlb.h declares (no compute calls here)."""

import ctypes
import os
import re

import pytest

from fml_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(fmlb_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_header_declares_functions():
    assert {"fmlb_last_error_string", "fmlb_coulomb_matrices", "fmlb_potrf_f64"} <= _declared()


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert _declared() == set(_lib.SIGNATURES)


def test_host_only_calls(lib):
    lib.fmlb_version.restype = ctypes.c_int
    assert lib.fmlb_version() >= 1
    lib.fmlb_last_error_string.restype = ctypes.c_char_p
    assert isinstance(lib.fmlb_last_error_string(), bytes)
    lib.fmlb_potrf_workspace_bytes.restype = ctypes.c_size_t
    assert lib.fmlb_potrf_workspace_bytes(1000) >= 1000 * 8
    lib.fmlb_arad_workspace_bytes.restype = ctypes.c_size_t
    assert lib.fmlb_arad_workspace_bytes(10, 12, 23, 0) > lib.fmlb_arad_workspace_bytes(10, 12, 23, 1)


def test_argument_errors_need_no_gpu(lib):
    """Argument validation runs on the host before any CUDA call."""
    lib.fmlb_gaussian_kernel_f64.restype = ctypes.c_int
    one = (ctypes.c_double * 1)(1.0)
    rc = lib.fmlb_gaussian_kernel_f64(None, 10, 5, None, 10, 5, 8, one, 1, None,
                                      ctypes.c_longlong(10), ctypes.c_longlong(100), 0, None)
    assert rc == -22  # lda < d
    lib.fmlb_last_error_string.restype = ctypes.c_char_p
    assert b"leading dimension" in lib.fmlb_last_error_string()


def _rc_and_message(lib, fn, *args):
    f = getattr(lib, fn)
    f.restype = ctypes.c_int
    rc = f(*args)
    lib.fmlb_last_error_string.restype = ctypes.c_char_p
    return rc, lib.fmlb_last_error_string()


def test_tensor_core_and_refinement_argument_errors_need_no_gpu(lib):
    """The int8 factorisation, the int8 trailing update and the double-double
    refinement reject bad sizes on the host, before any CUDA call."""
    info = ctypes.c_int(0)
    ll = ctypes.c_longlong
    # n < 0
    rc, msg = _rc_and_message(lib, "fmlb_potrf_ozaki_f64", None, ll(4), -1, 6, None,
                              ctypes.c_size_t(0), ctypes.byref(info), None)
    assert rc == -22 and b"fmlb_potrf_ozaki_f64: bad n" in msg
    # digit planes outside 1..max
    for s in (0, 99):
        rc, msg = _rc_and_message(lib, "fmlb_potrf_ozaki_f64", None, ll(4), 4, s, None,
                                  ctypes.c_size_t(0), ctypes.byref(info), None)
        assert rc == -22 and b"nslices" in msg
    # int8 update: k above the int32-exact bound of 8192
    rc, msg = _rc_and_message(lib, "fmlb_syrk_lower_ozaki", None, ll(16), 16, None,
                              ll(16384), 16384, 0, 6, None, ctypes.c_size_t(0),
                              ctypes.byref(info), None)
    assert rc == -22 and b"8192" in msg
    # double-double refinement: negative iteration count
    rc, msg = _rc_and_message(lib, "fmlb_krr_refine_dd", None, ll(4), 4, None, None, None,
                              None, None, -1, None, None, None)
    assert rc == -22 and b"fmlb_krr_refine_dd: bad sizes" in msg


def test_noalloc_prediction_limits_need_no_gpu(lib):
    """The allocation-free prediction checks its kind and its fixed scratch
    limit, ceil(nt/1024) * nsigma * nq <= 2^20 doubles, before it touches a
    device."""
    sig = (ctypes.c_double * 8)(*([100.0] * 8))
    ll = ctypes.c_longlong
    rc, msg = _rc_and_message(lib, "fmlb_kernel_predict_f64_noalloc", 2, None, 1, 4, None, 1,
                              4, 4, sig, 1, None, ll(1), None, ll(1), None)
    assert rc == -22 and b"kind" in msg
    nq = (1 << 20) // 8 + 1  # 8 sigmas, one 1024-row split: one row above the limit
    rc, msg = _rc_and_message(lib, "fmlb_kernel_predict_f64_noalloc", 0, None, nq, 4, None,
                              1024, 4, 4, sig, 8, None, ll(1024), None, ll(nq), None)
    assert rc == -22 and b"exceeds the fixed scratch" in msg


def test_integration_stubs_match_the_abi():
    """The ctypes stubs shown to maintainers declare the argument and result
    types the library's own binding table (checked against the header above)
    uses for the same functions."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```python\n(.*?)```", text, flags=re.S)
    ns = {"ctypes": ctypes, "_vp": ctypes.c_void_p, "_i": ctypes.c_int,
          "_ll": ctypes.c_longlong}
    seen = set()
    for block in blocks:
        for name, kind, expr in re.findall(r"_lib\.(fmlb_\w+)\.(argtypes|restype)\s*=\s*"
                                           r"(\[.*?\]|[\w.]+)", block, flags=re.S):
            value = eval(expr, ns)  # the stub's own expression
            restype, argtypes = _lib.SIGNATURES[name]
            if kind == "argtypes":
                assert value == argtypes, name
                seen.add(name)
            else:
                assert value == restype, name
    assert {"fmlb_gaussian_kernel_f64", "fmlb_potrf_f64", "fmlb_potrs_f64",
            "fmlb_potri_f64"} <= seen
