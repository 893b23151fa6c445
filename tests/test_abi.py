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
