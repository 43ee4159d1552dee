"""The C-ABI library loads and exports every symbol include/imaged11_b200.h declares.

No compute calls here (no GPU needed)."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "imaged11_b200.h")
LIB = os.path.join(REPO, "imaged11_b200", "libimaged11_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(id11b_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from imaged11_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    from imaged11_b200 import _lib
    assert set(declared_symbols()) <= set(_lib.exported_symbols())


def test_status_strings(lib):
    lib.id11b_status_string.restype = ctypes.c_char_p
    assert lib.id11b_status_string(0) == b"ok"
    assert b"CUDA" in lib.id11b_status_string(2)
    assert lib.id11b_version() >= 100


def test_argument_errors_without_gpu(lib):
    """Argument checks run on the host before any CUDA call."""
    f = lib.id11b_dev_score_many_fp64
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    # ntol beyond the maximum
    tols = (ctypes.c_double * 8)()
    assert f(None, 1, None, 1, tols, 9, None, None) == 1
    g = lib.id11b_dev_compute_gv
    g.restype = ctypes.c_int
    g.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_double] * 4 + [ctypes.c_void_p] * 3 + \
        [ctypes.c_int64, ctypes.c_void_p]
    t = (ctypes.c_double * 3)()
    assert g(None, None, 1., 1., 0., 0., t, None, None, -1, None) == 1
    assert g(None, None, 1., 1., 0., 0., t, None, None, 0, None) == 0
