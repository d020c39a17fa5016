"""The C-ABI library loads and exports every symbol include/mgc_b200.h declares."""

import ctypes
import os
import re

from mirgecom_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "mgc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mgc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "mgc_euler_rhs" in names and "mgc_ns_rhs" in names


def test_library_exports_all_declared_symbols():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_version_and_supports_without_gpu():
    lib = _lib.load()
    assert lib.mgc_version() >= 1
    assert lib.mgc_supports(3, 3, 0, 0) == 1
    assert lib.mgc_supports(3, 3, 7, 1) == 1
    assert lib.mgc_supports(3, 5, 0, 0) == 0
    assert lib.mgc_supports(2, 4, 2, 0) == 1


def test_invalid_arguments_rejected_without_gpu():
    lib = _lib.load()
    assert lib.mgc_euler_rhs(None, None, None, None, None, 0, None, None, None) == -1
    assert lib.mgc_rk4_stage(-1, None, None, None, None, None, 0, 0.1, None) == -1
