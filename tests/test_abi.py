"""The C ABI: the library loads and exports every symbol the header declares."""
import ctypes
import os

import thirring
from thirring import _lib


def test_header_declares_functions():
    names = _lib.header_functions()
    assert "thr_dslash" in names and "thr_create" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _lib.header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    missing = [n for n in _lib.header_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_status_strings():
    lib = thirring.lib()
    assert lib.thr_status_string(0) == b"ok"
    assert lib.thr_status_string(2) == b"bad shape"


def test_library_is_sm100a_only():
    # the shared library carries only Blackwell code (compute_100a / sm_100a)
    assert os.path.getsize(_lib.LIB_PATH) > 0
