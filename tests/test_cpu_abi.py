"""CPU-only checks of the C ABI: the library loads without a GPU and exports
every function include/cpsb200.h declares; entry points report a missing
device as a status code instead of crashing."""
import ctypes as C
import os
import re

import pytest

from cps_public_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cpsb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cpsb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cpsb_invcg" in names and "cpsb_dslash" in names and "cpsb_minvcg" in names
    assert set(names) == set(_lib.SYMBOLS), set(names) ^ set(_lib.SYMBOLS)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIBPATH):
        from cps_public_b200 import build
        build.build()
    lib = C.CDLL(_lib.LIBPATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_error_strings_and_no_device_status():
    lib = _lib.load()
    assert lib.cpsb_error_string(0) == b"ok"
    assert lib.cpsb_error_string(-4) == b"unsupported configuration"
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the no-device path is not reachable")
    assert lib.cpsb_init(0) == -6   # CPSB_ERR_NO_DEVICE, no abort
    h = C.c_void_p()
    assert lib.cpsb_serve_create(C.byref(h), 2, 0.5, 0) == -6
    assert not h.value
