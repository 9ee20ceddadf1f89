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


@pytest.mark.parametrize("cname,pyname", [("cpsb_dirac_params", "DiracParams"), ("cpsb_cg_arg", "CgArg"),
                                          ("cpsb_solve_result", "SolveResult"),
                                          ("cpsb_serve_stats_t", "ServeStats")])
def test_struct_layout_matches_header(cname, pyname, tmp_path):
    """The ctypes mirrors in _lib.py have the size and field offsets of the C
    structs as a C compiler lays them out from include/cpsb200.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    py = getattr(_lib, pyname)
    fields = [f for f, _ in py._fields_]
    lines = [f'printf("%zu\\n", sizeof({cname}));'] + [f'printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "cpsb200.h"\nint main(void) {\n'
                   + "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == C.sizeof(py), (cname, got[0], C.sizeof(py))
    assert got[1:] == [getattr(py, f).offset for f in fields], (cname, got[1:])
