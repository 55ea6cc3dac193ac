"""The C-ABI library loads without a GPU and exports what include/bdb200.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bdb200.h")
LIB = os.path.join(ROOT, "bd_box_b200", "libbdb200.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bdb_[A-Za-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from bd_box_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_header_declares_entry_points():
    names = declared()
    for must in ("bdb_create", "bdb_step", "bdb_compute_forces", "bdb_compute_D", "bdb_compute_r",
                 "bdb_compute_Rf", "bdb_destroy"):
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_matches_header():
    from bd_box_b200 import engine
    assert sorted(engine.EXPORTS) == sorted(n for n in declared() if n in engine.EXPORTS)
    assert set(engine.EXPORTS) <= set(declared())


def test_version_and_error_without_gpu(lib):
    lib.bdb_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.bdb_version()
    lib.bdb_create.argtypes = [ctypes.c_void_p] * 5
    # null arguments are rejected on the host, before any device call
    assert lib.bdb_create(None, None, None, None, None) == -1
    lib.bdb_last_error.restype = ctypes.c_char_p
    assert b"null" in lib.bdb_last_error()


def test_params_struct_layout():
    """bdb_params as seen by ctypes matches the C struct (offsetof via gcc)."""
    import subprocess
    import tempfile
    from bd_box_b200 import engine
    fields = [f[0] for f in engine.Params._fields_]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"bdb200.h\"\nint main(){\n"
    src += 'printf("%zu\\n", sizeof(bdb_params));\n'
    for f in fields:
        src += f'printf("%zu\\n", offsetof(bdb_params, {f}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(engine.Params)
    for f, off in zip(fields, out[1:]):
        assert getattr(engine.Params, f).offset == off, f
