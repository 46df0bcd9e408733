"""The C-ABI library loads and exports every entry point include/hc.h declares."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "hc.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from deepcharacters_b200 import _lib
    L = _lib.lib()
    names = declared()
    assert "hc_renderer_forward" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"symbols declared in hc.h but not exported: {missing}"


def test_binding_covers_header():
    from deepcharacters_b200 import _lib
    assert set(declared()) <= set(_lib.declared_symbols())


def test_version_and_error_string():
    from deepcharacters_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.hc_version()
    assert isinstance(L.hc_last_error(), bytes)


def test_create_rejects_bad_attributes_without_gpu():
    """Attribute validation happens before any device work."""
    from deepcharacters_b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    faces = (ctypes.c_int32 * 3)(0, 1, 2)
    st = L.hc_renderer_create(ctypes.byref(h), faces, 1, None, 0, 3, 1, 64, 64, b"bogus", b"shaded", 1, 1, b"none")
    assert st == 1
    assert b"ALBEDO" in L.hc_last_error()
    st = L.hc_renderer_create(ctypes.byref(h), faces, 1, None, 0, 3, 1, 64, 64, b"vertexColor", b"flat", 1, 1,
                              b"none")
    assert st == 1
    faces_bad = (ctypes.c_int32 * 3)(0, 1, 7)
    st = L.hc_renderer_create(ctypes.byref(h), faces_bad, 1, None, 0, 3, 1, 64, 64, b"vertexColor", b"shaded", 1,
                              1, b"none")
    assert st == 1 and b"outside" in L.hc_last_error()
