"""The C ABI library loads and exports every function include/*.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("libfive.h", "libfive_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b((?:libfive|lfb)_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_all_declared_symbols_exported(lib):
    names = declared_functions()
    assert len(names) > 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_signatures_cover_headers():
    from libfive_b200 import ffi
    bound = {n for n, _, _ in ffi.SIGNATURES}
    assert declared_functions() <= bound


def test_struct_layouts():
    from libfive_b200 import ffi
    assert ctypes.sizeof(ffi.Vec3) == 12
    assert ctypes.sizeof(ffi.Tri) == 12
    assert ctypes.sizeof(ffi.Region3) == 24
    assert ctypes.sizeof(ffi.Mesh) == 24
