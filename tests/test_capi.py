"""C ABI surface (no GPU needed): the in-tree library loads and exports every
entry point that include/zm_b200.h declares, with matching struct layouts."""
import ctypes
import os
import re

from zhenmode_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "zm_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(zm_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    names = _declared()
    assert "zm_create" in names and "zm_step" in names
    for name in names:
        assert hasattr(lib, name), f"{name} declared but not exported"


def test_binding_covers_header():
    assert set(_declared()) <= set(_native.EXPORTS)


def test_struct_layouts():
    # six 8-byte pointers after three int32 + a double, all naturally aligned
    assert ctypes.sizeof(_native.ZmGrid) == 4 * 3 + 4 + 8 + 7 * 8
    assert ctypes.sizeof(_native.ZmState) == 5 * 8
    p = _native.ZmParams
    assert p.tau_x.offset % 8 == 0
    assert ctypes.sizeof(p) == 16 * 8 + 10 * 4 + 10 * 8 + 4 * 4 + 8 + 4 * 8 + 8
    assert p.projection_rtol.offset % 8 == 0
