"""The C-ABI library loads and exports every entry point include/ins2d.h
declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "ins2d.h")) as fh:
        txt = fh.read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|const char \*|ins2d_ctx \*)\s*(ins2d_\w+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "ins2d_erk_step" in names and "ins2d_pressure_poisson" in names and "ins2d_F" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from ins2d_b200 import _lib
    lib = _lib.load()
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == _declared()


def test_library_links_no_torch():
    from ins2d_b200 import _lib
    with open(_lib.LIB_PATH, "rb") as fh:
        blob = fh.read()
    assert b"libtorch" not in blob and b"libc10" not in blob
