"""The C ABI: liblcb.so loads on a machine without a GPU and exports every
function include/lcb.h declares, and the ctypes binding declares each one."""
import ctypes
import os
import re

from lcodepy_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(lcb_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_symbols_exported():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 10
    for n in sorted(names):
        assert hasattr(L, n), f"{n} declared in include/ but not exported"


def test_binding_covers_header():
    assert declared() == set(_lib.declared_symbols())


def test_library_loads_without_gpu():
    L = _lib.load()
    assert L.lcb_version() >= 100
    assert L.lcb_compute_fields_workspace_bytes(129, 0) > 0
    assert L.lcb_plasma_deposit_workspace_bytes(129, 1) == 8 * 129 * 129 * 8  # int64 sums
