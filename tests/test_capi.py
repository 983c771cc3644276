"""CPU: the C ABI library loads, exports every declared entry point, and rejects
bad arguments before touching a GPU."""
import ctypes as C
import os
import re

import pytest

from hfem_b200.build import LIB
from hfem_b200.core import Dims, load_library

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "hfem_b200.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(hfem_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("hfem_create", "hfem_assemble", "hfem_gmres", "hfem_newton", "hfem_condense_noalloc"):
        assert n in names


def test_library_exports_all_declared_symbols():
    assert os.path.exists(LIB), "run __graft_entry__.build() first"
    lib = C.CDLL(LIB)
    for n in declared():
        assert hasattr(lib, n), n


def test_create_rejects_bad_dims_without_gpu():
    lib = load_library()
    h = C.c_void_p()
    bad = Dims(4, 3, 2, 3, 3, 2, 10, 15, 75)          # nd = 4
    assert lib.hfem_create(C.byref(bad), 0, C.byref(h)) == -1
    unsupported = Dims(2, 7, 3, 3, 6, 3, 10, 15, 75)  # no kernel for npv = 7
    assert lib.hfem_create(C.byref(unsupported), 0, C.byref(h)) == -2
    assert lib.hfem_create(None, 0, C.byref(h)) == -1
