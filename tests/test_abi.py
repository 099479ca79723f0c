"""The C-ABI library loads here (no GPU) and exports every entry point that
include/*.h declares; the ctypes binding covers them all."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"NKX_API\s+[\w\s\*]+?\b(nkx_\w+)\s*\(", src))
    return names


def test_header_declarations_found():
    assert {"nkx_plan_create", "nkx_fock_build", "nkx_becke_partition"} <= declared()


def test_library_exports_every_declared_symbol():
    from nukexc_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations():
    from nukexc_b200 import _lib
    assert declared() <= set(_lib.EXPORTS)


def test_error_path_without_gpu():
    # an invalid call returns a status and a message, never throws
    from nukexc_b200 import _lib
    L = _lib.lib()
    st = L.nkx_plan_create(None, None, None, 0, None, None, None, None, None)
    assert st == 1
    assert b"plan pointer" in L.nkx_last_error()
