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


def test_morton_order_host_entry():
    # nkx_morton_order runs on the host: a permutation along which the
    # interleaved 21-bit codes over the points' bounding box never decrease
    import numpy as np
    from nukexc_b200 import _lib
    rng = np.random.default_rng(5)
    pts = rng.normal(size=(5000, 3)) * np.array([3.0, 1.0, 0.5])
    perm = np.zeros(len(pts), np.int64)
    _lib.check(_lib.lib().nkx_morton_order(len(pts), pts.ctypes.data_as(ctypes.c_void_p),
                                           perm.ctypes.data_as(ctypes.c_void_p)))
    assert np.array_equal(np.sort(perm), np.arange(len(pts)))
    lo, hi = pts.min(0), pts.max(0)
    q = np.minimum(2097151.0, np.maximum(0.0, (pts - lo) / (hi - lo) * 2097151.0)).astype(np.uint64)
    code = np.zeros(len(pts), np.uint64)
    for bit in range(21):
        for d in range(3):
            code |= ((q[:, d] >> np.uint64(bit)) & np.uint64(1)) << np.uint64(3 * bit + d)
    assert np.all(np.diff(code[perm].astype(np.float64)) >= 0)


def test_api_cutoff_radii_match_oracle():
    # the Python mirror's cutoff radii (host bisection, used for the
    # neighbour lists) equal the oracle's restatement of compute_cutoff
    import sys
    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from nukexc_b200 import api as A
    funcs = [(n, l, 0, z, 0.0, 0.0, 0.0) for n, l in [(1, 0), (2, 1), (3, 2), (4, 3)] for z in (0.3, 1.0, 7.5)]
    for tol in (1e-10, 1e-6):
        ours = A.cutoff_radii(A.make_manual_basis(funcs, cutoff_tol=tol))
        ref = O.make_manual_basis(funcs, cutoff_tol=tol)["cutoff"]
        assert np.allclose(ours, ref, rtol=1e-9, atol=0.0)  # both solve ln N + (n-1) ln r - zeta r = ln tol
