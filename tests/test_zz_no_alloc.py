"""nkx_xc_dense_noalloc -- the dense XC build for callers that cannot
allocate device memory (graph capture, fixed memory budgets) -- against
nkx_xc_dense on the same device inputs, through the C ABI, twice in a row
(the fixed scratch array keeps the previous call's contents, so the second
call checks that everything that must start at zero is cleared).

This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import _lib as L  # noqa: E402
from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402


def _inputs():
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    phi, gx, gy, gz = A.fill_grad_collocation(b, g.quad_points)
    nbf, npts = phi.shape
    Cm = M.random_orbitals(nbf, 5, seed=11)
    flat = [A._flat_lmat(x) for x in (phi, gx, gy, gz)]
    w = A._dev(g.weights)
    Cd = A._flat_lmat(Cm)
    occ = A._dev(np.ones(5))
    return nbf, npts, flat, w, Cd, occ


def _call(fn, nbf, npts, flat, w, Cd, occ, opts):
    V = torch.full((nbf * nbf,), float("nan"), dtype=torch.float64, device="cuda")
    E = C.c_double(0)
    st = fn(nbf, npts, *[A._p(x) for x in flat], A._p(w), 1, 5, A._p(Cd), A._p(occ), C.byref(opts),
            C.byref(E), A._p(V), None)
    L.check(st)
    return E.value, V.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    lib = L.lib()
    nbf, npts, flat, w, Cd, occ = _inputs()
    assert 32 + 4 * npts + nbf * npts < (4 << 20)
    opts = A._opts(("GGA_X_PBE", "GGA_C_PBE"))
    E0, V0 = _call(lib.nkx_xc_dense, nbf, npts, flat, w, Cd, occ, opts)
    for _ in range(2):
        E1, V1 = _call(lib.nkx_xc_dense_noalloc, nbf, npts, flat, w, Cd, occ, opts)
        assert abs(E1 - E0) <= 1e-12 * abs(E0)
        assert np.abs(V1 - V0).max() <= 1e-12 * np.abs(V0).max()


def test_noalloc_rejects_oversize_problem():
    lib = L.lib()
    nbf, npts = 2000, 4096  # nbf * npts > 4 Mi doubles: rejected before any launch
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    opts = A._opts(("LDA_X",))
    E = C.c_double(0)
    st = lib.nkx_xc_dense_noalloc(nbf, npts, A._p(dummy), None, None, None, A._p(dummy), 1, 1, A._p(dummy),
                                  A._p(dummy), C.byref(opts), C.byref(E), A._p(dummy), None)
    assert st == L.NKX_OK + 1
    assert b"32 MiB" in lib.nkx_last_error()
