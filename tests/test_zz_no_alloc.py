"""nkx_xc_dense_noalloc, the dense XC build for callers that must not
allocate device memory (a host program whose own pool allocator owns the
GPU's memory, or a loop that cannot take the device-wide synchronisation of
cudaMalloc / cudaFree), checked through the C ABI against the allocating
nkx_xc_dense on the same device inputs.

Each case calls the no-alloc entry point twice in a row: its fixed scratch
array keeps the previous call's contents, so the second call shows that
everything that must start at zero is cleared by the call itself.  The
closed-shell and open-shell cases cover both layouts of the shared array.

This file is named so that pytest collects it last."""
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

NOCC = 5
SCRATCH_DOUBLES = 4 << 20  # NKX_NOALLOC_SCRATCH_DOUBLES
TOL = 1e-12  # relative; both entry points run the same FP64 kernels


def _inputs(nspin):
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    phi, gx, gy, gz = A.fill_grad_collocation(b, g.quad_points)
    nbf, npts = phi.shape
    # open shell: alpha and beta blocks from different seeds, different occupations
    Cm = np.concatenate([M.random_orbitals(nbf, NOCC, seed=11 + s) for s in range(nspin)], axis=1)
    occ = np.concatenate([np.ones(NOCC) if s == 0 else np.linspace(1.0, 0.2, NOCC) for s in range(nspin)])
    flat = [A._flat_lmat(x) for x in (phi, gx, gy, gz)]
    w = A._dev(g.weights)
    Cd = A._flat_lmat(Cm)
    occd = A._dev(occ)
    return nbf, npts, flat, w, Cd, occd


def _call(fn, nspin, nbf, npts, flat, w, Cd, occ, opts):
    V = torch.full((nspin * nbf * nbf,), float("nan"), dtype=torch.float64, device="cuda")
    E = C.c_double(0)
    st = fn(nbf, npts, *[A._p(x) for x in flat], A._p(w), nspin, NOCC, A._p(Cd), A._p(occ), C.byref(opts),
            C.byref(E), A._p(V), None)
    L.check(st)
    return E.value, V.cpu().numpy()


@pytest.mark.parametrize("nspin", [1, 2])
def test_noalloc_matches_allocating_entry_point_twice(nspin):
    lib = L.lib()
    nbf, npts, flat, w, Cd, occ = _inputs(nspin)
    assert nspin * npts * (nbf + 4) + 128 < SCRATCH_DOUBLES
    opts = A._opts(("GGA_X_PBE", "GGA_C_PBE"))
    E0, V0 = _call(lib.nkx_xc_dense, nspin, nbf, npts, flat, w, Cd, occ, opts)
    assert np.isfinite(V0).all() and np.abs(V0).max() > 0
    for _ in range(2):
        E1, V1 = _call(lib.nkx_xc_dense_noalloc, nspin, nbf, npts, flat, w, Cd, occ, opts)
        assert abs(E1 - E0) <= TOL * abs(E0)
        assert np.abs(V1 - V0).max() <= TOL * np.abs(V0).max()
    if nspin == 2:  # the two spin blocks really differ (the second block was read at its offset)
        assert np.abs(V0[: nbf * nbf] - V0[nbf * nbf:]).max() > 1e-6


@pytest.mark.parametrize("nbf,npts", [(2000, 4096), (64, 1 << 40)])
def test_noalloc_rejects_oversize_problem(nbf, npts):
    lib = L.lib()
    # rejected before any launch: the dummy buffers are never read
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    opts = A._opts(("LDA_X",))
    E = C.c_double(0)
    st = lib.nkx_xc_dense_noalloc(nbf, npts, A._p(dummy), None, None, None, A._p(dummy), 1, 1, A._p(dummy),
                                  A._p(dummy), C.byref(opts), C.byref(E), A._p(dummy), None)
    assert st == L.NKX_OK + 1
    assert b"32 MiB" in lib.nkx_last_error()
