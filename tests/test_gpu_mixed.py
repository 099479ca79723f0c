"""The mixed-precision Fock build (exact int8-digit contractions on the
tcgen05 tensor cores, kind::i8 with int32 accumulation and an FP64 combine)
against the FP64 CUDA path and the CPU oracle.  Accuracy gates: |dE_xc| <= 1e-6 Eh and max|dV_xc| <= 1e-7
(the mixed-precision target), tighter where the systems are small."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402

E_TOL = 1e-6
V_TOL = 1e-7


def case(n, seed=0, nrad=40, order=17):
    c, Z = (M.water() if n == 1 else M.water_cluster(n, seed))
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, nrad, order, weight_threshold=1e-15, radial="ta")
    return c, Z, funcs, g


@pytest.mark.parametrize("xc", [("LDA_X", "LDA_C_VWN"), ("GGA_X_PBE", "GGA_C_PBE")])
def test_mixed_water_vs_oracle(xc):
    c, Z, funcs, g = case(1)
    b = A.make_manual_basis(funcs)
    Cm = M.random_orbitals(len(funcs), 5, seed=1)
    occ = np.ones(5)
    fb = A.FockBuilder(c, Z, b, g, func_ids=xc)
    E, V, _ = fb.build([Cm], [occ], precision="mixed")
    ids = [A._FUNC_NAMES[f] for f in xc]
    Eo, Vo = O.xc_build(O.make_manual_basis(funcs), g.quad_points, g.weights, ids, [Cm], [occ])
    assert abs(E - Eo) < E_TOL
    assert np.abs(V[0] - Vo[0]).max() < V_TOL


def test_mixed_cluster_polarized_vs_fp64():
    c, Z, funcs, g = case(4, seed=2, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    nbf = len(funcs)
    Ca = M.random_orbitals(nbf, 20, seed=3)
    Cb = M.random_orbitals(nbf, 20, seed=4)
    occ = [np.ones(20), np.r_[np.ones(18), np.zeros(2)]]
    fb = A.FockBuilder(c, Z, b, g)
    E64, V64, _ = fb.build([Ca, Cb], occ, precision="fp64")
    Em, Vm, _ = fb.build([Ca, Cb], occ, precision="mixed")
    assert abs(Em - E64) < E_TOL
    for s in range(2):
        assert np.abs(Vm[s] - V64[s]).max() < V_TOL


def test_mixed_chunked_and_nocc_over_128():
    # nocc 150 spans two orbital tiles; a small workspace forces chunks
    c, Z, funcs, g = case(4, seed=5, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    Cm = M.random_orbitals(len(funcs), 150, seed=6)
    occ = np.ones(150)
    f1 = A.FockBuilder(c, Z, b, g)
    f2 = A.FockBuilder(c, Z, b, g, workspace_bytes=24 << 20)
    assert f2.info()["nchunks"] > 2
    E64, V64, _ = f1.build([Cm], [occ], precision="fp64")
    for fb in (f1, f2):
        Em, Vm, _ = fb.build([Cm], [occ], precision="mixed")
        assert abs(Em - E64) < E_TOL
        assert np.abs(Vm[0] - V64[0]).max() < V_TOL


def test_mixed_fused_coulomb_vs_fp64():
    c, Z, funcs, g = case(2, seed=7, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    aux = A.make_manual_basis(M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]},
                                          alpha=0.8, beta=2.5))
    Cm = M.random_orbitals(len(funcs), 10, seed=8)
    occ = np.ones(10)
    fb = A.FockBuilder(c, Z, b, g, aux=aux)
    E64, V64, J64 = fb.build([Cm], [occ], precision="fp64", want_J=True)
    Em, Vm, Jm = fb.build([Cm], [occ], precision="mixed", want_J=True)
    assert abs(Em - E64) < E_TOL
    assert np.abs(Vm[0] - V64[0]).max() < V_TOL
    assert np.abs(Jm - J64).max() < 1e-6 * np.abs(J64).max()
    Ef, Vf, _ = fb.build([Cm], [occ], precision="mixed", fuse_j=True)
    assert np.abs(Vf[0] - (V64[0] + J64)).max() < 1e-6 * np.abs(J64).max()


def test_mixed_gga_many_orbitals_gradient_path():
    # 264 and 260 occupied orbitals (padded to 320): the GGA density gradient
    # goes through Y = T0 (C occ)^T and the grad phi contraction
    c, Z, funcs, g = case(6, seed=7, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    nbf = len(funcs)
    assert nbf >= 264
    C1 = M.random_orbitals(nbf, 264, seed=8)
    fb = A.FockBuilder(c, Z, b, g)
    occ = np.linspace(1.0, 0.3, 264)
    E64, V64, _ = fb.build([C1], [occ], precision="fp64")
    Em, Vm, _ = fb.build([C1], [occ], precision="mixed")
    assert abs(Em - E64) < E_TOL
    assert np.abs(Vm[0] - V64[0]).max() < V_TOL
    Cb = np.concatenate([M.random_orbitals(nbf, 260, seed=9), np.zeros((nbf, 4))], 1)
    occ2 = [np.ones(264), np.r_[np.ones(260), np.zeros(4)]]
    E64, V64, _ = fb.build([C1, Cb], occ2, precision="fp64")
    Em, Vm, _ = fb.build([C1, Cb], occ2, precision="mixed")
    assert abs(Em - E64) < E_TOL
    for s in range(2):
        assert np.abs(Vm[s] - V64[s]).max() < V_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pinned_host_buffers_match_device_build(precision):
    """Host builds from page-locked CPU tensors (C column-major and occ passed
    as they are, V written into the caller's pinned out_V) equal the build
    from device tensors and the one from numpy arrays, twice in a row."""
    c, Z, funcs, g = case(2, seed=7)
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=("GGA_X_PBE", "GGA_C_PBE"))
    nbf = len(funcs)
    Cm = M.random_orbitals(nbf, 9, seed=8)
    occ = np.linspace(2.0, 1.0, 9)
    Ed, Vd, _ = fb.build([torch.as_tensor(Cm, device="cuda")], [torch.as_tensor(occ, device="cuda")],
                         precision=precision)
    En, Vn, _ = fb.build([Cm], [occ], precision=precision)
    Cp = torch.empty((9, nbf), dtype=torch.float64, pin_memory=True)
    Cp.copy_(torch.from_numpy(np.ascontiguousarray(Cm.T)))
    op = torch.empty(9, dtype=torch.float64, pin_memory=True)
    op.copy_(torch.from_numpy(occ))
    Vp = torch.empty(nbf * nbf, dtype=torch.float64, pin_memory=True)
    for _ in range(2):
        Vp.fill_(float("nan"))
        Ep, Vs, _ = fb.build([Cp.t()], [op], precision=precision, out_V=Vp)
        assert np.shares_memory(Vs[0], Vp.numpy())
        scale = float(Vd[0].abs().max())
        for E, V in ((Ed, Vd[0].cpu().numpy()), (En, Vn[0])):
            assert abs(Ep - E) <= 1e-12 * abs(E)
            assert np.abs(Vs[0] - V).max() <= 1e-12 * scale
    fb.close()
