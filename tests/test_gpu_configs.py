"""Parity with the CPU oracle on the benchmark workloads' own grid: Treutler-
Ahlrichs M4 75 radial x Lebedev 302 per atom, Becke with the Laqua clamp,
w > 1e-15, instead of the reduced grids of the other parity tests.

* the water case: Slater + VWN5, closed and open shell;
* the water-cluster case at n = 8: (H2O)_8 PBE (543,600 points before
  compaction, 384 functions, 40 orbitals);
* the grid itself, and the grid DF-J of water on it.

Tolerances: FP64 build vs oracle 1e-10 relative on E_xc and 1e-10 absolute on
V (V elements are O(1)); mixed build vs oracle at the accuracy gate of the
mixed scheme, |dE_xc| <= 1e-6 Eh and max|dV| <= 1e-7."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402

NRAD, ORDER = 75, 29  # Lebedev order 29 = 302 points
GATE_E, GATE_V = 1e-6, 1e-7


def config_grid(c, Z):
    return A.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=1e-15, radial="ta")


def check_fp64(E, V, Eo, Vo):
    assert abs(E - Eo) <= 1e-10 * abs(Eo), (E, Eo)
    for s in range(len(Vo)):
        Vs = V[s].cpu().numpy() if isinstance(V[s], torch.Tensor) else V[s]
        assert np.abs(Vs - Vo[s]).max() <= 1e-10 * max(1.0, np.abs(Vo[s]).max())


def check_gate(E, V, Eo, Vo):
    assert abs(E - Eo) <= GATE_E, (E, Eo)
    for s in range(len(Vo)):
        assert np.abs(V[s] - Vo[s]).max() <= GATE_V


def test_config_grid_matches_oracle_water_and_h2o8():
    # without compaction, so that weights within rounding of the 1e-15
    # threshold cannot drop a point on one side only; tiny weights come from
    # 1/2 (1 - p) near p = 1, where the fused multiply-adds of CPU and GPU
    # round differently (absolute tolerance)
    for n in (1, 8):
        c, Z = M.water() if n == 1 else M.water_cluster(n, 0)
        g = A.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, radial="ta")
        pts, w, own = O.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, scheme="ta")
        assert len(w) == 3 * n * NRAD * 302 and g.quad_points.shape == pts.shape
        assert np.array_equal(g.point_owner, own)
        np.testing.assert_allclose(g.quad_points, pts, rtol=0, atol=1e-13)
        np.testing.assert_allclose(g.weights, w, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("nspin", [1, 2])
def test_config1_water_slater_vwn5_fp64_and_mixed(nspin):
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    g = config_grid(c, Z)
    assert len(funcs) == 48 and len(g.weights) > 60000
    C_list = [M.random_orbitals(len(funcs), 5, seed=20 + s) for s in range(nspin)]
    occ_list = [np.ones(5) if s == 0 else np.array([1.0, 1.0, 1.0, 0.5, 0.0]) for s in range(nspin)]
    if nspin == 1:
        occ_list = [2.0 * np.ones(5)]
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=("LDA_X", "LDA_C_VWN"))
    Eo, Vo = O.xc_build(O.make_manual_basis(funcs), g.quad_points, g.weights, [1, 7], C_list, occ_list)
    E, V, _ = fb.build(C_list, occ_list, precision="fp64")
    check_fp64(E, V, Eo, Vo)
    Em, Vm, _ = fb.build(C_list, occ_list, precision="mixed")
    check_gate(Em, Vm, Eo, Vo)
    fb.close()


def test_config2_h2o8_pbe_fp64_and_mixed():
    c, Z = M.water_cluster(8, 0)
    funcs = M.sto_basis(c, Z)
    g = config_grid(c, Z)
    Cm = M.random_orbitals(len(funcs), 40, seed=0)
    occ = np.ones(40)
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=("GGA_X_PBE", "GGA_C_PBE"))
    Eo, Vo = O.xc_build(O.make_manual_basis(funcs), g.quad_points, g.weights, [101, 130], [Cm], [occ])
    E, V, _ = fb.build([Cm], [occ], precision="fp64")
    check_fp64(E, V, Eo, Vo)
    Em, Vm, _ = fb.build([Cm], [occ], precision="mixed")
    check_gate(Em, Vm, Eo, Vo)
    # device-resident orbitals give the same builds
    Cd, od = torch.as_tensor(Cm, device="cuda"), torch.as_tensor(occ, device="cuda")
    Ed, Vd, _ = fb.build([Cd], [od], precision="mixed")
    assert abs(Ed - Em) <= 1e-12 * abs(Em)
    assert float((Vd[0].cpu() - torch.as_tensor(Vm[0])).abs().max()) <= 1e-12
    fb.close()


def test_config_grid_coulomb_water():
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    aux = M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}, alpha=0.8, beta=2.5)
    g = config_grid(c, Z)
    Cm = M.random_orbitals(len(funcs), 5, seed=2)
    occ = 2.0 * np.ones(5)
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, aux=A.make_manual_basis(aux),
                       func_ids=("LDA_X", "LDA_C_VWN"))
    oaux = O.make_manual_basis(aux)
    S = O.aux_metric(oaux, g.quad_points, g.weights)
    Jo, _ = O.coulomb(O.make_manual_basis(funcs), oaux, g.quad_points, g.weights, Cm, occ, S=S)
    for prec, tol in (("fp64", 1e-9), ("mixed", 1e-7)):
        _, _, J = fb.build([Cm], [occ], precision=prec, want_J=True)
        assert np.abs(J - Jo).max() <= tol * np.abs(Jo).max(), prec
    fb.close()
