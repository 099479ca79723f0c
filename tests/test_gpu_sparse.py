"""The reference's sparse / tiled path (nukexc/octree.hpp, the *_sparse and
*_tiled functions of density.hpp, xc_integrals.hpp and coulomb.hpp) through
the Python mirror: Morton bounding boxes, neighbour lists, the grid Coulomb
metric, the caller's half inverse, J alone, per-call functionals and the
plan density, each against the oracle on seeded water inputs."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402


def case(n=1, seed=0, nrad=40, order=17):
    c, Z = (M.water() if n == 1 else M.water_cluster(n, seed))
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, nrad, order, weight_threshold=1e-15, radial="ta")
    return c, Z, funcs, g


def small_aux(c, Z):
    return M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}, alpha=0.8, beta=2.5)


def test_bounding_boxes_and_neighbor_list_match_brute_force():
    c, Z, funcs, g = case(2, seed=3, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    w0 = np.sort(g.weights.copy())
    own0 = np.bincount(g.point_owner, minlength=len(Z))
    m = 32
    boxes = A.create_bounding_boxes(g, m).cpu().numpy()
    G = len(g.weights)
    assert boxes.shape == ((G + m - 1) // m, 2, 3)
    # in-place permutation of points, weights and owners
    assert np.array_equal(np.sort(g.weights), w0)
    assert np.array_equal(np.bincount(g.point_owner, minlength=len(Z)), own0)
    p = g.quad_points.reshape(-1, 3)
    k = np.arange(G) // m
    assert np.all(p >= boxes[k, 0]) and np.all(p <= boxes[k, 1])
    nl = A.build_neighbor_list(b, boxes, m, G)
    off = nl.offsets.cpu().numpy()
    nb = nl.neighbors.cpu().numpy()
    ob = O.make_manual_basis(funcs)
    ctr, rc = ob["center"], ob["cutoff"]
    for j in range(len(boxes)):
        e = np.maximum(np.maximum(boxes[j, 0] - ctr, 0.0), ctr - boxes[j, 1])
        want = np.nonzero((e * e).sum(1) <= rc * rc)[0]
        assert np.array_equal(nb[off[j]:off[j + 1]], want)


@pytest.mark.parametrize("nspin", [1, 2])
def test_plan_density_and_sigma_match_oracle(nspin):
    c, Z, funcs, g = case(2, seed=1, nrad=30, order=11)
    b = A.make_manual_basis(funcs)
    ob = O.make_manual_basis(funcs)
    nbf = len(funcs)
    Cs = [M.random_orbitals(nbf, 6 - s, seed=10 + s) for s in range(nspin)]
    Cs = [np.concatenate([x, np.zeros((nbf, 6 - x.shape[1]))], 1) for x in Cs]
    occ = [np.linspace(1.0, 0.5, 6) for _ in range(nspin)]
    fb = A.FockBuilder(c, Z, b, g, func_ids=("LDA_X",))
    rho, grad, sigma = fb.density(Cs, occ, grad=True)
    phi, gx, gy, gz = O.collocation(ob, g.quad_points, grad=True)
    for s in range(nspin):
        psi = Cs[s].T @ phi
        r = (occ[s][:, None] * psi * psi).sum(0)
        gr = np.stack([2.0 * (occ[s][:, None] * psi * (Cs[s].T @ d)).sum(0) for d in (gx, gy, gz)])
        assert np.abs(rho[s] - r).max() <= 1e-12 * np.abs(r).max()
        assert np.abs(grad[s] - gr).max() <= 1e-11 * np.abs(gr).max()
        assert np.abs(sigma[s] - (gr * gr).sum(0)).max() <= 1e-11 * (gr * gr).sum(0).max()
    # the value-only call agrees with the gradient call
    assert np.abs(fb.density(Cs, occ) - rho).max() <= 1e-14 * np.abs(rho).max()


def test_aux_metric_half_inverse_and_j_alone():
    c, Z, funcs, g = case(1)
    b = A.make_manual_basis(funcs)
    ob = O.make_manual_basis(funcs)
    af = small_aux(c, Z)
    aux = A.make_manual_basis(af)
    oaux = O.make_manual_basis(af)
    S_o = O.aux_metric(oaux, g.quad_points, g.weights)
    S_d = A.coulomb_overlap_integral(aux, g.quad_points, g.weights).cpu().numpy()
    assert np.abs(S_d - S_o).max() <= 1e-12 * np.abs(S_o).max()
    # pivoted-Cholesky plan, then the caller's half inverse (compute_coulomb_sparse)
    fb = A.FockBuilder(c, Z, b, g, aux=aux, func_ids=("LDA_X",))
    assert np.abs(fb.aux_metric() - S_o).max() <= 1e-12 * np.abs(S_o).max()
    X = O.half_inverse(S_o, 1e-6)
    fb.set_half_inverse(X)
    Cm = M.random_orbitals(len(funcs), 5, seed=8)
    occ = np.ones(5)
    E, V, J = fb.build([Cm], [occ], want_J=True, want_V=False)
    assert V is None
    Jo, _ = O.coulomb(ob, oaux, g.quad_points, g.weights, Cm, occ, X=X)
    assert np.abs(J - Jo).max() < 1e-9 * np.abs(Jo).max()
    # the same J next to V, from device buffers
    Ct = torch.as_tensor(Cm, device="cuda")
    _, V2, J2 = fb.build([Ct], [torch.ones(5, dtype=torch.float64, device="cuda")], want_J=True)
    assert np.abs(J2.cpu().numpy() - J).max() <= 1e-13 * np.abs(J).max()


def test_set_functional_equals_new_plan():
    c, Z, funcs, g = case(1)
    b = A.make_manual_basis(funcs)
    Cm = M.random_orbitals(len(funcs), 5, seed=2)
    occ = np.ones(5)
    ref = A.FockBuilder(c, Z, b, g, func_ids=("GGA_X_PBE",))
    Er, Vr, _ = ref.build([Cm], [occ])
    fb = A.FockBuilder(c, Z, b, g, func_ids=("LDA_X",))
    El, _, _ = fb.build([Cm], [occ])
    fb.set_functional(("GGA_X_PBE",))
    E, V, _ = fb.build([Cm], [occ])
    assert E == pytest.approx(Er, rel=1e-14)
    assert np.abs(V[0] - Vr[0]).max() <= 1e-14 * np.abs(Vr[0]).max()
    assert abs(El - Er) > 1e-3


def test_neighbor_list_screening_regression():
    # tests/test_neighborlist.cxx:50-140 on a synthetic stand-in: 8-point
    # boxes, basis cutoff 1e-6; the CSR offsets are non-decreasing and a
    # (H2O)32 cluster screens away over 30 % of the box x function pairs
    # (36.7 % by a host brute-force count of the same boxes)
    c, Z = M.water_cluster(32, 4)
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs, cutoff_tol=1e-6)
    bb = A.create_bounding_boxes(g, 8)
    nl = A.build_neighbor_list(b, bb, 8, len(g.weights))
    off = nl.offsets.cpu().numpy()
    assert np.all(np.diff(off) >= 0)
    dense = (len(off) - 1) * b.nbf()
    screened = int(off[-1])
    assert screened < dense
    assert 1.0 - screened / dense > 0.3
