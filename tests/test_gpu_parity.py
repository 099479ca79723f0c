"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the reference's golden values.  FP64 tolerances are written per test."""
import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402


def basis_pair(funcs):
    return A.make_manual_basis(funcs), O.make_manual_basis(funcs)


def h1s():
    return basis_pair([(1, 0, 0, 1.0, 0, 0, 0)])


# ------------------------------------------------------------- golden ----
def test_golden_lda_x_h1s_plan():
    # tests/test_hydrogen.cxx:815-857 through the batched plan (FP64)
    g = A.make_flat_grid([[0, 0, 0]], [1], 100, 20, radial="becke")
    b, _ = h1s()
    fb = A.FockBuilder([[0, 0, 0]], [1], b, g, func_ids=("LDA_X",))
    E, V, _ = fb.build([np.ones((1, 1))], [np.ones(1)])
    assert E == pytest.approx(KAT["h1s_lda_x"]["E"], rel=1e-10)


def test_golden_pbe_x_h1s_dense_and_plan():
    # tests/test_hydrogen.cxx:859-912
    g = A.make_flat_grid([[0, 0, 0]], [1], 100, 20, radial="becke")
    b, _ = h1s()
    phi, gx, gy, gz = A.fill_grad_collocation(b, g.quad_points)
    E, V = A.compute_gga(phi, gx, gy, gz, g.weights, np.ones((1, 1)), np.ones(1), ("GGA_X_PBE",))
    assert E == pytest.approx(KAT["h1s_pbe_x"]["E"], rel=1e-10)
    assert V[0, 0].item() == pytest.approx(KAT["h1s_pbe_x"]["V00"], rel=1e-10)
    fb = A.FockBuilder([[0, 0, 0]], [1], b, g, func_ids=("GGA_X_PBE",))
    E2, V2, _ = fb.build([np.ones((1, 1))], [np.ones(1)])
    assert E2 == pytest.approx(KAT["h1s_pbe_x"]["E"], rel=1e-10)
    assert V2[0][0, 0] == pytest.approx(KAT["h1s_pbe_x"]["V00"], rel=1e-10)


def test_golden_pbe_x_he1s():
    # tests/test_helium.cxx:67-119 (Becke 2000 radial; spherical integrand)
    g = A.make_flat_grid([[0, 0, 0]], [2], 2000, 41, radial="becke")
    b = A.make_manual_basis([(1, 0, 0, 1.6875, 0, 0, 0)])
    fb = A.FockBuilder([[0, 0, 0]], [2], b, g, func_ids=("GGA_X_PBE",))
    E, V, _ = fb.build([np.ones((1, 1))], [2 * np.ones(1)])
    assert E == pytest.approx(KAT["he1s_pbe_x"]["E"], rel=1e-10)
    assert V[0][0, 0] == pytest.approx(KAT["he1s_pbe_x"]["V00"], rel=1e-10)


@pytest.mark.parametrize("svd", [0.0, 1e-4])
def test_golden_coulomb_h1s(svd):
    # tests/test_hydrogen.cxx:562-631: J_00 = 5/8 (Cholesky, and the
    # reference's half-inverse with threshold 1e-4)
    g = A.make_flat_grid([[0, 0, 0]], [1], 100, 20, radial="becke")
    b, _ = h1s()
    aux = A.make_manual_basis([(1, 0, 0, z, 0, 0, 0) for z in (0.5, 1.0, 2.0, 3.0, 4.0)])
    fb = A.FockBuilder([[0, 0, 0]], [1], b, g, aux=aux, func_ids=("LDA_X",), metric_svd_thr=svd)
    E, V, J = fb.build([np.ones((1, 1))], [np.ones(1)], want_J=True)
    assert J[0, 0] == pytest.approx(KAT["h1s_coulomb"]["J00"], rel=1e-10)


def test_golden_density_sigma():
    # tests/test_density.cxx:252-307
    g = A.make_flat_grid([[0, 0, 0]], [1], 200, 20, radial="becke")
    b, _ = h1s()
    phi, gx, gy, gz = A.fill_grad_collocation(b, g.quad_points)
    rho, grad, sig = A.compute_density_and_sigma(phi, gx, gy, gz, np.ones((1, 1)), np.ones(1))
    w = torch.as_tensor(g.weights, device="cuda")
    assert (rho * w).sum().item() == pytest.approx(1.0, rel=1e-10)
    assert (sig * w).sum().item() == pytest.approx(1 / (2 * math.pi), rel=1e-10)


# ------------------------------------------------------- kernel parity ----
def test_becke_grid_matches_oracle():
    c, Z = M.water()
    g = A.make_flat_grid(c, Z, 40, 17, weight_threshold=1e-15, radial="ta")
    pts, w, own = O.make_flat_grid(c, Z, 40, 17, 1e-15, scheme="ta")
    assert g.quad_points.shape == pts.shape
    assert np.array_equal(g.point_owner, own)
    np.testing.assert_allclose(g.quad_points, pts, rtol=0, atol=1e-13)
    # tiny weights come from 1/2 (1 - p) near p = 1, where rounding of the
    # fused multiply-adds differs between CPU and GPU: absolute tolerance
    np.testing.assert_allclose(g.weights, w, rtol=1e-12, atol=1e-13)


def test_becke_unclamped_one_half():
    # tests/test_partition.cxx:140-195 on the device
    centers = np.array([[-1.0, 0, 0], [1.0, 0, 0]])
    pts = np.array([[0, j / 10, k / 10] for i in range(2) for j in range(10) for k in range(10)], float)
    owner = np.repeat([0, 1], 100)
    w = A.partition_becke(centers, pts, owner, np.ones(200)).cpu().numpy()
    assert np.abs(w - 0.5).max() < 1e-15


def test_becke_screening_exact_on_cluster():
    # clamped Becke with the exact r_min + 2 Rc screening vs the full loop
    c, Z = M.water_cluster(8, seed=3)
    rng = np.random.default_rng(0)
    owner = rng.integers(0, len(Z), 4000)
    pts = c[owner] + rng.normal(scale=2.0, size=(4000, 3))
    w0 = np.ones(4000)
    wd = A.partition_becke_team(c, pts, owner, w0).cpu().numpy()
    wo = O.becke(c, pts, owner, w0)
    np.testing.assert_allclose(wd, wo, rtol=1e-12, atol=1e-14)


def test_collocation_matches_oracle():
    # every l the device supports (l <= 7), values and gradients; the
    # oracle's harmonics are pinned to the reference's definition for l <= 7
    # in test_oracle_golden.py
    funcs = [(l + 1 + k, l, m, 0.7 + 0.9 * k, 0.1 * l, -0.2, 0.3 * k)
             for l in range(0, 8) for m in range(-l, l + 1) for k in range(2)]
    b, ob = basis_pair(funcs)
    pts = np.random.default_rng(1).normal(scale=1.5, size=(500, 3))
    d = [x.cpu().numpy() for x in A.fill_grad_collocation(b, pts)]
    o = O.collocation(ob, pts, grad=True)
    for x, y in zip(d, o):
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-14 * np.abs(y).max())


@pytest.mark.parametrize("fid", [1, 7, 12, 13, 101, 130])
@pytest.mark.parametrize("nspin", [1, 2])
def test_functionals_match_oracle(fid, nspin):
    rng = np.random.default_rng(fid + nspin)
    n = 2000
    rho = 10 ** rng.uniform(-12, 2, size=n * nspin)
    sig = 10 ** rng.uniform(-14, 3, size=n * (1 if nspin == 1 else 3))
    if nspin == 2:
        s = sig.reshape(n, 3)
        s[:, 1] = rng.uniform(-1, 1, size=n) * np.sqrt(s[:, 0] * s[:, 2])
    de, dv, ds = A.xc_eval(fid, nspin, rho, sig)
    oe, ov, os_ = O.xc_eval(fid, nspin, rho, sig)
    # near rho -> 0 the PBE correlation energy per particle is a cancelling
    # difference (eps_c + H -> 0); an absolute floor of 1e-15 Eh per particle
    # covers the last-bit differences of CPU and GPU libm there
    np.testing.assert_allclose(de.cpu().numpy(), oe, rtol=1e-11, atol=1e-15)
    dvn = dv.cpu().numpy()
    if nspin == 2:
        # at extreme spin polarisation (zeta -> +-1) the minority-spin
        # potential is a cancelling difference; compare against the scale of
        # both spin potentials of the point
        scale = np.repeat(np.abs(ov.reshape(-1, 2)).sum(1), 2)
        assert (np.abs(dvn - ov) <= 1e-9 * np.abs(ov) + 1e-10 * scale + 1e-13).all()
    else:
        np.testing.assert_allclose(dvn, ov, rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(ds.cpu().numpy(), os_, rtol=1e-9, atol=1e-14 * np.abs(os_).max())


# --------------------------------------------------------- plan parity ----
def water_case(n=1, seed=0, nrad=40, order=17):
    c, Z = (M.water() if n == 1 else M.water_cluster(n, seed))
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, nrad, order, weight_threshold=1e-15, radial="ta")
    return c, Z, funcs, g


@pytest.mark.parametrize("funcs_xc", [("LDA_X", "LDA_C_VWN"), ("GGA_X_PBE", "GGA_C_PBE")])
def test_plan_xc_fp64_matches_oracle_water(funcs_xc):
    c, Z, funcs, g = water_case()
    b, ob = basis_pair(funcs)
    nbf = len(funcs)
    Cm = M.random_orbitals(nbf, 5, seed=4)
    occ = np.ones(5)
    fb = A.FockBuilder(c, Z, b, g, func_ids=funcs_xc)
    E, V, _ = fb.build([Cm], [occ])
    ids = [A._FUNC_NAMES[f] for f in funcs_xc]
    Eo, Vo = O.xc_build(ob, g.quad_points, g.weights, ids, [Cm], [occ])
    assert abs(E - Eo) < 1e-10 * abs(Eo)
    assert np.abs(V[0] - Vo[0]).max() < 1e-10 * max(1.0, np.abs(Vo).max())


def test_plan_xc_fp64_polarized_and_device_buffers():
    c, Z, funcs, g = water_case(2, seed=1, nrad=30, order=11)
    b, ob = basis_pair(funcs)
    nbf = len(funcs)
    Ca = M.random_orbitals(nbf, 6, seed=5)
    Cb = M.random_orbitals(nbf, 4, seed=6)
    occ = [np.ones(6), np.ones(6)]
    Cb6 = np.concatenate([Cb, np.zeros((nbf, 2))], 1)
    fb = A.FockBuilder(c, Z, b, g, func_ids=("GGA_X_PBE", "GGA_C_PBE"))
    E, V, _ = fb.build([torch.as_tensor(Ca, device="cuda"), torch.as_tensor(Cb6, device="cuda")],
                       [torch.as_tensor(o, device="cuda") for o in occ])
    Eo, Vo = O.xc_build(ob, g.quad_points, g.weights, [101, 130], [Ca, Cb6], occ)
    assert abs(E - Eo) < 1e-10 * abs(Eo)
    for s in range(2):
        assert np.abs(V[s].cpu().numpy() - Vo[s]).max() < 1e-10 * max(1.0, np.abs(Vo).max())


def test_plan_chunked_equals_single_chunk():
    # a tiny workspace forces many chunks (two-pass collocation)
    c, Z, funcs, g = water_case(2, seed=2, nrad=30, order=11)
    b, _ = basis_pair(funcs)
    Cm = M.random_orbitals(len(funcs), 10, seed=7)
    f1 = A.FockBuilder(c, Z, b, g)
    f2 = A.FockBuilder(c, Z, b, g, workspace_bytes=3 << 20)
    assert f2.info()["nchunks"] > 3
    E1, V1, _ = f1.build([Cm], [np.ones(10)])
    E2, V2, _ = f2.build([Cm], [np.ones(10)])
    assert abs(E1 - E2) < 1e-12 * abs(E1)
    assert np.abs(V1[0] - V2[0]).max() < 1e-12


def small_aux(c, Z):
    # compact even-tempered aux set whose grid metric is well conditioned
    return M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}, alpha=0.8, beta=2.5)


@pytest.mark.parametrize("svd", [0.0, 1e-6])
def test_plan_coulomb_matches_oracle(svd):
    c, Z, funcs, g = water_case(1, nrad=40, order=17)
    b, ob = basis_pair(funcs)
    aux, oaux = basis_pair(small_aux(c, Z))
    Cm = M.random_orbitals(len(funcs), 5, seed=8)
    occ = np.ones(5)
    fb = A.FockBuilder(c, Z, b, g, aux=aux, func_ids=("LDA_X",), metric_svd_thr=svd)
    assert fb.info()["naux"] == len(oaux["n"])
    E, V, J = fb.build([Cm], [occ], want_J=True)
    S = O.aux_metric(oaux, g.quad_points, g.weights)
    if svd:
        Jo, _ = O.coulomb(ob, oaux, g.quad_points, g.weights, Cm, occ, X=O.half_inverse(S, svd))
    else:
        Jo, _ = O.coulomb(ob, oaux, g.quad_points, g.weights, Cm, occ, S=S)
    assert np.abs(J - Jo).max() < 1e-9 * np.abs(Jo).max()
    # fused J folds into the XC contraction: V_fused = V_xc + J
    Ef, Vf, _ = fb.build([Cm], [occ], fuse_j=True)
    assert abs(Ef - E) < 1e-12 * abs(E)
    assert np.abs(Vf[0] - (V[0] + J)).max() < 1e-10 * np.abs(Jo).max()


def test_plan_coulomb_loose_aux_shells():
    # aux shells outside the (centre, l <= 3) groups -- a g shell (l = 4) and
    # a lone m = 0 d function -- go through the per-shell kernels
    c, Z, funcs, g = water_case(1, nrad=40, order=17)
    b, ob = basis_pair(funcs)
    af = list(small_aux(c, Z))
    o = c[0]
    af += [(5, 4, m, 2.0, o[0], o[1], o[2]) for m in range(-4, 5)]
    af += [(3, 2, 0, 1.3, o[0], o[1], o[2])]
    aux, oaux = basis_pair(af)
    Cm = M.random_orbitals(len(funcs), 5, seed=9)
    occ = np.ones(5)
    fb = A.FockBuilder(c, Z, b, g, aux=aux, func_ids=("LDA_X",), metric_svd_thr=1e-6)
    _, _, J = fb.build([Cm], [occ], want_J=True)
    S = O.aux_metric(oaux, g.quad_points, g.weights)
    Jo, _ = O.coulomb(ob, oaux, g.quad_points, g.weights, Cm, occ, X=O.half_inverse(S, 1e-6))
    assert np.abs(J - Jo).max() < 1e-9 * np.abs(Jo).max()


def test_plan_coulomb_pivoted_cholesky_baseline_aux():
    # the even-tempered zeta_k = 0.3 * 1.8^k aux set: the grid metric is
    # indefinite, the pivoted Cholesky drops near-dependent functions and J
    # stays symmetric and finite
    c, Z, funcs, g = water_case(1, nrad=40, order=17)
    b, _ = basis_pair(funcs)
    aux, _ = basis_pair(M.aux_basis(c, Z))
    fb = A.FockBuilder(c, Z, b, g, aux=aux, func_ids=("LDA_X",))
    Cm = M.random_orbitals(len(funcs), 5, seed=8)
    E, V, J = fb.build([Cm], [np.ones(5)], want_J=True)
    assert np.isfinite(J).all() and np.abs(J - J.T).max() < 1e-12 * np.abs(J).max()
    assert 0 < fb.info()["metric_min_diag"]


def test_golden_coulomb_h1s_dense():
    # tests/test_hydrogen.cxx:562-631 through the dense compute_coulomb
    # (nkx_coulomb_dense) with the reference's half inverse (thr 1e-4)
    g = A.make_flat_grid([[0, 0, 0]], [1], 100, 20, radial="becke")
    b, _ = h1s()
    aux = A.make_manual_basis([(1, 0, 0, z, 0, 0, 0) for z in (0.5, 1.0, 2.0, 3.0, 4.0)])
    phi = A.fill_collocation(b, g.quad_points)
    phi_aux = A.fill_collocation(aux, g.quad_points)
    Vw = A.sto_potential_collocation_scaled(aux, g.quad_points, g.weights)
    S = 0.5 * (phi_aux @ Vw.t() + Vw @ phi_aux.t())
    X = A.compute_half_inverse(S, 1e-4)
    J = A.compute_coulomb(np.ones((1, 1)), np.ones(1), phi, phi_aux, Vw, X)
    assert J[0, 0].item() == pytest.approx(KAT["h1s_coulomb"]["J00"], rel=1e-10)


def test_core_hamiltonian_matches_oracle():
    # nkx_core_hamiltonian_dense vs the oracle's quadrature (water, and the
    # exact H 1s values S = 1, T = 1/2, V = -1)
    c, Z, funcs, g = water_case(1, nrad=40, order=17)
    b, ob = basis_pair(funcs)
    S, T, V, H = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    So, To, Vo = O.core_hamiltonian(ob, c, Z, g.quad_points, g.weights)
    for X, Xo in ((S, So), (T, To), (V, Vo)):
        assert np.abs(X.cpu().numpy() - Xo).max() < 1e-11 * max(1.0, np.abs(Xo).max())
    gh = A.make_flat_grid([[0, 0, 0]], [1], 200, 20, radial="becke")
    bh, _ = h1s()
    S, T, V, _ = A.compute_core_hamiltonian(bh, [[0, 0, 0]], [1], gh.quad_points, gh.weights)
    assert S[0, 0].item() == pytest.approx(1.0, rel=1e-10)
    assert T[0, 0].item() == pytest.approx(0.5, rel=1e-9)
    assert V[0, 0].item() == pytest.approx(-1.0, rel=1e-9)


def test_golden_exchange_h1s_dense():
    # tests/test_hydrogen.cxx:688-758: K_00 = 5/8
    c, Z = np.zeros((1, 3)), np.array([1])
    g = A.make_flat_grid(c, Z, 100, 20, radial="becke")
    b = A.make_manual_basis([(1, 0, 0, 1.0, 0, 0, 0)])
    aux = A.make_manual_basis([(1, 0, 0, z, 0, 0, 0) for z in (0.5, 1.0, 2.0, 3.0, 4.0)])
    phi = A.fill_collocation(b, g.quad_points)
    phia = A.fill_collocation(aux, g.quad_points)
    vw = A.sto_potential_collocation_scaled(aux, g.quad_points, g.weights)
    S = (phia @ vw.t() + vw @ phia.t()) / 2
    X = A.compute_half_inverse(S, KAT["h1s_exchange"]["half_inverse_thr"])
    K = A.compute_exact_exchange(np.ones((1, 1)), np.ones(1), phi, phia, vw, X)
    assert float(K[0, 0]) == pytest.approx(KAT["h1s_exchange"]["K00"], rel=KAT["h1s_exchange"]["rel"])


def test_exchange_matches_oracle_water():
    c, Z, funcs, g = water_case(1, nrad=30, order=11)
    b, ob = basis_pair(funcs)
    aux, oaux = basis_pair(small_aux(c, Z))
    Cm = M.random_orbitals(len(funcs), 5, seed=12)
    occ = np.linspace(2.0, 1.0, 5)
    S = O.aux_metric(oaux, g.quad_points, g.weights)
    X = O.half_inverse(S, 1e-6)
    phi = A.fill_collocation(b, g.quad_points)
    phia = A.fill_collocation(aux, g.quad_points)
    vw = A.sto_potential_collocation_scaled(aux, g.quad_points, g.weights)
    K = A.compute_exact_exchange(Cm, occ, phi, phia, vw, X).cpu().numpy()
    Ko = O.exchange(ob, oaux, g.quad_points, g.weights, Cm, occ, X)
    assert np.abs(K - Ko).max() < 1e-10 * np.abs(Ko).max()
    assert np.abs(K - K.T).max() < 1e-12 * np.abs(Ko).max()


def test_core_hamiltonian_screened_plan_matches_dense():
    # nkx_plan_core_hamiltonian integrates only the significant (batch,
    # block) pairs of the plan; on (H2O)4 (two function blocks, some pairs
    # screened out) it equals the dense quadrature up to what the 1e-10
    # cutoff drops (the reference asks 1e-6 of its screened variants,
    # tests/test_integration.cxx:83-311)
    # four waters 50 bohr apart on a line: two function blocks, and the
    # batches at one end are out of reach of the other end's functions
    c1, Z1 = M.water()
    c = np.concatenate([np.asarray(c1, float) + [0.0, 0.0, 50.0 * k] for k in range(4)])
    Z = np.concatenate([Z1] * 4)
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    b, ob = basis_pair(funcs)
    fb = A.FockBuilder(c, Z, b, g, func_ids=("LDA_X",))
    assert fb.info()["npairs"] < fb.info()["nbatches"] * fb.info()["nblocks"]  # screening active
    S, T, V = fb.core_hamiltonian(c, Z)
    Sd, Td, Vd, _ = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    for X, Xd in ((S, Sd), (T, Td), (V, Vd)):
        Xd = Xd.cpu().numpy()
        assert np.abs(X - X.T).max() <= 1e-14 * np.abs(Xd).max()
        assert np.abs(X - Xd).max() <= 1e-8 * max(1.0, np.abs(Xd).max())
    So, To, Vo = O.core_hamiltonian(ob, c, Z, g.quad_points, g.weights)
    assert np.abs(S - So).max() <= 1e-8 and np.abs(T - To).max() <= 1e-8 * np.abs(To).max()
    fb.close()
