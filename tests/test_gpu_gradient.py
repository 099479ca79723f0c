"""The XC nuclear gradient (nkx_xc_gradient, FP64 and mixed) against central finite
differences of E_xc at fixed orbitals, with the grid rebuilt at each displaced
geometry (points move with their owner atom, Becke weights recomputed, no
weight-threshold compaction).  The finite-difference oracle is the CPU
oracle's dense XC build: central differences at h = 1e-4 and h/2 bohr,
Richardson-extrapolated (error O(h^4)).  Gate: 1e-5 Eh/bohr (the force
tolerance of the mixed-precision target); checked here at 1e-8."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402

H = 1e-4
NRAD, ORDER = 30, 11


def funcs_at(c, Z, shells=None):
    return M.sto_basis(c, Z, shells) if shells else M.sto_basis(c, Z)


def oracle_energy(c, Z, ids, C_list, occ_list, shells=None):
    pts, w, _ = O.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, scheme="ta")
    E, _ = O.xc_build(O.make_manual_basis(funcs_at(c, Z, shells)), pts, w, ids, C_list, occ_list)
    return E


def fd_component(c, Z, a, k, ids, C_list, occ_list, shells=None):
    def central(h):
        cp, cm = c.copy(), c.copy()
        cp[a, k] += h
        cm[a, k] -= h
        return (oracle_energy(cp, Z, ids, C_list, occ_list, shells) -
                oracle_energy(cm, Z, ids, C_list, occ_list, shells)) / (2 * h)
    return (4.0 * central(H / 2) - central(H)) / 3.0


def fd_gradient(c, Z, ids, C_list, occ_list, shells=None, atoms=None):
    c = np.asarray(c, float)
    G = np.zeros_like(c)
    for a in (range(len(Z)) if atoms is None else atoms):
        for k in range(3):
            G[a, k] = fd_component(c, Z, a, k, ids, C_list, occ_list, shells)
    return G


def analytic(c, Z, func_ids, C_list, occ_list, shells=None):
    g = A.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, radial="ta")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs_at(c, Z, shells)), g, func_ids=func_ids)
    return fb.xc_gradient(C_list, occ_list)


@pytest.mark.parametrize("xc", [("LDA_X", "LDA_C_VWN"), ("GGA_X_PBE", "GGA_C_PBE")])
def test_water_gradient_vs_oracle_fd(xc):
    c, Z = M.water()
    c = np.asarray(c) + np.random.default_rng(1).normal(0, 0.05, size=np.shape(c))
    nbf = len(funcs_at(c, Z))
    Cm = M.random_orbitals(nbf, 5, seed=2)
    occ = 2.0 * np.ones(5)
    ids = [A._FUNC_NAMES[f] for f in xc]
    Ga = analytic(c, Z, xc, [Cm], [occ])
    Gf = fd_gradient(c, Z, ids, [Cm], [occ])
    assert np.abs(Ga - Gf).max() < 1e-8
    # translation invariance of E_xc (points and weights move with the atoms)
    assert np.abs(Ga.sum(0)).max() < 1e-9


def test_open_shell_gradient_vs_oracle_fd():
    c, Z = M.water()
    c = np.asarray(c) + np.random.default_rng(3).normal(0, 0.05, size=np.shape(c))
    nbf = len(funcs_at(c, Z))
    Ca, Cb = M.random_orbitals(nbf, 5, seed=4), M.random_orbitals(nbf, 4, seed=5)
    Cb = np.concatenate([Cb, np.zeros((nbf, 1))], axis=1)
    occ = [np.ones(5), np.r_[np.ones(4), 0.0]]
    xc = ("GGA_X_PBE", "GGA_C_PBE")
    Ga = analytic(c, Z, xc, [Ca, Cb], occ)
    Gf = fd_gradient(c, Z, [101, 130], [Ca, Cb], occ, atoms=[0, 1])
    assert np.abs(Ga[:2] - Gf[:2]).max() < 1e-8
    assert np.abs(Ga.sum(0)).max() < 1e-9


def test_cluster_gradient_translation_invariance_and_fd_spot_check():
    # (H2O)2 with d functions: two FD components against the oracle, and the
    # translation sum over all six atoms
    c, Z = M.water_cluster(2, seed=6)
    nbf = len(funcs_at(c, Z))
    Cm = M.random_orbitals(nbf, 10, seed=7)
    occ = 2.0 * np.ones(10)
    xc = ("GGA_X_PBE", "GGA_C_PBE")
    Ga = analytic(c, Z, xc, [Cm], [occ])
    assert np.abs(Ga.sum(0)).max() < 1e-8
    cc = np.asarray(c, float)
    for a, k in ((0, 2), (4, 0)):
        fd = fd_component(cc, Z, a, k, [101, 130], [Cm], [occ])
        assert abs(Ga[a, k] - fd) < 1e-8


# ------------------------------------------- autograd wrapper (test only) ----
class XcEnergy(torch.autograd.Function):
    """E_xc(R) of a fixed set of orbitals as a differentiable function of the
    nuclear coordinates R (natoms x 3, bohr, FP64): forward rebuilds the grid
    (points moving with their owner atoms, Becke weights, no compaction), the
    basis centres and the plan at R and returns the FP64 E_xc of the GPU build;
    backward returns grad_output * dE_xc/dR from nkx_xc_gradient.  It lives in
    the test harness only: the library's interface is the C ABI."""

    @staticmethod
    def forward(ctx, R, Z, func_ids, C_list, occ_list, clamp):
        c = R.detach().cpu().numpy()
        g = A.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, radial="ta", becke_clamp=clamp)
        fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs_at(c, Z)), g, func_ids=func_ids)
        E, _, _ = fb.build(C_list, occ_list, precision="fp64")
        G = fb.xc_gradient(C_list, occ_list, becke_clamp=clamp)
        fb.close()
        ctx.save_for_backward(torch.as_tensor(G, dtype=R.dtype))
        return torch.tensor(E, dtype=R.dtype)

    @staticmethod
    def backward(ctx, gE):
        (G,) = ctx.saved_tensors
        return gE * G, None, None, None, None, None


def test_autograd_wrapper_gradcheck_water():
    # torch.autograd.gradcheck: central differences of the wrapped FP64 E_xc
    # (eps 1e-4 bohr) against backward() for all nine coordinates
    c, Z = M.water()
    c = np.asarray(c) + np.random.default_rng(8).normal(0, 0.05, size=np.shape(c))
    Cm = M.random_orbitals(len(funcs_at(c, Z)), 5, seed=9)
    occ = 2.0 * np.ones(5)
    R = torch.tensor(c, dtype=torch.float64, requires_grad=True)
    f = lambda x: XcEnergy.apply(x, Z, ("GGA_X_PBE", "GGA_C_PBE"), [Cm], [occ], 5.0)  # noqa: E731
    assert torch.autograd.gradcheck(f, (R,), eps=1e-4, atol=1e-7, rtol=1e-6)
    E = f(R)
    E.backward()
    assert torch.abs(R.grad.sum(0)).max() < 1e-9  # translation invariance


def test_screened_becke_gradient_short_clamp_cluster():
    # a short Laqua clamp (2 bohr) on (H2O)4 makes the per-point candidate
    # list of the Becke-weight term drop most atoms (r >= r_min + 2 Rc); the
    # analytic gradient still equals Richardson central differences of the
    # GPU E_xc built on grids with the same clamp
    c, Z = M.water_cluster(4, seed=10)
    c = np.asarray(c, float)
    Cm = M.random_orbitals(len(funcs_at(c, Z)), 20, seed=11)
    occ = 2.0 * np.ones(20)
    xc = ("GGA_X_PBE", "GGA_C_PBE")
    R = torch.tensor(c, dtype=torch.float64, requires_grad=True)
    E = XcEnergy.apply(R, Z, xc, [Cm], [occ], 2.0)
    E.backward()
    G = R.grad.numpy()
    assert np.abs(G.sum(0)).max() < 1e-8

    def energy(cc):
        return float(XcEnergy.apply(torch.tensor(cc), Z, xc, [Cm], [occ], 2.0))

    for a, k in ((1, 0), (6, 2), (11, 1)):
        def central(h):
            cp, cm = c.copy(), c.copy()
            cp[a, k] += h
            cm[a, k] -= h
            return (energy(cp) - energy(cm)) / (2 * h)
        fd = (4.0 * central(H / 2) - central(H)) / 3.0
        assert abs(G[a, k] - fd) < 1e-8, (a, k, G[a, k], fd)


@pytest.mark.parametrize("xc", [("LDA_X", "LDA_C_VWN"), ("GGA_X_PBE", "GGA_C_PBE")])
def test_mixed_gradient_matches_fp64(xc):
    # the mixed-precision gradient (orbital values and density from the int8
    # digit contraction) against the FP64 one on (H2O)4, closed and open
    # shell: well inside the 1e-5 Eh/bohr force target, translation invariant
    c, Z = M.water_cluster(4, seed=12)
    c = np.asarray(c, float)
    nbf = len(funcs_at(c, Z))
    g = A.make_flat_grid(c, Z, NRAD, ORDER, weight_threshold=-1.0, radial="ta")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs_at(c, Z)), g, func_ids=xc)
    Ca, Cb = M.random_orbitals(nbf, 20, seed=13), M.random_orbitals(nbf, 20, seed=14)
    for C_list, occ_list in (([Ca], [2.0 * np.ones(20)]), ([Ca, Cb], [np.ones(20), np.r_[np.ones(17), np.zeros(3)]])):
        G64 = fb.xc_gradient(C_list, occ_list)
        for _ in range(2):
            Gm = fb.xc_gradient(C_list, occ_list, precision="mixed")
            assert np.abs(Gm - G64).max() < 1e-6, np.abs(Gm - G64).max()
            assert np.abs(Gm.sum(0)).max() < 1e-8
    fb.close()
