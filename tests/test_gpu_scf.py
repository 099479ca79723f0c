"""The water case: Slater + VWN5, TA-M4 75 x Lebedev 302,
plain closed-shell SCF to 1e-8 Eh with the stand-in driver
(nukexc_b200/scf.py) -- on the GPU (core Hamiltonian by quadrature through
nkx_core_hamiltonian_dense, XC and grid DF-J through nkx_fock_build) and on
the CPU (the oracle's core Hamiltonian, XC build and J).  Both converge and
agree; the mixed-precision Fock build converges to the same energy within
the mixed-precision gate."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402
from nukexc_b200 import scf  # noqa: E402

XC = ("LDA_X", "LDA_C_VWN")
AUX = {8: [(0, 6), (1, 5), (2, 4), (3, 2)], 1: [(0, 4), (1, 3), (2, 1)]}


def water_setup():
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    aux = M.sto_basis(c, Z, AUX, alpha=0.8, beta=2.5)
    return c, Z, funcs, aux


def gpu_scf(precision="fp64"):
    c, Z, funcs, aux = water_setup()
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    fb = A.FockBuilder(c, Z, b, g, aux=A.make_manual_basis(aux), func_ids=XC)
    S, T, V, H = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    return scf.rks(S.cpu().numpy(), H.cpu().numpy(), scf.gpu_fock(fb, precision), 5,
                   scf.nuclear_repulsion(c, Z))


def cpu_scf():
    c, Z, funcs, aux = water_setup()
    pts, w, _ = O.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, scheme="ta")
    b = O.make_manual_basis(funcs)
    ab = O.make_manual_basis(aux)
    S, T, V = O.core_hamiltonian(b, c, Z, pts, w)
    Sa = O.aux_metric(ab, pts, w)

    def fock(Cocc):
        occ = 2.0 * np.ones(Cocc.shape[1])
        E, Vx = O.xc_build(b, pts, w, [1, 7], [Cocc], [occ])
        J, _ = O.coulomb(b, ab, pts, w, Cocc, occ, S=Sa)
        return E, Vx[0], J
    return scf.rks(S, T + V, fock, 5, scf.nuclear_repulsion(c, Z))


def test_water_lda_scf_gpu_matches_cpu():
    rg = gpu_scf("fp64")
    rc = cpu_scf()
    assert rg["converged"] and rc["converged"]
    assert abs(rg["energy"] - rc["energy"]) < 1e-8
    assert abs(rg["energies"][-1] - rg["energies"][-2]) < 1e-8
    # the SCF lowers the energy from the core guess and ends bound
    assert rg["energy"] < rg["energies"][0] and rg["energy"] < -70.0


def test_water_lda_scf_mixed_precision_converges_to_fp64():
    r64 = gpu_scf("fp64")
    rmx = gpu_scf("mixed")
    assert rmx["converged"]
    assert abs(rmx["energy"] - r64["energy"]) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_water_lda_scf_device_resident_matches_host_loop(precision):
    # the same SCF with S, H, C, P, F on the GPU and device-buffer Fock
    # builds (scf.rks_device): the same energy as the host loop
    c, Z, funcs, aux = water_setup()
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    fb = A.FockBuilder(c, Z, b, g, aux=A.make_manual_basis(aux), func_ids=XC)
    S, T, V, H = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    enuc = scf.nuclear_repulsion(c, Z)
    rd = scf.rks_device(S, H, fb, 5, enuc, precision=precision)
    rh = scf.rks(S.cpu().numpy(), H.cpu().numpy(), scf.gpu_fock(fb, precision), 5, enuc)
    assert rd["converged"] and rh["converged"]
    assert abs(rd["energy"] - rh["energy"]) < (1e-9 if precision == "fp64" else 1e-6)
    fb.close()
