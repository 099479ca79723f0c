"""The sharded build of the C ABI on one GPU: the grid is split in two with
shard.balanced_split, each half gets its own plan, and the two "ranks" are
driven one after the other from this process (their kernels never wait for
each other).  The sums play the all-reduces: metric_0 + metric_1 is installed
in both plans (nkx_plan_set_metric), y_0 + y_1 from nkx_fock_build_phase1
goes into both nkx_fock_build_phase2 calls, and the partial E, V and J must
add up to the whole grid's single-plan build."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402
from nukexc_b200 import shard  # noqa: E402

XC = ("GGA_X_PBE", "GGA_C_PBE")


def _case():
    c, Z = M.water_cluster(2, seed=5)
    funcs = M.sto_basis(c, Z)
    aux = M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}, alpha=0.8, beta=2.5)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    Cm = M.random_orbitals(len(funcs), 10, seed=6)
    return c, Z, funcs, aux, g, Cm, 2.0 * np.ones(10)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-7)])
def test_two_plans_two_phases_equal_the_whole_grid(precision, tol):
    c, Z, funcs, aux, g, Cm, occ = _case()
    b, a = A.make_manual_basis(funcs), A.make_manual_basis(aux)
    full = A.FockBuilder(c, Z, b, g, aux=a, func_ids=XC)
    Ef, Vf, Jf = full.build([Cm], [occ], precision="fp64", want_J=True)
    parts = shard.balanced_split(g.quad_points, b.center, A.cutoff_radii(b), 10, 2)
    assert sum(len(p) for p in parts) == len(g.weights)
    fbs = [A.FockBuilder(c, Z, b, (g.quad_points[p], g.weights[p]), aux=a, func_ids=XC) for p in parts]
    S = sum(fb.aux_metric() for fb in fbs)
    assert np.abs(S - full.aux_metric()).max() <= 1e-12 * np.abs(S).max()
    for fb in fbs:
        fb.set_metric(S)
    y = sum(fb.build_phase1([Cm], [occ], precision=precision) for fb in fbs)
    outs = [fb.build_phase2(y, want_J=True) for fb in fbs]
    E = sum(o[0] for o in outs)
    V = sum(o[1][0] for o in outs)
    J = sum(o[2] for o in outs)
    assert abs(E - Ef) <= (1e-10 * abs(Ef) if precision == "fp64" else 1e-6)
    assert np.abs(V - Vf[0]).max() <= tol * max(1.0, np.abs(Vf[0]).max())
    assert np.abs(J - Jf).max() <= tol * np.abs(Jf).max()
    # device buffers take the same route (y stays on the GPU)
    yd = sum(fb.build_phase1([torch.as_tensor(Cm, device="cuda")], [torch.as_tensor(occ, device="cuda")],
                             precision=precision) for fb in fbs)
    Jd = sum(fb.build_phase2(yd, want_J=True)[2] for fb in fbs)
    assert float((Jd.cpu() - torch.as_tensor(J)).abs().max()) <= 1e-12 * np.abs(Jf).max()
    for fb in fbs + [full]:
        fb.close()


def test_phase2_needs_phase1():
    c, Z, funcs, aux, g, Cm, occ = _case()
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, aux=A.make_manual_basis(aux), func_ids=XC)
    fb._phase_nspin = 1
    with pytest.raises(Exception):
        fb.build_phase2(np.zeros(fb.naux), want_J=True)
    fb.close()

