"""CUDA-graph replay of the Fock build (nkx_plan_set_graph): builds with
device buffers are recorded into a graph on the second call of a kind and
replayed from then on.  Replayed builds must equal ordinary ones (up to the
order of atomic FP64 additions: 1e-12, and 1e-10 for what carries the
Coulomb fit), with the caller passing new buffers
each time; a change of kind (precision, J mode) or of the plan re-records;
the water SCF on the device converges to the same energy with replays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402
from nukexc_b200 import scf  # noqa: E402

AUX = {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}


def _plan(graph):
    c, Z = M.water_cluster(2, seed=4)
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, aux=A.make_manual_basis(M.sto_basis(c, Z, AUX, 0.8, 2.5)),
                       func_ids=("GGA_X_PBE", "GGA_C_PBE"))
    fb.set_graph(graph)
    Cm = torch.as_tensor(M.random_orbitals(len(funcs), 10, seed=5), device="cuda")
    return fb, Cm, torch.full((10,), 2.0, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("jmode", ["none", "fused", "separate"])
def test_replayed_builds_equal_ordinary_builds(precision, jmode):
    kw = {"none": {}, "fused": {"fuse_j": True}, "separate": {"want_J": True}}[jmode]
    ref, Cm, occ = _plan(False)
    Er, Vr, Jr = ref.build([Cm], [occ], precision=precision, **kw)
    fb, _, _ = _plan(True)
    for it in range(4):
        C2 = (Cm * (1.0 + 1e-3 * it)).contiguous()  # new buffer and new values each call
        E, V, J = fb.build([C2], [occ], precision=precision, **kw)
        Eo, Vo, Jo = ref.build([C2], [occ], precision=precision, **kw)
        assert abs(E - Eo) <= 1e-12 * abs(Eo)
        # with J fused, V holds the Coulomb potential, whose fit vector varies
        # at rounding level from build to build (below)
        vtol = 1e-10 if jmode == "fused" else 1e-12
        assert float((V[0] - Vo[0]).abs().max()) <= vtol * float(Vo[0].abs().max())
        if jmode == "separate":
            # the fit vector y is summed with atomic FP64 adds in varying order
            # and the solve with the grid metric (condition number about 1e5 for
            # this aux set) magnifies that rounding in J
            assert float((J - Jo).abs().max()) <= 1e-10 * float(Jo.abs().max())
    assert fb.info()["graph_replays"] >= 2
    ref.close()
    fb.close()


def test_kind_and_plan_changes_re_record():
    fb, Cm, occ = _plan(True)
    ref, _, _ = _plan(False)
    for prec in ("mixed", "fp64", "mixed", "mixed", "fp64", "fp64"):
        E, V, _ = fb.build([Cm], [occ], precision=prec)
        Eo, Vo, _ = ref.build([Cm], [occ], precision=prec)
        assert abs(E - Eo) <= 1e-12 * abs(Eo)
    n = fb.info()["graph_replays"]
    assert n >= 2
    fb.set_functional(("LDA_X",))
    ref.set_functional(("LDA_X",))
    for _ in range(3):
        E, V, _ = fb.build([Cm], [occ], precision="mixed")
        Eo, Vo, _ = ref.build([Cm], [occ], precision="mixed")
        assert abs(E - Eo) <= 1e-12 * abs(Eo)
    assert fb.info()["graph_replays"] > n


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_scf_with_graph_replays(precision):
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    aux = M.sto_basis(c, Z, {8: [(0, 6), (1, 5), (2, 4), (3, 2)], 1: [(0, 4), (1, 3), (2, 1)]}, alpha=0.8, beta=2.5)
    g = A.make_flat_grid(c, Z, 75, 29, weight_threshold=1e-15, radial="ta")
    b = A.make_manual_basis(funcs)
    S, T, V, H = A.compute_core_hamiltonian(b, c, Z, g.quad_points, g.weights)
    enuc = scf.nuclear_repulsion(c, Z)
    out = []
    for graph in (False, True):
        fb = A.FockBuilder(c, Z, b, g, aux=A.make_manual_basis(aux), func_ids=("LDA_X", "LDA_C_VWN"))
        fb.set_graph(graph)
        r = scf.rks_device(S, H, fb, 5, enuc, precision=precision, conv=1e-10 if precision == "fp64" else 1e-8)
        assert r["converged"]
        out.append((r["energy"], fb.info()["graph_replays"]))
        fb.close()
    # FP64 (converged to 1e-10 Eh between iterations): the same energy.  Mixed
    # (converged to 1e-8, its practical floor: the orbitals' int8 digits round
    # differently from one iteration to the next, which moves E by about
    # 1e-9, and the small-system V adds batch splits atomically in varying
    # order): the two runs stop within about two thresholds of each other
    assert abs(out[0][0] - out[1][0]) < (1e-10 if precision == "fp64" else 3e-8)
    assert out[0][1] == 0 and out[1][1] >= 5
