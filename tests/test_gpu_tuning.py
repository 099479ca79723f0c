"""The mixed build's tunable choices and the autotuner (nkx_plan_autotune).

Every combination of the V contraction's shape (one CTA per tile at
N = 128 / 64, or CTA pairs at M = 256 x N = 64), the density MMA width
(N = 64 / 128) and the Y path of the GGA density gradient must give the
same build: bit-for-bit up to the order of FP64 additions for the same
algorithm (1e-12), and within the mixed scheme's gate of the FP64 build
(|dE| <= 1e-6 Eh, max|dV| <= 1e-7) across the Y-path switch.  Re-chunking
changes nothing either.  The autotuner returns valid choices, stores them in
its cache file and applies them from there on the next plan of the same
problem."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402

XC = ("GGA_X_PBE", "GGA_C_PBE")


@pytest.fixture(scope="module")
def case():
    c, Z = M.water_cluster(4, seed=1)
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    Cm = M.random_orbitals(len(funcs), 20, seed=2)
    return c, Z, funcs, g, Cm, np.ones(20)


def test_widths_and_y_path_give_the_same_build(case):
    c, Z, funcs, g, Cm, occ = case
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=XC)
    E64, V64, _ = fb.build([Cm], [occ], precision="fp64")
    ref = {}
    # V shapes: one CTA at N = 128 with 16 or 8 epilogue warps, one CTA at
    # N = 64, CTA pairs with 8 or 16 epilogue warps a CTA
    shapes = ((128, 16, 0), (128, 8, 0), (64, 16, 0), (64, 8, 1), (64, 16, 1))
    for (v_n, v_w, v_p), d_n, yp in itertools.product(shapes, (64, 128), (0, 1)):
        fb.set_tuning(v_n=v_n, dens_n=d_n, ypath=yp, v_warps=v_w, v_pair=v_p)
        E, V, _ = fb.build([Cm], [occ], precision="mixed")
        assert abs(E - E64) <= 1e-6 and np.abs(V[0] - V64[0]).max() <= 1e-7, (v_n, v_w, v_p, d_n, yp)
        if yp in ref:
            Er, Vr = ref[yp]
            assert abs(E - Er) <= 1e-12 * abs(Er) and np.abs(V[0] - Vr).max() <= 1e-12, (v_n, v_w, v_p, d_n, yp)
        else:
            ref[yp] = (E, V[0])
    fb.close()


def test_rechunking_keeps_the_build(case):
    c, Z, funcs, g, Cm, occ = case
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=XC)
    E0, V0, _ = fb.build([Cm], [occ], precision="mixed")
    n0 = fb.info()["nchunks"]
    fb.set_tuning(chunk_pairs=7)
    assert fb.info()["nchunks"] > n0
    E1, V1, _ = fb.build([Cm], [occ], precision="mixed")
    assert abs(E1 - E0) <= 1e-12 * abs(E0) and np.abs(V1[0] - V0[0]).max() <= 1e-12
    E2, V2, _ = fb.build([Cm], [occ], precision="fp64")
    assert abs(E2 - E0) <= 1e-6
    fb.close()


def test_autotune_chooses_applies_and_caches(case, tmp_path):
    c, Z, funcs, g, Cm, occ = case
    cache = str(tmp_path / "tuning.txt")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=XC)
    t = fb.autotune([Cm], [occ], cache_path=cache)
    assert t["from_cache"] == 0 and t["trials"] >= 4
    assert t["v_n"] in (64, 128) and t["dens_n"] in (64, 128) and t["ypath"] in (-1, 0, 1)
    assert t["v_warps"] in (8, 16) and t["v_pair"] in (0, 1)
    assert 0 < t["best_ms"] <= t["default_ms"] * 1.0001
    assert fb.tuning()["v_n"] == t["v_n"] and fb.tuning()["chunk_pairs"] == t["chunk_pairs"]
    E, V, _ = fb.build([Cm], [occ], precision="mixed")
    E64, V64, _ = fb.build([Cm], [occ], precision="fp64")
    assert abs(E - E64) <= 1e-6 and np.abs(V[0] - V64[0]).max() <= 1e-7
    fb.close()
    fb2 = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=XC)
    t2 = fb2.autotune([Cm], [occ], cache_path=cache)
    assert t2["from_cache"] == 1
    keys = ("v_n", "dens_n", "ypath", "v_warps", "v_pair", "chunk_pairs")
    assert tuple(t2[k] for k in keys) == tuple(t[k] for k in keys)
    fb2.close()
