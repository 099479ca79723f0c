"""Failure reporting of the Fock build, made on the host, on the GPU.

* Non-finite inputs: a NaN or Inf injected into the orbital coefficients or
  the occupations on the host must end the build with NKX_ERR_NUMERIC in
  both precisions (the mixed path would otherwise turn it into finite int8
  digits and return a finite, wrong V), and the next build on the same plan
  must be correct again.
* Bounded waits: with the plan's stall switch on, every tensor-core kernel
  first waits on an mbarrier that nothing completes; the wait runs out after
  the plan's (short) limit, the kernel drains what it issued, frees its
  tensor memory and returns, and the build reports NKX_ERR_TIMEOUT.  The next
  builds on the same plan (which allocate the same tensor memory again) must
  match the build made before.

No GPU fault, trap or endless loop is involved: the failures are host-made
inputs and a wait with a limit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from nukexc_b200 import _lib as L  # noqa: E402
from nukexc_b200 import api as A  # noqa: E402
from nukexc_b200 import molecules as M  # noqa: E402

NKX_ERR_TIMEOUT, NKX_ERR_NUMERIC = 4, 5
FUNCS = ("GGA_X_PBE", "GGA_C_PBE")


@pytest.fixture(scope="module")
def water():
    c, Z = M.water()
    funcs = M.sto_basis(c, Z)
    g = A.make_flat_grid(c, Z, 30, 11, weight_threshold=1e-15, radial="ta")
    fb = A.FockBuilder(c, Z, A.make_manual_basis(funcs), g, func_ids=FUNCS)
    Cm = M.random_orbitals(len(funcs), 5, seed=3)
    yield fb, Cm, np.ones(5)
    fb.close()


def _expect(code, fn):
    with pytest.raises(L.NkxError) as e:
        fn()
    assert e.value.code == code, str(e.value)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("where,value", [("C", np.nan), ("C", np.inf), ("occ", np.nan)])
def test_nonfinite_input_reports_numeric(water, precision, where, value):
    fb, Cm, occ = water
    E0, V0, _ = fb.build([Cm], [occ], precision=precision)
    Cb, ob = Cm.copy(), occ.copy()
    if where == "C":
        Cb[7, 2] = value
    else:
        ob[1] = value
    _expect(NKX_ERR_NUMERIC, lambda: fb.build([Cb], [ob], precision=precision))
    # device buffers take the same check
    _expect(NKX_ERR_NUMERIC, lambda: fb.build([torch.as_tensor(Cb, device="cuda")],
                                              [torch.as_tensor(ob, device="cuda")], precision=precision))
    E1, V1, _ = fb.build([Cm], [occ], precision=precision)
    assert abs(E1 - E0) <= 1e-12 * abs(E0)
    assert np.abs(V1[0] - V0[0]).max() <= 1e-12 * np.abs(V0[0]).max()


def test_nonfinite_orbitals_in_density_and_gradient(water):
    fb, Cm, occ = water
    Cb = Cm.copy()
    Cb[0, 0] = np.nan
    _expect(NKX_ERR_NUMERIC, lambda: fb.density([Cb], [occ], grad=True))
    _expect(NKX_ERR_NUMERIC, lambda: fb.xc_gradient([Cb], [occ]))
    assert np.isfinite(fb.density([Cm], [occ])).all()


@pytest.mark.parametrize("v_pair", [0, 1])
def test_stalled_wait_reports_timeout_and_plan_recovers(water, v_pair):
    """v_pair = 1: the V contraction on CTA pairs, whose waits give up in
    one CTA and stop the other through the cluster's shared memory."""
    fb, Cm, occ = water
    fb.set_tuning(v_pair=v_pair, v_warps=8 if v_pair else 16)
    E0, V0, _ = fb.build([Cm], [occ], precision="mixed")
    try:
        fb.set_wait_limit(ns=2_000_000, stall=True)  # 2 ms
        for _ in range(2):
            _expect(NKX_ERR_TIMEOUT, lambda: fb.build([Cm], [occ], precision="mixed"))
    finally:
        fb.set_wait_limit(0, stall=False)
    # every kernel freed its tensor memory: the next builds allocate it again
    for _ in range(2):
        E1, V1, _ = fb.build([Cm], [occ], precision="mixed")
        assert abs(E1 - E0) <= 1e-12 * abs(E0)
        assert np.abs(V1[0] - V0[0]).max() <= 1e-12 * np.abs(V0[0]).max()
    fb.set_tuning()


def test_short_wait_limit_without_stall_still_builds(water):
    """A limit far above the kernels' own wait times changes nothing."""
    fb, Cm, occ = water
    E0, V0, _ = fb.build([Cm], [occ], precision="mixed")
    try:
        fb.set_wait_limit(ns=200_000_000)  # 200 ms
        E1, V1, _ = fb.build([Cm], [occ], precision="mixed")
    finally:
        fb.set_wait_limit(0)
    assert abs(E1 - E0) <= 1e-12 * abs(E0)
    assert np.abs(V1[0] - V0[0]).max() <= 1e-12 * np.abs(V0[0]).max()
