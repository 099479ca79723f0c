"""ctypes binding of ``libnkx.so`` (the C ABI declared in include/nkx.h).

The library is loaded from the package directory; there is no fallback:
if it is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnkx.so")

NKX_OK = 0
PREC_FP64, PREC_MIXED = 0, 1
RADIAL_BECKE, RADIAL_TA = 0, 1
SIZING_UNIFORM, SIZING_PYSCF = 0, 1
MEM_DEVICE, MEM_HOST = 0, 1
XC_LDA_X, XC_LDA_C_VWN, XC_GGA_X_PBE, XC_GGA_C_PBE = 1, 7, 101, 130
XC_LDA_C_PW, XC_LDA_C_PW_MOD = 12, 13

EXPORTS = [
    "nkx_make_flat_grid", "nkx_becke_partition", "nkx_fill_collocation", "nkx_density_dense",
    "nkx_xc_dense", "nkx_xc_dense_noalloc", "nkx_xc_eval", "nkx_potential_collocation", "nkx_half_inverse", "nkx_coulomb_dense", "nkx_core_hamiltonian_dense",
    "nkx_plan_create", "nkx_plan_get_info", "nkx_fock_build", "nkx_get_last_timing",
    "nkx_plan_last_density", "nkx_plan_batch_blocks", "nkx_plan_destroy", "nkx_last_error", "nkx_xc_gradient",
    "nkx_plan_set_functional", "nkx_plan_set_half_inverse", "nkx_plan_aux_metric", "nkx_plan_density",
    "nkx_morton_order", "nkx_neighbor_list", "nkx_aux_metric", "nkx_exchange_dense", "nkx_plan_set_wait_limit",
    "nkx_fock_build_phase1", "nkx_fock_build_phase2", "nkx_plan_set_metric",
    "nkx_plan_autotune", "nkx_plan_get_tuning", "nkx_plan_set_tuning", "nkx_plan_core_hamiltonian",
    "nkx_plan_set_graph",
]


class Molecule(C.Structure):
    _fields_ = [("natoms", C.c_int), ("xyz", C.c_void_p), ("Z", C.c_void_p)]


class Basis(C.Structure):
    _fields_ = [("nbf", C.c_int), ("n", C.c_void_p), ("l", C.c_void_p), ("m", C.c_void_p),
                ("zeta", C.c_void_p), ("center", C.c_void_p), ("cutoff_tol", C.c_double)]


class GridSpec(C.Structure):
    _fields_ = [("radial_scheme", C.c_int), ("nrad", C.c_int), ("nang_order", C.c_int),
                ("weight_threshold", C.c_double), ("ta_alpha", C.c_double), ("sizing", C.c_int),
                ("becke_clamp", C.c_double)]


class PlanOptions(C.Structure):
    _fields_ = [("batch_points", C.c_int), ("screen_tol", C.c_double), ("nfunc", C.c_int),
                ("func_ids", C.c_int * 4), ("dens_threshold", C.c_double),
                ("workspace_bytes", C.c_size_t), ("metric_svd_thr", C.c_double)]


class PlanInfo(C.Structure):
    _fields_ = [("npoints", C.c_long), ("nbatches", C.c_long), ("nbf", C.c_int), ("naux", C.c_int),
                ("nblocks", C.c_int), ("npairs", C.c_long), ("nchunks", C.c_int),
                ("metric_min_diag", C.c_double), ("graph_replays", C.c_long)]


class BuildTiming(C.Structure):
    _fields_ = [("colloc_ms", C.c_float), ("density_ms", C.c_float), ("functional_ms", C.c_float),
                ("coulomb_ms", C.c_float), ("zbuild_ms", C.c_float), ("vgemm_ms", C.c_float),
                ("total_ms", C.c_float), ("launches", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("v_n", C.c_int), ("dens_n", C.c_int), ("ypath", C.c_int), ("v_warps", C.c_int),
                ("v_pair", C.c_int), ("chunk_pairs", C.c_long),
                ("from_cache", C.c_int), ("trials", C.c_int), ("default_ms", C.c_float), ("best_ms", C.c_float)]


class NkxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"nkx status {code}: {msg}")
        self.code = code


_L = None


def lib():
    """Load libnkx.so (raises if it has not been built)."""
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m nukexc_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, l_, d = C.c_void_p, C.c_int, C.c_long, C.c_double
        sig = {
            "nkx_make_flat_grid": [vp, vp, vp, vp, vp, vp],
            "nkx_becke_partition": [vp, i, vp, vp, l_, vp, d, vp],
            "nkx_fill_collocation": [vp, vp, l_, vp, vp, vp, vp, vp],
            "nkx_density_dense": [i, l_, vp, vp, vp, vp, i, vp, vp, vp, vp, vp, vp],
            "nkx_xc_dense": [i, l_, vp, vp, vp, vp, vp, i, i, vp, vp, vp, vp, vp, vp],
            "nkx_xc_dense_noalloc": [i, l_, vp, vp, vp, vp, vp, i, i, vp, vp, vp, vp, vp, vp],
            "nkx_xc_eval": [i, i, l_, vp, vp, d, vp, vp, vp, vp],
            "nkx_potential_collocation": [vp, vp, vp, l_, vp, vp],
            "nkx_half_inverse": [i, vp, d, vp, vp, vp],
            "nkx_coulomb_dense": [i, i, l_, vp, vp, vp, i, i, vp, vp, vp, vp],
            "nkx_exchange_dense": [i, i, l_, vp, vp, vp, i, i, vp, vp, vp, vp],
            "nkx_core_hamiltonian_dense": [vp, vp, vp, vp, l_, vp, vp, vp, vp],
            "nkx_plan_create": [vp, vp, vp, l_, vp, vp, vp, vp, vp],
            "nkx_plan_get_info": [vp, vp],
            "nkx_fock_build": [vp, i, i, i, vp, vp, i, i, vp, vp, vp, vp],
            "nkx_fock_build_phase1": [vp, i, i, i, vp, vp, i, vp, vp],
            "nkx_fock_build_phase2": [vp, vp, i, i, vp, vp, vp, vp],
            "nkx_plan_set_metric": [vp, vp, i],
            "nkx_plan_autotune": [vp, i, i, vp, vp, i, C.c_char_p, vp, vp],
            "nkx_plan_get_tuning": [vp, vp],
            "nkx_plan_core_hamiltonian": [vp, vp, vp, vp, vp, i, vp],
            "nkx_plan_set_graph": [vp, i],
            "nkx_plan_set_tuning": [vp, vp],
            "nkx_xc_gradient": [vp, i, i, i, vp, vp, i, d, vp, vp],
            "nkx_get_last_timing": [vp, vp],
            "nkx_plan_last_density": [vp, vp, vp],
            "nkx_plan_batch_blocks": [vp, vp],
            "nkx_plan_destroy": [vp],
            "nkx_plan_set_functional": [vp, i, vp, d],
            "nkx_plan_set_half_inverse": [vp, i, vp, i],
            "nkx_plan_set_wait_limit": [vp, C.c_ulonglong, i],
            "nkx_plan_aux_metric": [vp, vp, i],
            "nkx_plan_density": [vp, i, i, vp, vp, i, i, vp, vp, vp, vp],
            "nkx_morton_order": [l_, vp, vp],
            "nkx_neighbor_list": [i, vp, vp, l_, vp, vp, vp, vp, vp],
            "nkx_aux_metric": [vp, l_, vp, vp, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.nkx_last_error.restype = C.c_char_p
        L.nkx_last_error.argtypes = []
        _L = L
    return _L


def check(status):
    if status != NKX_OK:
        raise NkxError(status, lib().nkx_last_error().decode())
