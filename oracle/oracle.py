"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes front end of ``liboracle.so`` (the C++/OpenMP FP64 restatement of the
NuKEXC grid-integration algorithms in ``oracle.cpp``) plus the host-side
grid assembly of ``make_flat_grid`` (nukexc/grid.hpp:172-348).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use this module, as the checker or the timed CPU baseline.  The product
package ``nukexc_b200`` never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")

ANG_TO_BOHR = 1.8897259885681697  # nukexc/atomic_properties.hpp:49

# Treutler-Ahlrichs radial scale xi per element (JCP 102, 346 (1995),
# Table 1; the reference's TA_XI, nukexc/grid.hpp:98-102)
TA_XI = [0.00, 0.8, 0.9, 1.8, 1.4, 1.3, 1.1, 0.9, 0.9, 0.9, 0.9, 1.4, 1.3,
         1.3, 1.2, 1.1, 1.0, 1.0, 1.0, 1.5, 1.4, 1.3, 1.2, 1.2, 1.2,
         1.2, 1.2, 1.2, 1.1, 1.1, 1.1, 1.1, 1.0, 0.9, 0.9, 0.9, 0.9]
# Bragg-Slater radii in Angstrom, H modified by Becke (JCP 88, 2547 (1988);
# the reference's BECKE_SLATER_RADII, nukexc/grid.hpp:71-96), Z <= 36
BRAGG = [0.00, 0.35, 0.35, 1.45, 1.05, 0.85, 0.70, 0.65, 0.60, 0.50, 0.35,
         1.80, 1.50, 1.25, 1.10, 1.00, 1.00, 1.00, 0.70, 2.20, 1.80, 1.60,
         1.45, 1.40, 1.35, 1.40, 1.35, 1.35, 1.35, 1.35, 1.35, 1.30, 1.25,
         1.15, 1.10, 1.00, 0.90]
PYSCF_RADIAL_RATIO = [1.0, 1.5, 1.6, 1.8, 1.9, 2.0, 2.1]  # grid.hpp:142


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib():
    global _L
    try:
        return _L
    except NameError:
        pass
    if not os.path.exists(_SO):
        build()
    L = C.CDLL(_SO)
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L.orc_lebedev_npts.argtypes = [C.c_int]
    L.orc_lebedev.argtypes = [C.c_int, dp, dp]
    L.orc_radial.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, dp, dp]
    L.orc_becke.argtypes = [C.c_int, dp, C.c_int, dp, ip, dp, C.c_double]
    L.orc_atom_grids.restype = C.c_long
    L.orc_atom_grids.argtypes = [C.c_int, dp, ip, dp, C.c_int, C.c_double, C.c_int,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_cutoff.restype = C.c_double
    L.orc_cutoff.argtypes = [C.c_int, C.c_double, C.c_double]
    L.orc_sto_norm.restype = C.c_double
    L.orc_sto_norm.argtypes = [C.c_int, C.c_double]
    L.orc_solid_harmonic.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp]
    L.orc_collocation.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp,
                                  C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_xc_eval.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_void_p, C.c_double, dp, dp, C.c_void_p]
    L.orc_xc_build.restype = C.c_double
    L.orc_xc_build.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp, C.c_int, ip,
                               C.c_int, C.c_int, dp, dp, C.c_double, dp, C.c_void_p]
    L.orc_sto_potential.restype = C.c_double
    L.orc_sto_potential.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double]
    L.orc_potential_collocation.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp, dp]
    L.orc_half_inverse.restype = C.c_int
    L.orc_half_inverse.argtypes = [C.c_int, dp, C.c_double, dp]
    L.orc_cholesky_solve.restype = C.c_int
    L.orc_cholesky_solve.argtypes = [C.c_int, dp, dp, dp]
    L.orc_aux_metric.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, dp, dp]
    L.orc_coulomb.restype = C.c_int
    L.orc_coulomb.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, ip, ip, ip, dp, dp,
                              C.c_int, dp, dp, C.c_int, dp, dp, C.c_void_p, C.c_int,
                              C.c_void_p, dp, C.c_void_p]
    _L = L
    return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- grids ----
def lebedev(order):
    L = _lib()
    n = L.orc_lebedev_npts(order)
    xyz = np.zeros(3 * n)
    w = np.zeros(n)
    L.orc_lebedev(order, xyz, w)
    return xyz.reshape(n, 3), w


def radial(scheme, n, R, alpha=0.6):
    r = np.zeros(n)
    w = np.zeros(n)
    _lib().orc_radial({"becke": 0, "ta": 1}[scheme], n, float(R), float(alpha), r, w)
    return r, w


def _period(Z):
    for p, zmax in enumerate([2, 10, 18, 36, 54, 86]):
        if Z <= zmax:
            return p + 1
    return 7


def radial_scale(Z, scheme):
    """Per-atom radial scale R (nukexc/grid.hpp:227-235)."""
    if scheme == "ta":
        return TA_XI[Z] if Z < len(TA_XI) else 1.0
    return 0.5 * BRAGG[Z] * ANG_TO_BOHR if Z < len(BRAGG) else 1.0


def becke(centers, pts, owner, weights, clamp_R=5.0):
    """partition_becke_team (clamp_R=5) or partition_becke (clamp_R=0)."""
    w = _f64(weights).copy()
    c = _f64(centers).reshape(-1)
    p = _f64(pts).reshape(-1)
    _lib().orc_becke(len(c) // 3, c, len(w), p, _i32(owner), w, float(clamp_R))
    return w


def make_flat_grid(centers, Z, nrad=50, nang_order=30, weight_threshold=1e-30,
                   scheme="ta", ta_alpha=0.6, sizing="uniform", partition=True):
    """make_flat_grid (nukexc/grid.hpp:172-348): per-atom grids, Becke
    partition (Laqua-clamped team variant), then removal of points with
    w <= weight_threshold.  The compaction keeps the original order (the
    reference's atomic fetch-add order is nondeterministic, grid.hpp:329-338).
    """
    centers = _f64(centers).reshape(-1, 3)
    Z = list(Z)
    na = len(Z)
    nr = np.array([int(nrad * PYSCF_RADIAL_RATIO[_period(z) - 1] + 0.5) if sizing == "pyscf" else nrad
                   for z in Z], dtype=np.int32)
    Rs = np.array([radial_scale(z, scheme) for z in Z])
    L = _lib()
    sch = {"becke": 0, "ta": 1}[scheme]
    tot = L.orc_atom_grids(na, centers.reshape(-1), nr, Rs, sch, ta_alpha, nang_order, None, None, None)
    pts = np.zeros((tot, 3))
    w = np.zeros(tot)
    owner = np.zeros(tot, dtype=np.int32)
    L.orc_atom_grids(na, centers.reshape(-1), nr, Rs, sch, ta_alpha, nang_order,
                     _ptr(pts), _ptr(w), _ptr(owner))
    if (w < 0).any():
        raise RuntimeError("Detected negative weights aborting")
    if partition:
        w = becke(centers, pts, owner, w)
    keep = w > weight_threshold
    return pts[keep].copy(), w[keep].copy(), owner[keep].copy()


# ---------------------------------------------------------------- basis ----
def make_manual_basis(funcs, cutoff_tol=1e-10):
    """make_manual_basis (nukexc/stobasis.hpp:175-225); funcs are
    (n, l, m, zeta, ox, oy, oz)."""
    L = _lib()
    f = list(funcs)
    b = {
        "n": _i32([x[0] for x in f]), "l": _i32([x[1] for x in f]), "m": _i32([x[2] for x in f]),
        "zeta": _f64([x[3] for x in f]), "center": _f64([[x[4], x[5], x[6]] for x in f]).reshape(-1, 3),
    }
    b["norm"] = _f64([L.orc_sto_norm(int(x[0]), float(x[3])) for x in f])
    b["cutoff"] = _f64([L.orc_cutoff(int(x[0]), float(x[3]), cutoff_tol) for x in f])
    return b


def _bargs(b):
    return (len(b["n"]), b["n"], b["l"], b["m"], b["zeta"], _f64(b["center"]).reshape(-1))


def collocation(b, pts, grad=False):
    """Column-major (nbf x npts) Phi and optionally its gradient; returned as
    numpy arrays of shape (nbf, npts)."""
    pts = _f64(pts).reshape(-1, 3)
    nbf = len(b["n"])
    np_ = len(pts)
    phi = np.zeros(nbf * np_)
    g = [np.zeros(nbf * np_) for _ in range(3)] if grad else [None] * 3
    _lib().orc_collocation(*_bargs(b), np_, pts.reshape(-1), phi, *[_ptr(x) for x in g])
    sh = lambda a: a.reshape(np_, nbf).T.copy()  # noqa: E731
    if grad:
        return sh(phi), sh(g[0]), sh(g[1]), sh(g[2])
    return sh(phi)


def solid_harmonic(l, m, x, y, z):
    out = np.zeros(4)
    _lib().orc_solid_harmonic(l, m, x, y, z, out)
    return out


# ------------------------------------------------------------------- XC ----
def xc_eval(func_id, nspin, rho, sigma=None, thr=1e-15):
    rho = _f64(rho)
    npt = len(rho) // nspin
    exc = np.zeros(npt)
    vrho = np.zeros(npt * nspin)
    vs = np.zeros(npt * (1 if nspin == 1 else 3)) if sigma is not None else None
    sg = _f64(sigma) if sigma is not None else None
    _lib().orc_xc_eval(func_id, nspin, npt, rho, _ptr(sg), thr, exc, vrho, _ptr(vs))
    return exc, vrho, vs


def xc_build(b, pts, w, func_ids, C_list, occ_list, thr=1e-15, want_rho=False):
    """Dense XC build; C_list/occ_list hold one (C, occ) per spin.  Returns
    (E_xc, V) with V of shape (nspin, nbf, nbf)."""
    nspin = len(C_list)
    nbf = len(b["n"])
    nocc = C_list[0].shape[1]
    Cc = np.concatenate([_f64(np.asarray(c, dtype=np.float64).T).reshape(-1) for c in C_list])
    oc = np.concatenate([_f64(o) for o in occ_list])
    pts = _f64(pts).reshape(-1, 3)
    V = np.zeros(nspin * nbf * nbf)
    rho = np.zeros(len(pts) * nspin) if want_rho else None
    E = _lib().orc_xc_build(*_bargs(b), len(pts), pts.reshape(-1), _f64(w), len(func_ids),
                            _i32(func_ids), nspin, nocc, Cc, oc, thr, V, _ptr(rho))
    Vs = V.reshape(nspin, nbf, nbf).transpose(0, 2, 1).copy()
    if want_rho:
        return E, Vs, rho.reshape(-1, nspin)
    return E, Vs


# -------------------------------------------------------------- Coulomb ----
def sto_potential(n, l, m, x, y, z, zeta):
    return _lib().orc_sto_potential(n, l, m, x, y, z, zeta)


def potential_collocation(aux, pts, w):
    pts = _f64(pts).reshape(-1, 3)
    na = len(aux["n"])
    out = np.zeros(na * len(pts))
    _lib().orc_potential_collocation(*_bargs(aux), len(pts), pts.reshape(-1), _f64(w), out)
    return out.reshape(len(pts), na).T.copy()


def aux_metric(aux, pts, w):
    pts = _f64(pts).reshape(-1, 3)
    na = len(aux["n"])
    S = np.zeros(na * na)
    _lib().orc_aux_metric(*_bargs(aux), len(pts), pts.reshape(-1), _f64(w), S)
    return S.reshape(na, na).T.copy()


def half_inverse(S, thr=1e-5):
    S = np.asarray(S, dtype=np.float64)
    N = S.shape[0]
    X = np.zeros(N * N)
    K = _lib().orc_half_inverse(N, _f64(S.T).reshape(-1), thr, X)
    return X.reshape(N, N).T[:, :K].copy()


def coulomb(b, aux, pts, w, C, occ, X=None, S=None):
    """Dense grid RI-J (nukexc/coulomb.hpp:56-115).  Pass X (half inverse) or
    S (metric, solved by Cholesky).  Returns (J, c)."""
    pts = _f64(pts).reshape(-1, 3)
    nbf = len(b["n"])
    na = len(aux["n"])
    C = np.asarray(C, dtype=np.float64)
    nocc = C.shape[1]
    J = np.zeros(nbf * nbf)
    c = np.zeros(na)
    Xc = _f64(np.asarray(X).T).reshape(-1) if X is not None else None
    K = X.shape[1] if X is not None else 0
    Sc = _f64(np.asarray(S).T).reshape(-1) if S is not None else None
    rc = _lib().orc_coulomb(*_bargs(b), *_bargs(aux), len(pts), pts.reshape(-1), _f64(w), nocc,
                            _f64(C.T).reshape(-1), _f64(occ), _ptr(Xc), K, _ptr(Sc), J, _ptr(c))
    if rc != 0:
        raise RuntimeError("oracle Cholesky failed: metric not positive definite")
    return J.reshape(nbf, nbf).T.copy(), c


def exchange(b, aux, pts, w, C, occ, X):
    """Grid RI-K of the reference's dense path (nukexc/exact_exchange.hpp:57-119):
    T = C^T Phi; per orbital i, (P|mu i) = Vw (Phi o T_i)^T, Y_i = (P|mu i)^T X,
    K = sum_i occ_i Y_i Y_i^T (numpy, small cases)."""
    phi = collocation(b, pts)
    vw = potential_collocation(aux, pts, w)
    T = np.asarray(C).T @ phi
    K = np.zeros((phi.shape[0], phi.shape[0]))
    for i in range(T.shape[0]):
        three = vw @ (phi * T[i]).T
        Y = three.T @ X
        K += occ[i] * (Y @ Y.T)
    return K


def core_hamiltonian(b, centers, Z, pts, w):
    """compute_core_hamiltonian (nukexc/core_hamiltonian.hpp:133-289) by
    quadrature: S = sum w phi phi^T, T = 1/2 sum w grad phi . grad phi^T,
    V = -sum w (sum_A Z_A / (|r - R_A| + 1e-30)) phi phi^T (the shift of
    nukexc/nukexc_config.hpp:61).  Returns (S, T, V)."""
    pts = np.asarray(pts, float)
    w = np.asarray(w, float)
    phi, gx, gy, gz = collocation(b, pts, grad=True)
    v = np.zeros(len(w))
    for c, z in zip(np.asarray(centers, float), Z):
        v += float(z) / (np.linalg.norm(pts - c, axis=1) + 1e-30)
    S = (phi * w) @ phi.T
    T = 0.5 * ((gx * w) @ gx.T + (gy * w) @ gy.T + (gz * w) @ gz.T)
    V = -(phi * (w * v)) @ phi.T
    return S, T, V
