"""Python mirror of the NuKEXC hot-path interface over the C ABI.

Names and argument meanings follow the reference headers (grid.hpp,
partitioning.hpp, stobasis.hpp, density.hpp, xc_integrals.hpp,
coulomb.hpp, stopotential.hpp, nukexc_utils.hpp).  Device buffers are torch
CUDA tensors (torch is used only as a device allocator); every computation
runs in libnkx.so.  Matrices are returned in the reference's LayoutLeft
convention as torch tensors M with M[i, j] = element (i, j).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._lib import check

_FUNC_NAMES = {"LDA_X": 1, "LDA_C_VWN": 7, "LDA_C_PW": 12, "LDA_C_PW_MOD": 13, "GGA_X_PBE": 101, "GGA_C_PBE": 130}


def _dev(x, dtype=torch.float64):
    if isinstance(x, torch.Tensor):
        return x.to(device="cuda", dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _np(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ----------------------------------------------------------------- basis --
@dataclass
class STOBasisSet:
    """STOBasisSet (nukexc/stobasis.hpp:54-64): SoA host arrays."""
    n: np.ndarray
    l: np.ndarray
    m: np.ndarray
    zeta: np.ndarray
    center: np.ndarray  # (nbf, 3)
    cutoff_tol: float = 1e-10

    def nbf(self):
        return len(self.n)

    def as_c(self):
        self._keep = [_np(self.n, np.int32), _np(self.l, np.int32), _np(self.m, np.int32),
                      _np(self.zeta, np.float64), _np(self.center, np.float64).reshape(-1)]
        k = self._keep
        return L.Basis(len(self.n), *(a.ctypes.data_as(C.c_void_p) for a in k), self.cutoff_tol)


def make_manual_basis(funcs, cutoff_tol=1e-10):
    """make_manual_basis (nukexc/stobasis.hpp:175-225); funcs = (n,l,m,zeta,ox,oy,oz)."""
    f = list(funcs)
    return STOBasisSet(np.array([x[0] for x in f], np.int32), np.array([x[1] for x in f], np.int32),
                       np.array([x[2] for x in f], np.int32), np.array([x[3] for x in f], np.float64),
                       np.array([[x[4], x[5], x[6]] for x in f], np.float64).reshape(-1, 3), cutoff_tol)


# ------------------------------------------------------------------ grid --
@dataclass
class FlatGrid:
    """FlatGrid (nukexc/grid.hpp:150-160), host numpy arrays in bohr."""
    quad_points: np.ndarray  # (npts, 3)
    weights: np.ndarray
    atom_centers: np.ndarray
    Z: np.ndarray
    point_owner: np.ndarray


def _mol(centers, Z):
    c = _np(centers, np.float64).reshape(-1)
    z = _np(Z, np.int32)
    return L.Molecule(len(z), c.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p)), (c, z)


def make_flat_grid(centers, Z, nrad=50, nang_order=30, weight_threshold=1e-30, ta_alpha=0.6,
                   radial="ta", sizing="uniform", becke_clamp=5.0):
    """make_flat_grid (nukexc/grid.hpp:172-348)."""
    mol, keep = _mol(centers, Z)
    spec = L.GridSpec({"becke": L.RADIAL_BECKE, "ta": L.RADIAL_TA}[radial], nrad, nang_order,
                      weight_threshold, ta_alpha, {"uniform": 0, "pyscf": 1}[sizing], becke_clamp)
    n = C.c_long(0)
    check(L.lib().nkx_make_flat_grid(C.byref(mol), C.byref(spec), C.byref(n), None, None, None))
    xyz = np.zeros((n.value, 3))
    w = np.zeros(n.value)
    own = np.zeros(n.value, np.int32)
    check(L.lib().nkx_make_flat_grid(C.byref(mol), C.byref(spec), C.byref(n), xyz.ctypes.data_as(C.c_void_p),
                                     w.ctypes.data_as(C.c_void_p), own.ctypes.data_as(C.c_void_p)))
    return FlatGrid(xyz, w, np.asarray(centers, float).reshape(-1, 3), np.asarray(Z), own)


def partition_becke_team(atom_centers, quadrature_points, point_owner, weights, clamp=5.0):
    """partition_becke_team (nukexc/partitioning.hpp:126-213); returns new weights
    (a CUDA tensor).  clamp <= 0 gives partition_becke (:63-120)."""
    c = _dev(atom_centers).reshape(-1)
    p = _dev(quadrature_points).reshape(-1)
    o = _dev(point_owner, torch.int32)
    w = _dev(weights).clone()
    check(L.lib().nkx_becke_partition(_p(c), c.numel() // 3, _p(p), _p(o), w.numel(), _p(w), clamp, None))
    return w


def partition_becke(atom_centers, quadrature_points, point_owner, weights):
    return partition_becke_team(atom_centers, quadrature_points, point_owner, weights, clamp=0.0)


# ------------------------------------------------------------ collocation --
def _lmat(flat, rows, cols):
    """column-major flat buffer -> tensor M[i, j]"""
    return flat.view(cols, rows).t()


def fill_collocation(basis, points):
    """fill_collocation (nukexc/stobasis.hpp:494-532): Phi[nbf, npts]."""
    pts = _dev(points).reshape(-1)
    npts = pts.numel() // 3
    phi = torch.empty(basis.nbf() * npts, dtype=torch.float64, device="cuda")
    b = basis.as_c()
    check(L.lib().nkx_fill_collocation(C.byref(b), _p(pts), npts, _p(phi), None, None, None, None))
    return _lmat(phi, basis.nbf(), npts)


def fill_grad_collocation(basis, points):
    """fill_collocation + fill_grad_collocation (stobasis.hpp:494-584)."""
    pts = _dev(points).reshape(-1)
    npts = pts.numel() // 3
    bufs = [torch.empty(basis.nbf() * npts, dtype=torch.float64, device="cuda") for _ in range(4)]
    b = basis.as_c()
    check(L.lib().nkx_fill_collocation(C.byref(b), _p(pts), npts, *[_p(x) for x in bufs], None))
    return tuple(_lmat(x, basis.nbf(), npts) for x in bufs)


def _flat_lmat(M):
    """tensor M[i, j] -> column-major contiguous flat buffer"""
    return _dev(M).t().contiguous().reshape(-1)


# ---------------------------------------------------------------- density --
def compute_density_and_sigma(phi, gx, gy, gz, mo_orbitals, mo_coeff):
    """compute_density_and_sigma (nukexc/density.hpp:188-255): returns
    (rho, grad[3, npts], sigma) as CUDA tensors."""
    nbf, npts = phi.shape
    C_ = _flat_lmat(mo_orbitals)
    occ = _dev(mo_coeff)
    rho = torch.empty(npts, dtype=torch.float64, device="cuda")
    grad = torch.empty(3 * npts, dtype=torch.float64, device="cuda")
    sig = torch.empty(npts, dtype=torch.float64, device="cuda")
    fl = [_flat_lmat(x) for x in (phi, gx, gy, gz)]
    check(L.lib().nkx_density_dense(nbf, npts, *[_p(x) for x in fl], occ.numel(), _p(C_), _p(occ),
                                    _p(rho), _p(grad), _p(sig), None))
    return rho, grad.view(3, npts), sig


def compute_density(phi, mo_orbitals, mo_coeff):
    """compute_density (nukexc/density.hpp:150-186)."""
    nbf, npts = phi.shape
    C_ = _flat_lmat(mo_orbitals)
    occ = _dev(mo_coeff)
    rho = torch.empty(npts, dtype=torch.float64, device="cuda")
    f = _flat_lmat(phi)
    check(L.lib().nkx_density_dense(nbf, npts, _p(f), None, None, None, occ.numel(), _p(C_), _p(occ),
                                    _p(rho), None, None, None))
    return rho


# --------------------------------------------------------------------- XC --
def _opts(func_ids, dens_threshold=1e-15, metric_svd_thr=0.0, workspace_bytes=0):
    ids = [(_FUNC_NAMES[f] if isinstance(f, str) else int(f)) for f in func_ids]
    arr = (C.c_int * 4)(*(ids + [0] * (4 - len(ids))))
    return L.PlanOptions(256, 1e-10, len(ids), arr, dens_threshold, workspace_bytes, metric_svd_thr)


def _xc_dense(phi, grads, weights, C_list, occ_list, func_ids, dens_threshold):
    nbf, npts = phi.shape
    nspin = len(C_list)
    nocc = C_list[0].shape[1]
    Cc = torch.cat([_flat_lmat(c) for c in C_list])
    oc = torch.cat([_dev(o) for o in occ_list])
    fl = [_flat_lmat(phi)] + ([_flat_lmat(g) for g in grads] if grads else [None] * 3)
    w = _dev(weights)
    V = torch.empty(nspin * nbf * nbf, dtype=torch.float64, device="cuda")
    E = C.c_double(0)
    o = _opts(func_ids, dens_threshold)
    check(L.lib().nkx_xc_dense(nbf, npts, *[_p(x) for x in fl], _p(w), nspin, nocc, _p(Cc), _p(oc),
                               C.byref(o), C.byref(E), _p(V), None))
    Vs = [V[s * nbf * nbf:(s + 1) * nbf * nbf].view(nbf, nbf).t() for s in range(nspin)]
    return E.value, Vs


def compute_lda(phi, weights, mo_orbitals, mo_coeff, func_ids=("LDA_X",), dens_threshold=1e-15):
    """compute_lda (nukexc/xc_integrals.hpp:73-166): (E_xc, V)."""
    E, V = _xc_dense(phi, None, weights, [mo_orbitals], [mo_coeff], func_ids, dens_threshold)
    return E, V[0]


def compute_gga(phi, gx, gy, gz, weights, mo_orbitals, mo_coeff, func_ids=("GGA_X_PBE",),
                dens_threshold=1e-15):
    """compute_gga (nukexc/xc_integrals.hpp:424-541): (E_xc, V)."""
    E, V = _xc_dense(phi, (gx, gy, gz), weights, [mo_orbitals], [mo_coeff], func_ids, dens_threshold)
    return E, V[0]


def compute_lsda(phi, weights, mo_alpha, occ_alpha, mo_beta, occ_beta, func_ids=("LDA_X",),
                 dens_threshold=1e-15):
    """compute_lsda (nukexc/xc_integrals.hpp:168-261): (E_xc, V_alpha, V_beta)."""
    E, V = _xc_dense(phi, None, weights, [mo_alpha, mo_beta], [occ_alpha, occ_beta], func_ids, dens_threshold)
    return E, V[0], V[1]


def compute_gga_lsda(phi, gx, gy, gz, weights, mo_alpha, occ_alpha, mo_beta, occ_beta,
                     func_ids=("GGA_X_PBE",), dens_threshold=1e-15):
    """compute_gga_lsda (nukexc/xc_integrals.hpp:543-726)."""
    E, V = _xc_dense(phi, (gx, gy, gz), weights, [mo_alpha, mo_beta], [occ_alpha, occ_beta], func_ids,
                     dens_threshold)
    return E, V[0], V[1]


def xc_eval(func_id, nspin, rho, sigma=None, dens_threshold=1e-15):
    """libxc-layout functional evaluation on the device: (exc, vrho, vsigma)."""
    fid = _FUNC_NAMES[func_id] if isinstance(func_id, str) else int(func_id)
    r = _dev(rho)
    n = r.numel() // nspin
    s = _dev(sigma) if sigma is not None else None
    exc = torch.empty(n, dtype=torch.float64, device="cuda")
    vr = torch.empty(n * nspin, dtype=torch.float64, device="cuda")
    vs = torch.empty(n * (1 if nspin == 1 else 3), dtype=torch.float64, device="cuda") if s is not None else None
    check(L.lib().nkx_xc_eval(fid, nspin, n, _p(r), _p(s), dens_threshold, _p(exc), _p(vr), _p(vs), None))
    return exc, vr, vs


# ---------------------------------------------------------------- Coulomb --
def sto_potential_collocation_scaled(basis_aux, points, weights):
    """sto_potential_collocation_scaled (nukexc/stopotential.hpp:101-124)."""
    pts = _dev(points).reshape(-1)
    npts = pts.numel() // 3
    w = _dev(weights)
    out = torch.empty(basis_aux.nbf() * npts, dtype=torch.float64, device="cuda")
    b = basis_aux.as_c()
    check(L.lib().nkx_potential_collocation(C.byref(b), _p(pts), _p(w), npts, _p(out), None))
    return _lmat(out, basis_aux.nbf(), npts)


def compute_half_inverse(S, lin_dep_threshold=1e-5):
    """compute_half_inverse (nukexc/nukexc_utils.hpp:198-270): X (N x K)."""
    N = S.shape[0]
    Sf = _flat_lmat(S)
    X = torch.empty(N * N, dtype=torch.float64, device="cuda")
    K = C.c_int(0)
    check(L.lib().nkx_half_inverse(N, _p(Sf), lin_dep_threshold, _p(X), C.byref(K), None))
    return _lmat(X, N, N)[:, :K.value]


def compute_coulomb(mo_orbitals, mo_coeff, basis_collocation, basis_aux_collocation,
                    potential_collocation_scaled, half_inverse_X):
    """compute_coulomb (nukexc/coulomb.hpp:56-115), dense, through
    nkx_coulomb_dense: J (nbf x nbf) from rho, y = Vw rho, c = X X^T y,
    v = Vw^T c and J = Phi diag(v) Phi^T."""
    nbf, npts = basis_collocation.shape
    naux, K = half_inverse_X.shape
    f = _flat_lmat(basis_collocation)
    Vw = _flat_lmat(potential_collocation_scaled)
    X = _flat_lmat(half_inverse_X)
    C_ = _flat_lmat(mo_orbitals)
    occ = _dev(mo_coeff)
    J = torch.empty(nbf * nbf, dtype=torch.float64, device="cuda")
    check(L.lib().nkx_coulomb_dense(nbf, naux, npts, _p(f), _p(Vw), _p(X), K, occ.numel(), _p(C_), _p(occ),
                                    _p(J), None))
    J = J.view(nbf, nbf).t()
    return J


def compute_exact_exchange(mo_orbitals, mo_coeff, basis_collocation, basis_aux_collocation,
                           potential_collocation_scaled, half_inverse_X):
    """compute_exact_exchange (nukexc/exact_exchange.hpp:57-119), the dense
    grid RI-K, through nkx_exchange_dense: K = sum_i occ_i Y_i Y_i^T with
    Y_i = ((Vw (Phi o T_i)^T)^T X) and T = C^T Phi."""
    nbf, npts = basis_collocation.shape
    naux, K = half_inverse_X.shape
    f = _flat_lmat(basis_collocation)
    Vw = _flat_lmat(potential_collocation_scaled)
    X = _flat_lmat(half_inverse_X)
    C_ = _flat_lmat(mo_orbitals)
    occ = _dev(mo_coeff)
    Km = torch.empty(nbf * nbf, dtype=torch.float64, device="cuda")
    check(L.lib().nkx_exchange_dense(nbf, naux, npts, _p(f), _p(Vw), _p(X), K, occ.numel(), _p(C_), _p(occ),
                                     _p(Km), None))
    return Km.view(nbf, nbf).t()


def compute_core_hamiltonian(basis, centers, Z, points, weights):
    """compute_core_hamiltonian (nukexc/core_hamiltonian.hpp:133-289) by
    quadrature: (S, T, V_nuc, H = T + V_nuc) as nbf x nbf CUDA tensors."""
    pts = _dev(points).reshape(-1)
    w = _dev(weights)
    n = basis.nbf()
    out = [torch.empty(n * n, dtype=torch.float64, device="cuda") for _ in range(3)]
    mol, keep = _mol(centers, Z)
    b = basis.as_c()
    check(L.lib().nkx_core_hamiltonian_dense(C.byref(b), C.byref(mol), _p(pts), _p(w), w.numel(),
                                             *[_p(o) for o in out], None))
    S, T, V = (o.view(n, n).t() for o in out)
    return S, T, V, T + V


# ------------------------------------------------------------------ plan --
class FockBuilder:
    """The batched grid-integration Fock build behind nkx_plan_* (the hot
    path): once per geometry the grid is batched and screened and the aux
    metric factorised; each build() is one SCF iteration's XC (+ J) work.

    grid: FlatGrid or (points, weights) or (points, weights, point_owner);
    basis/aux: STOBasisSet.  The point owners (given by a FlatGrid or the
    3-tuple) are needed only by xc_gradient.
    """

    def __init__(self, centers, Z, basis, grid, aux=None, func_ids=("GGA_X_PBE", "GGA_C_PBE"),
                 dens_threshold=1e-15, metric_svd_thr=0.0, workspace_bytes=0):
        owner = None
        if isinstance(grid, FlatGrid):
            pts, w, owner = grid.quad_points, grid.weights, grid.point_owner
        elif len(grid) == 3:
            pts, w, owner = grid
        else:
            pts, w = grid
        self._pts = _np(pts, np.float64).reshape(-1)
        self._w = _np(w, np.float64)
        self._owner = _np(owner, np.int32) if owner is not None else None
        mol, self._mk = _mol(centers, Z)
        self.basis = basis
        self._b = basis.as_c()
        self._a = aux.as_c() if aux is not None else None
        self._o = _opts(func_ids, dens_threshold, metric_svd_thr, workspace_bytes)
        self.nbf = basis.nbf()
        self.naux = aux.nbf() if aux is not None else 0
        h = C.c_void_p()
        check(L.lib().nkx_plan_create(C.byref(mol), C.byref(self._b), C.byref(self._a) if self._a else None,
                                      len(self._w), self._pts.ctypes.data_as(C.c_void_p),
                                      self._w.ctypes.data_as(C.c_void_p),
                                      self._owner.ctypes.data_as(C.c_void_p) if self._owner is not None else None,
                                      C.byref(self._o), C.byref(h)))
        self._h = h

    def info(self):
        i = L.PlanInfo()
        check(L.lib().nkx_plan_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in L.PlanInfo._fields_}

    def timing(self):
        t = L.BuildTiming()
        check(L.lib().nkx_get_last_timing(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in L.BuildTiming._fields_}

    def build(self, C_list, occ_list, precision="fp64", want_J=False, fuse_j=False, stream=None, want_V=True,
              out_V=None):
        """One Fock build.  C_list/occ_list: one (nbf x nocc, nocc) per spin,
        numpy or CPU tensors (host: copied inside the call) or CUDA tensors
        (device).  Returns (E_xc, [V per spin], J or None); with fuse_j, V
        includes J.  want_V=False (with want_J) returns J alone: (E_xc, None, J).
        Host builds with page-locked buffers copy at full PCIe / C2C speed: a
        single spin's C as a pinned CPU tensor stored column-major (C.t()
        contiguous) and occ as a pinned CPU tensor are passed as they are, and
        out_V, a pinned CPU tensor of nspin * nbf^2 doubles, receives V (the
        returned matrices are views of it)."""
        if not want_V and not (want_J and not fuse_j):
            raise ValueError("want_V=False needs want_J=True and fuse_j=False")
        nspin = len(C_list)
        host = not (isinstance(C_list[0], torch.Tensor) and C_list[0].is_cuda)
        nocc = C_list[0].shape[1]
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        nn = self.nbf * self.nbf
        if host and isinstance(C_list[0], torch.Tensor):
            # CPU tensors: used in place when already in the C-ABI's layout
            if nspin == 1 and C_list[0].dtype == torch.float64 and C_list[0].t().is_contiguous():
                Cc = C_list[0]
            else:
                Cc = torch.cat([c.to(torch.float64).t().contiguous().reshape(-1) for c in C_list])
            oc = occ_list[0] if nspin == 1 and occ_list[0].dtype == torch.float64 and occ_list[0].is_contiguous() \
                else torch.cat([o.to(torch.float64).reshape(-1) for o in occ_list])
            if out_V is not None and want_V:
                if out_V.dtype != torch.float64 or out_V.numel() != nspin * nn or not out_V.is_contiguous():
                    raise ValueError("out_V must be a contiguous float64 CPU tensor of nspin * nbf^2 elements")
                V = out_V.reshape(-1).numpy()
            else:
                V = np.empty(nspin * nn) if want_V else None
            J = np.empty(nn) if want_J and not fuse_j else None
            pC, po = C.c_void_p(Cc.data_ptr()), C.c_void_p(oc.data_ptr())
            pV, pJ = (a.ctypes.data_as(C.c_void_p) if a is not None else None for a in (V, J))
        elif host:
            Cc = np.concatenate([np.ascontiguousarray(np.asarray(c, np.float64).T).reshape(-1) for c in C_list])
            oc = np.concatenate([_np(o, np.float64) for o in occ_list])
            V = np.empty(nspin * nn) if want_V else None
            J = np.empty(nn) if want_J and not fuse_j else None
            pC, po, pV, pJ = (a.ctypes.data_as(C.c_void_p) if a is not None else None for a in (Cc, oc, V, J))
        else:
            Cc = torch.cat([c.t().contiguous().reshape(-1) for c in C_list])
            oc = torch.cat([o.reshape(-1) for o in occ_list]).to(torch.float64)
            V = torch.empty(nspin * nn, dtype=torch.float64, device="cuda") if want_V else None
            J = torch.empty(nn, dtype=torch.float64, device="cuda") if want_J and not fuse_j else None
            pC, po, pV, pJ = _p(Cc), _p(oc), _p(V), _p(J)
        E = C.c_double(0)
        s = C.c_void_p(stream) if stream else None
        check(L.lib().nkx_fock_build(self._h, prec, nspin, nocc, pC, po, L.MEM_HOST if host else L.MEM_DEVICE,
                                     1 if fuse_j else 0, C.byref(E), pV, pJ, s))
        if V is None:
            Vs = None
            Jm = J.reshape(self.nbf, self.nbf) if host else J.view(self.nbf, self.nbf).t()
        elif host:
            # V and J are symmetric, so the column-major buffers read row-major
            # are the matrices themselves (no transposing copy)
            Vs = [V[k * nn:(k + 1) * nn].reshape(self.nbf, self.nbf) for k in range(nspin)]
            Jm = J.reshape(self.nbf, self.nbf) if J is not None else None
        else:
            Vs = [V[k * nn:(k + 1) * nn].view(self.nbf, self.nbf).t() for k in range(nspin)]
            Jm = J.view(self.nbf, self.nbf).t() if J is not None else None
        return E.value, Vs, Jm

    def xc_gradient(self, C_list, occ_list, becke_clamp=5.0, stream=None, precision="fp64"):
        """dE_xc/dR (natoms x 3, Eh/bohr) at fixed orbitals, with the grid
        points moving with their owner atoms and the Becke weights
        differentiated (nkx_xc_gradient).  precision "mixed" takes the
        orbital values and the density from the int8-digit tensor-core
        contraction; the rest is FP64."""
        nspin = len(C_list)
        nocc = C_list[0].shape[1]
        Cc = np.concatenate([np.ascontiguousarray(np.asarray(c, np.float64).T).reshape(-1) for c in C_list])
        oc = np.concatenate([_np(o, np.float64) for o in occ_list])
        natoms = len(self._mk[0]) // 3
        g = np.zeros(3 * natoms)
        s = C.c_void_p(stream) if stream else None
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        check(L.lib().nkx_xc_gradient(self._h, prec, nspin, nocc, Cc.ctypes.data_as(C.c_void_p),
                                      oc.ctypes.data_as(C.c_void_p), L.MEM_HOST, becke_clamp,
                                      g.ctypes.data_as(C.c_void_p), s))
        return g.reshape(natoms, 3)

    def density(self, C_list, occ_list, grad=False, stream=None):
        """rho (nspin x npts) on the plan's grid in the caller's point order,
        FP64 (compute_density_sparse / compute_density_and_sigma_sparse,
        nukexc/density.hpp:97-148, :261-328; nkx_plan_density).  With grad,
        also grad rho (nspin x 3 x npts) and sigma = |grad rho|^2 (nspin x npts)."""
        nspin = len(C_list)
        nocc = C_list[0].shape[1]
        n = self.info()["npoints"]
        Cc = np.concatenate([np.ascontiguousarray(np.asarray(c, np.float64).T).reshape(-1) for c in C_list])
        oc = np.concatenate([_np(o, np.float64) for o in occ_list])
        rho = np.zeros(nspin * n)
        g = np.zeros(3 * nspin * n) if grad else None
        sg = np.zeros(nspin * n) if grad else None
        s = C.c_void_p(stream) if stream else None
        ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None  # noqa: E731
        check(L.lib().nkx_plan_density(self._h, nspin, nocc, ptr(Cc), ptr(oc), L.MEM_HOST, 0, ptr(rho), ptr(g),
                                       ptr(sg), s))
        if grad:
            return rho.reshape(nspin, n), g.reshape(nspin, 3, n), sg.reshape(nspin, n)
        return rho.reshape(nspin, n)

    def set_wait_limit(self, ns=0, stall=False):
        """Limit of the tensor-core kernels' device waits in ns (0: default,
        2 s); stall=True makes the following mixed builds give up after it
        (a test of the NKX_ERR_TIMEOUT path; nkx_plan_set_wait_limit)."""
        check(L.lib().nkx_plan_set_wait_limit(self._h, int(ns), 1 if stall else 0))

    def set_functional(self, func_ids, dens_threshold=1e-15):
        """Evaluate these functionals in the following builds (nkx_plan_set_functional)."""
        ids = [_FUNC_NAMES.get(f, f) for f in func_ids]
        arr = (C.c_int * len(ids))(*ids)
        check(L.lib().nkx_plan_set_functional(self._h, len(ids), arr, dens_threshold))

    def set_half_inverse(self, X):
        """Fit J with the caller's half inverse X (naux x K): c = X X^T y
        (compute_coulomb_sparse's half_inverse_X; nkx_plan_set_half_inverse)."""
        Xa = np.asarray(X, np.float64)
        assert Xa.shape[0] == self.naux, "X must be naux x K"
        col = np.ascontiguousarray(Xa.T).reshape(-1)
        check(L.lib().nkx_plan_set_half_inverse(self._h, Xa.shape[1], col.ctypes.data_as(C.c_void_p), L.MEM_HOST))

    def aux_metric(self):
        """The plan's symmetrised grid Coulomb metric (A|B), naux x naux."""
        S = np.zeros(self.naux * self.naux)
        check(L.lib().nkx_plan_aux_metric(self._h, S.ctypes.data_as(C.c_void_p), L.MEM_HOST))
        return S.reshape(self.naux, self.naux).T.copy()

    def autotune(self, C_list, occ_list, cache_path=None, stream=None):
        """Time the mixed build's knobs on these orbitals and keep the fastest
        (nkx_plan_autotune); returns the choices and timings as a dict."""
        nspin = len(C_list)
        host = not isinstance(C_list[0], torch.Tensor)
        nocc = C_list[0].shape[1]
        if host:
            Cc = np.concatenate([np.ascontiguousarray(np.asarray(c, np.float64).T).reshape(-1) for c in C_list])
            oc = np.concatenate([_np(o, np.float64) for o in occ_list])
            pC, po = Cc.ctypes.data_as(C.c_void_p), oc.ctypes.data_as(C.c_void_p)
        else:
            Cc = torch.cat([c.t().contiguous().reshape(-1) for c in C_list])
            oc = torch.cat([o.reshape(-1) for o in occ_list]).to(torch.float64)
            pC, po = _p(Cc), _p(oc)
        t = L.Tuning()
        s = C.c_void_p(stream) if stream else None
        check(L.lib().nkx_plan_autotune(self._h, nspin, nocc, pC, po, L.MEM_HOST if host else L.MEM_DEVICE,
                                        cache_path.encode() if cache_path else None, C.byref(t), s))
        return {k: getattr(t, k) for k, _ in L.Tuning._fields_}

    def tuning(self):
        t = L.Tuning()
        check(L.lib().nkx_plan_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in L.Tuning._fields_
                if k in ("v_n", "dens_n", "ypath", "v_warps", "v_pair", "chunk_pairs")}

    def set_tuning(self, v_n=128, dens_n=0, ypath=-1, chunk_pairs=0, v_warps=16, v_pair=0):
        t = L.Tuning(v_n=v_n, dens_n=dens_n, ypath=ypath, v_warps=v_warps, v_pair=v_pair, chunk_pairs=chunk_pairs)
        check(L.lib().nkx_plan_set_tuning(self._h, C.byref(t)))

    def core_hamiltonian(self, centers, Z):
        """S, T, V_n by quadrature over the plan's screened batches (the
        reference's compute_core_hamiltonian_screened family;
        nkx_plan_core_hamiltonian), FP64 numpy matrices."""
        mol, keep = _mol(centers, Z)
        n = self.nbf * self.nbf
        S, T, V = np.empty(n), np.empty(n), np.empty(n)
        check(L.lib().nkx_plan_core_hamiltonian(self._h, C.byref(mol), S.ctypes.data_as(C.c_void_p),
                                                T.ctypes.data_as(C.c_void_p), V.ctypes.data_as(C.c_void_p),
                                                L.MEM_HOST, None))
        return tuple(M.reshape(self.nbf, self.nbf) for M in (S, T, V))

    def set_graph(self, enable=True):
        """Replay device-buffer builds from a CUDA graph (nkx_plan_set_graph)."""
        check(L.lib().nkx_plan_set_graph(self._h, 1 if enable else 0))

    def set_metric(self, S):
        """Replace the plan's Coulomb metric (A|B) (naux x naux) and factor it
        again (nkx_plan_set_metric); for a sharded grid, the sum over ranks of
        aux_metric()."""
        Sa = np.asarray(S, np.float64)
        assert Sa.shape == (self.naux, self.naux), "S must be naux x naux"
        col = np.ascontiguousarray(Sa.T).reshape(-1)
        check(L.lib().nkx_plan_set_metric(self._h, col.ctypes.data_as(C.c_void_p), L.MEM_HOST))

    def build_phase1(self, C_list, occ_list, precision="fp64", stream=None):
        """First half of a build on a sharded grid (nkx_fock_build_phase1):
        the density pass and this plan's share of the J fit vector y
        (naux; numpy for host orbitals, a CUDA tensor for device ones)."""
        nspin = len(C_list)
        host = not isinstance(C_list[0], torch.Tensor)
        nocc = C_list[0].shape[1]
        prec = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}[precision]
        if host:
            Cc = np.concatenate([np.ascontiguousarray(np.asarray(c, np.float64).T).reshape(-1) for c in C_list])
            oc = np.concatenate([_np(o, np.float64) for o in occ_list])
            y = np.empty(self.naux)
            pC, po, py = (a.ctypes.data_as(C.c_void_p) for a in (Cc, oc, y))
        else:
            Cc = torch.cat([c.t().contiguous().reshape(-1) for c in C_list])
            oc = torch.cat([o.reshape(-1) for o in occ_list]).to(torch.float64)
            y = torch.empty(self.naux, dtype=torch.float64, device="cuda")
            pC, po, py = _p(Cc), _p(oc), _p(y)
        s = C.c_void_p(stream) if stream else None
        check(L.lib().nkx_fock_build_phase1(self._h, prec, nspin, nocc, pC, po, L.MEM_HOST if host else L.MEM_DEVICE,
                                            py, s))
        self._phase_nspin = nspin
        return y

    def build_phase2(self, y_total, want_J=False, fuse_j=False, stream=None):
        """Second half (nkx_fock_build_phase2) with the fit vector summed over
        the ranks; returns this plan's partial (E_xc, [V per spin], J or None)
        like build(); host or device outputs follow y_total."""
        nspin = self._phase_nspin
        host = not isinstance(y_total, torch.Tensor)
        nn = self.nbf * self.nbf
        if host:
            yv = _np(y_total, np.float64)
            V = np.empty(nspin * nn)
            J = np.empty(nn) if want_J and not fuse_j else None
            py, pV, pJ = (a.ctypes.data_as(C.c_void_p) if a is not None else None for a in (yv, V, J))
        else:
            yv = y_total.to(torch.float64).contiguous()
            V = torch.empty(nspin * nn, dtype=torch.float64, device="cuda")
            J = torch.empty(nn, dtype=torch.float64, device="cuda") if want_J and not fuse_j else None
            py, pV, pJ = _p(yv), _p(V), _p(J)
        E = C.c_double(0)
        s = C.c_void_p(stream) if stream else None
        check(L.lib().nkx_fock_build_phase2(self._h, py, L.MEM_HOST if host else L.MEM_DEVICE, 1 if fuse_j else 0,
                                            C.byref(E), pV, pJ, s))
        if host:
            Vs = [V[k * nn:(k + 1) * nn].reshape(self.nbf, self.nbf) for k in range(nspin)]
            Jm = J.reshape(self.nbf, self.nbf) if J is not None else None
        else:
            Vs = [V[k * nn:(k + 1) * nn].view(self.nbf, self.nbf).t() for k in range(nspin)]
            Jm = J.view(self.nbf, self.nbf).t() if J is not None else None
        return E.value, Vs, Jm

    def batch_blocks(self):
        """Significant 128-function blocks per batch."""
        n = self.info()["nbatches"]
        out = np.zeros(n, np.int32)
        check(L.lib().nkx_plan_batch_blocks(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def last_density(self, nspin=1):
        npts = self.info()["npoints"]
        rho = np.zeros(npts * nspin)
        perm = np.zeros(npts, np.int64)
        check(L.lib().nkx_plan_last_density(self._h, rho.ctypes.data_as(C.c_void_p),
                                            perm.ctypes.data_as(C.c_void_p)))
        out = np.zeros((npts, nspin))
        out[perm] = rho.reshape(npts, nspin)
        return out

    def close(self):
        if getattr(self, "_h", None):
            L.lib().nkx_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------ sparse set-up ----
def cutoff_radii(basis):
    """Per function, the largest r with N r^(n-1) e^(-zeta r) >= cutoff_tol
    (the reference's cutoff radius, nukexc/stobasis.hpp:203-222), by bisection
    on the decreasing tail beyond the maximum at r = (n-1)/zeta."""
    from math import lgamma, log
    out = np.zeros(basis.nbf())
    lt = log(basis.cutoff_tol)
    for i, (n, z) in enumerate(zip(basis.n, basis.zeta)):
        n, z = int(n), float(z)
        lnN = (n + 0.5) * log(2.0 * z) - 0.5 * lgamma(2.0 * n + 1.0)
        g = lambda r: lnN + (n - 1) * log(max(r, 1e-300)) - z * r  # noqa: E731
        lo = (n - 1) / z
        hi = lo + 1.0
        while g(hi) > lt:
            hi *= 2.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if g(mid) > lt:
                lo = mid
            else:
                hi = mid
        out[i] = hi
    return out


@dataclass
class NeighborList:
    """NeighborList (nukexc/octree.hpp:279-285): CSR of the basis functions
    meeting each box, ascending per box (CUDA int32 tensors)."""
    neighbors: torch.Tensor
    offsets: torch.Tensor
    max_points_per_box: int
    total_points: int


def create_bounding_boxes(grid, max_points_per_bb):
    """create_bounding_boxes (nukexc/octree.hpp:70-144): permutes
    grid.quad_points, grid.weights and grid.point_owner in place into Morton
    order (nkx_morton_order) and returns the bounds of each run of
    max_points_per_bb consecutive points as a CUDA tensor (nboxes, 2, 3) of
    (min corner, max corner)."""
    if max_points_per_bb <= 0:
        raise ValueError("max_points_per_bb must be positive")
    pts = _np(grid.quad_points, np.float64).reshape(-1, 3)
    G = len(pts)
    perm = np.zeros(G, np.int64)
    check(L.lib().nkx_morton_order(G, pts.ctypes.data_as(C.c_void_p), perm.ctypes.data_as(C.c_void_p)))
    sp = pts[perm]  # a copy: pts may be the grid's own array
    grid.quad_points[...] = sp.reshape(np.shape(grid.quad_points))
    grid.weights[...] = np.asarray(grid.weights)[perm]
    if grid.point_owner is not None and len(grid.point_owner) == G:
        grid.point_owner[...] = np.asarray(grid.point_owner)[perm]
    starts = np.arange(0, G, max_points_per_bb)
    boxes = np.stack([np.minimum.reduceat(sp, starts, axis=0), np.maximum.reduceat(sp, starts, axis=0)], 1)
    return _dev(boxes)


def build_neighbor_list(basis, bounding_boxes, max_points_per_box, total_points):
    """build_neighbor_list (nukexc/octree.hpp:317-390): functions whose
    cutoff sphere meets each box (nkx_neighbor_list, on the device)."""
    boxes = _dev(bounding_boxes).reshape(-1, 6)
    nb = boxes.shape[0]
    centers = _dev(basis.center)
    radii = _dev(cutoff_radii(basis))
    offsets = torch.zeros(nb + 1, dtype=torch.int32, device="cuda")
    nnz = C.c_long(0)
    check(L.lib().nkx_neighbor_list(basis.nbf(), _p(centers), _p(radii), nb, _p(boxes), _p(offsets), None,
                                    C.byref(nnz), None))
    neighbors = torch.zeros(max(1, nnz.value), dtype=torch.int32, device="cuda")
    if nnz.value:
        check(L.lib().nkx_neighbor_list(basis.nbf(), _p(centers), _p(radii), nb, _p(boxes), _p(offsets),
                                        _p(neighbors), C.byref(nnz), None))
    return NeighborList(neighbors[:nnz.value], offsets, max_points_per_box, total_points)


def coulomb_overlap_integral(basis_aux, points, weights):
    """Symmetrised grid Coulomb metric (A|B) of an aux basis
    (coulomb_overlap_integral_sparse / _tiled, nukexc/coulomb.hpp:691-958;
    nkx_aux_metric), as a CUDA tensor naux x naux."""
    pts = _dev(points).reshape(-1)
    w = _dev(weights)
    na = basis_aux.nbf()
    S = torch.zeros(na * na, dtype=torch.float64, device="cuda")
    b = basis_aux.as_c()
    check(L.lib().nkx_aux_metric(C.byref(b), len(w), _p(pts), _p(w), _p(S), None))
    return S.view(na, na).t()
