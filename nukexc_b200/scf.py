"""Stand-in closed-shell Kohn-Sham SCF around the Fock build.

The reference's driver (tests/standalone.cxx:572-846) diagonalises
F = H_core + J + V_xc in the metric S every iteration, where H_core and S
come by quadrature (core_hamiltonian.hpp:133-289), J from the grid
density fit (coulomb.hpp:56-115) and V_xc from the XC build.  This loop does
the same with DIIS extrapolation (error F P S - S P F) and a core-Hamiltonian
guess, so the Fock build can be run to SCF convergence; the Fock builds
themselves (`fock` callables) are supplied by the caller: `gpu_fock` uses
the plan (nkx_fock_build), the tests supply a CPU one from the oracle.
"""
from __future__ import annotations

import time

import numpy as np
import scipy.linalg as sla


def nuclear_repulsion(centers, Z):
    c = np.asarray(centers, float)
    z = np.asarray(Z, float)
    e = 0.0
    for a in range(len(z)):
        for b in range(a):
            e += z[a] * z[b] / np.linalg.norm(c[a] - c[b])
    return e


def rks(S, H, fock, nocc, e_nuc, conv=1e-8, maxiter=60, ndiis=8):
    """Closed-shell SCF.  fock(C_occ) -> (E_xc, V_xc, J) for orbitals C_occ
    (nbf x nocc, occupation 2).  Returns a dict with the total energy, the
    per-iteration energies and times, and the converged orbitals."""
    S = np.asarray(S, float)
    H = np.asarray(H, float)
    eps, C = sla.eigh(H, S)
    Cocc = C[:, :nocc]
    focks, errs, energies, times = [], [], [], []
    E_old = None
    converged = False
    for it in range(maxiter):
        t0 = time.perf_counter()
        E_xc, Vxc, J = fock(Cocc)
        P = 2.0 * Cocc @ Cocc.T
        F = H + J + Vxc
        E = float(np.sum(P * H) + 0.5 * np.sum(P * J) + E_xc + e_nuc)
        err = F @ P @ S - S @ P @ F
        focks.append(F)
        errs.append(err)
        focks, errs = focks[-ndiis:], errs[-ndiis:]
        if len(focks) > 1:
            n = len(focks)
            B = -np.ones((n + 1, n + 1))
            B[n, n] = 0.0
            for i in range(n):
                for j in range(n):
                    B[i, j] = np.sum(errs[i] * errs[j])
            rhs = np.zeros(n + 1)
            rhs[n] = -1.0
            try:
                coef = np.linalg.solve(B, rhs)[:n]
                F = sum(c * f for c, f in zip(coef, focks))
            except np.linalg.LinAlgError:
                pass
        eps, C = sla.eigh(F, S)
        Cocc = C[:, :nocc]
        times.append(time.perf_counter() - t0)
        energies.append(E)
        if E_old is not None and abs(E - E_old) < conv and np.abs(err).max() < 1e-5:
            converged = True
            break
        E_old = E
    return {"energy": energies[-1], "energies": energies, "iterations": len(energies), "converged": converged,
            "seconds_per_iteration": times, "C_occ": Cocc, "orbital_energies": eps}


def gpu_fock(fb, precision="fp64"):
    """fock callable over a FockBuilder with an aux basis (XC + separate J)."""
    def fock(Cocc):
        E, V, J = fb.build([np.ascontiguousarray(Cocc)], [2.0 * np.ones(Cocc.shape[1])], precision=precision,
                           want_J=True)
        return E, np.asarray(V[0]), np.asarray(J)
    return fock


def rks_device(S, H, fb, nocc, e_nuc, precision="fp64", conv=1e-8, maxiter=60, ndiis=8):
    """The closed-shell SCF of `rks` with every matrix on the GPU: S, H, the
    orbitals, the density and the Fock matrices stay in device memory
    (torch, FP64), the Fock builds take and return device buffers
    (nkx_fock_build with NKX_MEM_DEVICE), and the generalised eigenproblem is
    solved in the orthogonal basis X = S^-1/2 (symmetric orthogonalisation).
    Only the energy and the convergence test cross to the host each
    iteration -- the glue of the reference's driver (tests/standalone.cxx:590-646,
    :815-846) copies C and the matrices between Armadillo and the device
    every iteration instead.  fb is a FockBuilder with an aux basis."""
    import torch

    dev = "cuda"
    S = torch.as_tensor(S, dtype=torch.float64, device=dev).contiguous()
    H = torch.as_tensor(H, dtype=torch.float64, device=dev).contiguous()
    s, U = torch.linalg.eigh(S)
    X = U @ torch.diag(s.rsqrt()) @ U.t()

    def orbitals(F):
        e, Cp = torch.linalg.eigh(X.t() @ F @ X)
        return e, (X @ Cp)[:, :nocc].contiguous()

    eps, Cocc = orbitals(H)
    occ = torch.full((nocc,), 2.0, dtype=torch.float64, device=dev)
    focks, errs, energies, times = [], [], [], []
    E_old = None
    converged = False
    for it in range(maxiter):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E_xc, V, J = fb.build([Cocc], [occ], precision=precision, want_J=True)
        P = 2.0 * Cocc @ Cocc.t()
        F = H + J + V[0]
        E = float((P * H).sum() + 0.5 * (P * J).sum()) + E_xc + e_nuc
        err = F @ P @ S - S @ P @ F
        focks.append(F)
        errs.append(err)
        focks, errs = focks[-ndiis:], errs[-ndiis:]
        if len(focks) > 1:
            n = len(focks)
            B = -torch.ones((n + 1, n + 1), dtype=torch.float64, device=dev)
            B[n, n] = 0.0
            for i in range(n):
                for j in range(n):
                    B[i, j] = (errs[i] * errs[j]).sum()
            rhs = torch.zeros(n + 1, dtype=torch.float64, device=dev)
            rhs[n] = -1.0
            try:
                coef = torch.linalg.solve(B, rhs)[:n]
                F = sum(c * f for c, f in zip(coef, focks))
            except RuntimeError:
                pass
        eps, Cocc = orbitals(F)
        err_max = float(err.abs().max())
        times.append(time.perf_counter() - t0)
        energies.append(E)
        if E_old is not None and abs(E - E_old) < conv and err_max < 1e-5:
            converged = True
            break
        E_old = E
    return {"energy": energies[-1], "energies": energies, "iterations": len(energies), "converged": converged,
            "seconds_per_iteration": times, "C_occ": Cocc, "orbital_energies": eps}
