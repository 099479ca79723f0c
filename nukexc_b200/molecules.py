"""Synthetic molecules and even-tempered STO basis sets for the benchmark
workloads (seeded, deterministic).

Geometries are in bohr.  A basis is a list of STO functions
``(n, l, m, zeta, ox, oy, oz)`` in the order of the reference's
``make_manual_basis`` / ``load_adf_basis`` (nukexc/stobasis.hpp:175-292):
per atom, per shell, m = -l..l.
"""
from __future__ import annotations

import math

import numpy as np

ANG_TO_BOHR = 1.8897259885681697  # nukexc/atomic_properties.hpp:49

# Single water: O-H 0.9572 Angstrom, H-O-H 104.52 degrees
_OH = 0.9572
_HOH = math.radians(104.52)


def water():
    """One H2O, O at the origin, molecule in the xz plane (bohr)."""
    h = _OH * ANG_TO_BOHR
    a = _HOH / 2
    c = np.array([[0.0, 0.0, 0.0],
                  [h * math.sin(a), 0.0, h * math.cos(a)],
                  [-h * math.sin(a), 0.0, h * math.cos(a)]])
    return c, [8, 1, 1]


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def water_cluster(n, seed=0, spacing=3.0, jitter=0.3):
    """(H2O)_n: rigid waters, uniformly random orientations, centred on the
    first n sites of a ceil(n^(1/3))^3 cubic lattice of the given spacing
    (Angstrom), each molecule shifted by U(-jitter, jitter) Angstrom per
    coordinate.  Sites are taken in x-fastest lattice order."""
    rng = np.random.default_rng(seed)
    side = int(math.ceil(round(n ** (1.0 / 3.0), 9)))
    base, Z1 = water()
    base = base - base.mean(0)
    coords, Z = [], []
    for i in range(n):
        ix, iy, iz = i % side, (i // side) % side, i // (side * side)
        site = np.array([ix, iy, iz], dtype=float) * spacing
        site = (site + rng.uniform(-jitter, jitter, size=3)) * ANG_TO_BOHR
        R = _random_rotation(rng)
        coords.append(base @ R.T + site)
        Z += Z1
    return np.concatenate(coords), Z


def aggregate(natoms=1500, seed=0, dmin=1.0, density=0.09):
    """Large C/H/N/O aggregate (ratio 3:5:1:1) by random sequential packing
    inside a sphere (Angstrom inputs): points are drawn uniformly in the
    sphere and rejected when closer than dmin to an accepted atom.  The
    sphere radius gives `density` atoms per cubic Angstrom."""
    rng = np.random.default_rng(seed)
    radius = (3 * natoms / (4 * math.pi * density)) ** (1 / 3)
    counts = {6: 3, 1: 5, 7: 1, 8: 1}
    unit = sum(counts.values())
    Z = []
    for z, c in counts.items():
        Z += [z] * (natoms * c // unit)
    Z += [1] * (natoms - len(Z))
    Z = list(rng.permutation(Z))
    cell = dmin
    grid = {}
    pts = []
    while len(pts) < natoms:
        p = rng.uniform(-radius, radius, size=3)
        if p @ p > radius * radius:
            continue
        key = tuple(np.floor(p / cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        if np.sum((q - p) ** 2) < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pts.append(p)
            grid.setdefault(key, []).append(p)
    return np.array(pts) * ANG_TO_BOHR, [int(z) for z in Z]


# ------------------------------------------------------------------ bases --
def even_tempered(alpha, beta, k):
    return alpha * beta ** k


# shells per element: list of (l, number of exponents)
PRIMARY_SHELLS = {8: [(0, 6), (1, 4), (2, 2)], 1: [(0, 4), (1, 2)]}        # O 6s4p2d, H 4s2p
AUX_SHELLS = {8: [(0, 10), (1, 8), (2, 5), (3, 4)], 1: [(0, 6), (1, 4), (2, 2)]}
# 1500-atom aggregate: heavy 3s2p1d (14 functions), H 2s (2 functions)
AGG_SHELLS = {6: [(0, 3), (1, 2), (2, 1)], 7: [(0, 3), (1, 2), (2, 1)],
              8: [(0, 3), (1, 2), (2, 1)], 1: [(0, 2)]}


def sto_basis(coords, Z, shells=None, alpha=0.5, beta=2.2, alpha_by_z=None):
    """Even-tempered STO basis zeta_k = alpha * beta^k per (element, l), n = l+1,
    functions ordered atom by atom, shell by shell, m = -l..l."""
    shells = PRIMARY_SHELLS if shells is None else shells
    funcs = []
    for a, z in enumerate(Z):
        al = alpha if alpha_by_z is None else alpha_by_z.get(z, alpha)
        ox, oy, oz = coords[a]
        for l, nk in shells[z]:
            for k in range(nk):
                zeta = even_tempered(al, beta, k)
                for m in range(-l, l + 1):
                    funcs.append((l + 1, l, m, zeta, ox, oy, oz))
    return funcs


def aux_basis(coords, Z):
    """Even-tempered auxiliary STO basis zeta_k = 0.3 * 1.8^k up to l = 3
    (about 3x the primary size for water)."""
    return sto_basis(coords, Z, AUX_SHELLS, alpha=0.3, beta=1.8)


def aggregate_basis(coords, Z):
    """Synthetic basis of the 1500-atom aggregate: heavy atoms 3s2p1d with
    zeta_k = 1.4 * 2.4^k, H 2s with zeta_k = 1.2 * 2.4^k."""
    return sto_basis(coords, Z, AGG_SHELLS, alpha=1.4, beta=2.4, alpha_by_z={1: 1.2})


def random_orbitals(nbf, nocc, seed=0):
    """C (nbf x nocc) of i.i.d. N(0,1) entries orthonormalised by QR."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(nbf, nocc)))
    return np.ascontiguousarray(q)
