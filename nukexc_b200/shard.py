"""Sharding of one Fock build over ranks (one process per GPU).

Grid points are independent, so every rank integrates its own share of the
grid with its own plan, and the partial V (per spin, plus J) and E are summed
with one all-reduce.  The split is static and cost-balanced: the points are
put in Morton order (the order the plans batch them in), cut into 256-point
batches, each batch is costed by the basis functions whose cutoff sphere meets
its bounding box (n_b), cost_b = n_b (n_b + n_occ) + 64 n_b (the V and density
contractions and the collocation), and the batch list is cut into contiguous,
equal-cost ranges -- a spatially compact region per rank.

The grid RI-J fit needs the whole grid's fit vector y before any potential,
so a build with J runs in two phases around one more all-reduce (of y, N_aux
doubles); the metric (A|B) is a sum over points too and is all-reduced once
per geometry (shard_metric).  Every rank takes the same collective steps in
the same order.
"""
from __future__ import annotations

import numpy as np

BATCH = 256
COLLOC_WEIGHT = 64.0


def atom_range(natoms: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of the atoms for `rank` of `world`."""
    if not (0 <= rank < world):
        raise ValueError("rank outside [0, world)")
    return (natoms * rank) // world, (natoms * (rank + 1)) // world


def select_points(point_owner, natoms: int, rank: int, world: int) -> np.ndarray:
    """Boolean mask of the points owned by `rank`'s contiguous share of the atoms."""
    lo, hi = atom_range(natoms, rank, world)
    own = np.asarray(point_owner)
    return (own >= lo) & (own < hi)


def morton_order(xyz) -> np.ndarray:
    """Morton permutation of the points (nkx_morton_order, host code of the
    library: the plans' own point order)."""
    import ctypes as C

    from . import _lib as L
    p = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    perm = np.zeros(len(p), np.int64)
    L.check(L.lib().nkx_morton_order(len(p), p.ctypes.data_as(C.c_void_p), perm.ctypes.data_as(C.c_void_p)))
    return perm


def batch_costs(xyz_sorted, centers, cutoffs, nocc: int, batch: int = BATCH, chunk: int = 4096) -> np.ndarray:
    """cost_b = n_b (n_b + nocc) + COLLOC_WEIGHT n_b of each `batch`-point
    batch of the (Morton-sorted) points, n_b = basis functions whose cutoff
    sphere (centre, radius) meets the batch's bounding box (the plans'
    screening test at function granularity)."""
    p = np.asarray(xyz_sorted, np.float64).reshape(-1, 3)
    nb = (len(p) + batch - 1) // batch
    pad = np.concatenate([p, np.repeat(p[-1:], nb * batch - len(p), 0)]) if len(p) % batch else p
    box = pad.reshape(nb, batch, 3)
    lo, hi = box.min(1), box.max(1)
    ctr = np.asarray(centers, np.float64).reshape(-1, 3)
    cut = np.asarray(cutoffs, np.float64)
    # functions grouped by centre: per distinct centre, its sorted cutoff radii
    uc, inv = np.unique(ctr, axis=0, return_inverse=True)
    inv = np.asarray(inv).reshape(-1)
    groups = [np.sort(cut[inv == k]) for k in range(len(uc))]
    n = np.zeros(nb)
    for b0 in range(0, nb, chunk):
        l, h = lo[b0:b0 + chunk, None, :], hi[b0:b0 + chunk, None, :]
        d = np.sqrt((np.maximum(np.maximum(l - uc[None], uc[None] - h), 0.0) ** 2).sum(-1))  # (batches, centres)
        for k, g in enumerate(groups):
            n[b0:b0 + chunk] += len(g) - np.searchsorted(g, d[:, k], side="left")
    return n * (n + nocc) + COLLOC_WEIGHT * n


def balanced_split(xyz, centers, cutoffs, nocc: int, world: int, batch: int = BATCH):
    """Point index arrays (into xyz) of the `world` ranks: contiguous ranges
    of the Morton-ordered batch list with equal summed cost."""
    perm = morton_order(xyz)
    cost = batch_costs(np.asarray(xyz, np.float64).reshape(-1, 3)[perm], centers, cutoffs, nocc, batch)
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    cuts = [0] + [int(np.searchsorted(cum, cum[-1] * r / world, side="left")) for r in range(1, world)] + [len(cost)]
    cuts = np.maximum.accumulate(np.asarray(cuts))
    return [perm[cuts[r] * batch:min(len(perm), cuts[r + 1] * batch)] for r in range(world)]


def _as_tensor(x):
    import torch
    return x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x, np.float64))


def allreduce_fock(E: float, V_list, dist, device=None):
    """Sum E and the V matrices over the process group in one all-reduce.
    V_list holds torch tensors (device or host, one per spin/J plane);
    returns (E_total, [V_total ...])."""
    import torch

    dev = device if device is not None else V_list[0].device
    flat = torch.cat([v.reshape(-1).to(dev, torch.float64) for v in V_list] +
                     [torch.tensor([E], dtype=torch.float64, device=dev)])
    dist.all_reduce(flat)
    out, off = [], 0
    for v in V_list:
        n = v.numel()
        out.append(flat[off:off + n].view(v.shape))
        off += n
    return float(flat[-1].item()), out


def shard_metric(fb, dist):
    """All-reduce the ranks' grid Coulomb metrics (A|B) into the full grid's
    and install it in every rank's plan (once per geometry)."""
    S = _as_tensor(fb.aux_metric()).contiguous().to("cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(S)
    fb.set_metric(S.cpu().numpy())
    return S


def sharded_build(fb, C_list, occ_list, dist, precision="fp64", want_J=True, fuse_j=False, stream=None):
    """One Fock build with J on a sharded grid: phase 1 (density and this
    rank's share of y), all-reduce of y, phase 2 (fit, functional, V and J on
    this rank's points), all-reduce of E, V and J.  Returns the whole grid's
    (E_xc, [V per spin], J or None) on every rank."""
    y = _as_tensor(fb.build_phase1(C_list, occ_list, precision=precision, stream=stream))
    host = not y.is_cuda
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"  # NCCL reduces device tensors only
    y = y.to(dev)
    dist.all_reduce(y)
    E, V, J = fb.build_phase2(y.cpu().numpy() if host else y, want_J=want_J, fuse_j=fuse_j, stream=stream)
    mats = [_as_tensor(v) for v in V] + ([_as_tensor(J)] if J is not None else [])
    E, out = allreduce_fock(E, mats, dist, device=dev)
    return E, out[:len(V)], (out[-1] if J is not None else None)
