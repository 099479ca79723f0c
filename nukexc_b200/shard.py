"""Sharding of one Fock build over ranks (one process per GPU).

Grid points are independent, so rank r integrates the points owned by its
contiguous share of the atoms (a Morton-local region of space; the plan of
each rank screens only its own batches) and the partial V (per spin, plus J)
and E are summed with one all-reduce.  Every rank takes the same collective
steps in the same order.
"""
from __future__ import annotations

import numpy as np


def atom_range(natoms: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of the atoms for `rank` of `world`."""
    if not (0 <= rank < world):
        raise ValueError("rank outside [0, world)")
    return (natoms * rank) // world, (natoms * (rank + 1)) // world


def select_points(point_owner, natoms: int, rank: int, world: int) -> np.ndarray:
    """Boolean mask of the grid points this rank integrates."""
    lo, hi = atom_range(natoms, rank, world)
    own = np.asarray(point_owner)
    return (own >= lo) & (own < hi)


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
