"""The N > 1 sharding of a Fock build (nukexc_b200/shard.py, used by bench.py)
on CPU: two gloo ranks integrate the points of their atom shares with the
oracle's dense XC build and sum E and V with shard.allreduce_fock; the sum
must equal the single-process build on the whole grid."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nukexc_b200 import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from nukexc_b200 import molecules as M
    from oracle import oracle as O
    c, Z = M.water_cluster(2, seed=3)
    pts, w, owner = O.make_flat_grid(c, Z, 20, 11, weight_threshold=1e-15, scheme="ta")
    funcs = M.sto_basis(c, Z)
    Cm = M.random_orbitals(len(funcs), 10, seed=4)
    return c, Z, pts, w, owner, funcs, Cm


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c, Z, pts, w, owner, funcs, Cm = _case()
        sel = shard.select_points(owner, len(Z), rank, world)
        b = O.make_manual_basis(funcs)
        if sel.any():
            E, V = O.xc_build(b, pts[sel], w[sel], [101, 130], [Cm], [2 * np.ones(10)])
            V = V[0]
        else:
            E, V = 0.0, np.zeros((len(funcs), len(funcs)))
        Et, (Vt,) = shard.allreduce_fock(E, [torch.as_tensor(V)], dist)
        counts = torch.tensor([int(sel.sum())], dtype=torch.int64)
        dist.all_reduce(counts)
        if rank == 0:
            np.savez(out, E=Et, V=Vt.numpy(), n=int(counts.item()))
    finally:
        dist.destroy_process_group()


def test_atom_ranges_partition_the_atoms():
    for natoms in (1, 2, 5, 192):
        for world in (1, 2, 3, 8):
            r = [shard.atom_range(natoms, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == natoms
            assert all(r[k][1] == r[k + 1][0] for k in range(world - 1))
    with pytest.raises(ValueError):
        shard.atom_range(4, 2, 2)


def test_two_gloo_ranks_sum_to_the_whole_grid(tmp_path):
    from oracle import oracle as O
    import torch.multiprocessing as mp
    out = str(tmp_path / "r0.npz")
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    r = np.load(out)
    c, Z, pts, w, owner, funcs, Cm = _case()
    E, V = O.xc_build(O.make_manual_basis(funcs), pts, w, [101, 130], [Cm], [2 * np.ones(10)])
    assert int(r["n"]) == len(w)
    assert float(r["E"]) == pytest.approx(E, rel=1e-12)
    assert np.abs(r["V"] - V[0]).max() < 1e-12 * max(1.0, np.abs(V[0]).max())
