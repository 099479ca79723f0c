"""The N > 1 sharding of a Fock build (nukexc_b200/shard.py, used by bench.py)
on CPU: two gloo ranks integrate their cost-balanced, Morton-contiguous
batch ranges with the oracle's dense XC build and sum E and V with
shard.allreduce_fock; with J, the two-phase build sums the fit vector y and
the metric as well.  The sums must equal the single-process build on the
whole grid."""
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
        b = O.make_manual_basis(funcs)
        sel = np.zeros(len(w), bool)
        sel[shard.balanced_split(pts, b["center"], b["cutoff"], 10, world)[rank]] = True
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


# ------------------------------------------------ DF-J on a sharded grid ----
class OracleShardBuilder:
    """Stands in for FockBuilder on CPU in the two-phase build: the same
    methods (aux_metric, set_metric, build_phase1, build_phase2) with the
    oracle's dense restatement on this rank's points.  Phase 1 returns this
    rank's y = Vw rho; phase 2 solves c = S^-1 y with the installed (summed)
    metric and returns this rank's E_xc, V_xc and J = Phi diag(Vw^T c) Phi^T."""

    def __init__(self, funcs, aux, pts, w, ids):
        from oracle import oracle as O
        self.O = O
        self.b, self.a = O.make_manual_basis(funcs), O.make_manual_basis(aux)
        self.pts, self.w, self.ids = pts, w, ids
        self.Vw = O.potential_collocation(self.a, pts, w)
        self.phi = O.collocation(self.b, pts)
        self.S = O.aux_metric(self.a, pts, w)
        self.Sfull = None

    def aux_metric(self):
        return self.S

    def set_metric(self, S):
        self.Sfull = np.asarray(S)

    def build_phase1(self, C_list, occ_list, precision="fp64", stream=None):
        self.E, self.V, rho = self.O.xc_build(self.b, self.pts, self.w, self.ids, C_list, occ_list, want_rho=True)
        return self.Vw @ rho.sum(1)

    def build_phase2(self, y, want_J=True, fuse_j=False, stream=None):
        c = np.linalg.solve(self.Sfull, np.asarray(y))
        J = (self.phi * (self.Vw.T @ c)) @ self.phi.T
        return self.E, list(self.V), J


def _jcase():
    from nukexc_b200 import molecules as M
    c, Z, pts, w, owner, funcs, Cm = _case()
    aux = M.sto_basis(c, Z, {8: [(0, 4), (1, 3), (2, 2)], 1: [(0, 3), (1, 2)]}, alpha=0.8, beta=2.5)
    return c, Z, pts, w, funcs, aux, Cm


def _split(pts, funcs, world):
    from oracle import oracle as O
    b = O.make_manual_basis(funcs)
    return shard.balanced_split(pts, b["center"], b["cutoff"], 10, world)


def _rank_main_j(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c, Z, pts, w, funcs, aux, Cm = _jcase()
        sel = _split(pts, funcs, world)[rank]
        fb = OracleShardBuilder(funcs, aux, pts[sel], w[sel], [101, 130])
        shard.shard_metric(fb, dist)
        E, V, J = shard.sharded_build(fb, [Cm], [2 * np.ones(10)], dist)
        if rank == 0:
            np.savez(out, E=E, V=V[0].numpy(), J=J.numpy())
    finally:
        dist.destroy_process_group()


def test_balanced_split_partitions_morton_ranges_of_equal_cost():
    from oracle import oracle as O
    c, Z, pts, w, owner, funcs, Cm = _case()
    b = O.make_manual_basis(funcs)
    for world in (1, 2, 3, 4):
        parts = _split(pts, funcs, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(pts)))
        perm = shard.morton_order(pts)
        cost = shard.batch_costs(pts[perm], b["center"], b["cutoff"], 10)
        per = []
        off = 0
        for p in parts:
            assert np.array_equal(p, perm[off:off + len(p)])  # Morton-contiguous
            per.append(cost[off // shard.BATCH:(off + len(p) + shard.BATCH - 1) // shard.BATCH].sum())
            off += len(p)
        # equal cost up to one batch
        assert max(per) - min(per) <= cost.max() + 1e-9 * sum(per)


def test_two_gloo_ranks_sharded_coulomb_build(tmp_path):
    from oracle import oracle as O
    import torch.multiprocessing as mp
    out = str(tmp_path / "j0.npz")
    mp.spawn(_rank_main_j, args=(2, _free_port(), out), nprocs=2, join=True)
    r = np.load(out)
    c, Z, pts, w, funcs, aux, Cm = _jcase()
    ob, oa = O.make_manual_basis(funcs), O.make_manual_basis(aux)
    occ = 2 * np.ones(10)
    E, V = O.xc_build(ob, pts, w, [101, 130], [Cm], [occ])
    J, _ = O.coulomb(ob, oa, pts, w, Cm, occ, S=O.aux_metric(oa, pts, w))
    assert float(r["E"]) == pytest.approx(E, rel=1e-12)
    assert np.abs(r["V"] - V[0]).max() < 1e-12 * max(1.0, np.abs(V[0]).max())
    assert np.abs(r["J"] - J).max() < 1e-9 * np.abs(J).max()
