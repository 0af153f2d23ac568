"""Multi-rank host logic of the q-sharded GW path, on CPU with gloo.

Each rank computes the partial self-energy of its q range (the oracle stands in
for the device here), the partial results are summed with the same reduction
helper the multi-GPU bench uses, and the sum must equal the unsharded
self-energy (gw_cpu_kernel.cpp:45-48,53-54).
"""
import os
import socket

import numpy as np
import pytest

from gb200 import shard


def test_q_shard_partition():
    for nq in range(0, 40):
        for ws in range(1, 10):
            ranges = [shard.q_shard(nq, ws, r) for r in range(ws)]
            assert ranges[0][0] == 0 and ranges[-1][1] == nq
            for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
                assert a1 == b0
            sizes = [b - a for a, b in ranges]
            assert min(sizes) >= 0 and max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.q_shard(5, 2, 2)
    with pytest.raises(ValueError):
        shard.q_shard(5, 0, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, name, out_dir):
    import torch
    import torch.distributed as dist

    import gw_oracle as O
    from _systems import system

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        s = system(name)
        bz = O.NoSymBZ(s.mesh)
        q0, q1 = shard.q_shard(s.nk, ws, rank)
        part = O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), bz, s.grid.Tnt_b, s.grid.Ttn_b, s.ns, s.NQ,
                          q_list=range(q0, q1))
        t = torch.from_numpy(part)
        shard.reduce_partial_sigma(t, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "sigma.npy"), t.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


class _RecordingPairs:
    """Half-stored integrals restricted to a pair subset: records every stored pair read and
    refuses one outside the subset (the oracle's gw_solve stands in for the device here)."""

    def __init__(self, V_half, held):
        self.V_half, self.held, self.read = V_half, set(int(p) for p in held), set()

    def pair(self, k1, k2):
        import gw_oracle as O
        p = O.pair_index(k1, k2)
        if p not in self.held:
            raise KeyError(f"pair ({k1}, {k2}) is not in this rank's subset")
        self.read.add(p)
        return O.HalfStoredIntegrals(self.V_half).pair(k1, k2)


def _subset_rank_main(rank, ws, port, name, out_dir):
    import torch
    import torch.distributed as dist

    import gw_oracle as O
    from _systems import system
    from gb200 import solvers

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        s = system(name)
        kp, _ = solvers.kq_maps(s.mesh)
        q0, q1 = shard.q_shard(s.nk, ws, rank)
        held = shard.pairs_for_q_range(kp, q0, q1)
        ints = _RecordingPairs(s.V_half, held)
        part = O.gw_solve(s.G, ints, O.NoSymBZ(s.mesh), s.grid.Tnt_b, s.grid.Ttn_b, s.ns, s.NQ, q_list=range(q0, q1))
        # the rank's subset is exactly what its q range reads
        assert ints.read == set(int(p) for p in held), (rank, sorted(set(held) - ints.read))
        np.save(os.path.join(out_dir, f"pairs{rank}.npy"), held)
        t = torch.from_numpy(part)
        shard.reduce_partial_sigma(t, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "sigma.npy"), t.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,ws", [("small", 2), ("odd_mesh", 2)])
def test_rank_pair_subsets_match_reads(tmp_path, name, ws):
    """Per-rank integral storage for the q split: each gloo rank keeps only
    shard.pairs_for_q_range of its q range, the oracle's GW sweep over that range reads exactly
    those pairs (no more, no fewer), the partial self-energies still sum to the full one, and
    together the ranks hold every stored pair."""
    import torch.multiprocessing as mp

    import gw_oracle as O
    from _systems import system

    mp.start_processes(_subset_rank_main, args=(ws, _free_port(), name, str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    s = system(name)
    full = O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), s.grid.Tnt_b, s.grid.Ttn_b, s.ns, s.NQ)
    got = np.load(tmp_path / "sigma.npy")
    assert np.abs(got - full).max() <= 1e-12 * np.abs(full).max()
    union = set()
    for r in range(ws):
        union |= set(np.load(tmp_path / f"pairs{r}.npy").tolist())
    assert union == set(range(s.nk * (s.nk + 1) // 2))


def test_pair_subset_sizes():
    """At nk = 125 (5x5x5) and 8 ranks each rank keeps 20-26% of the ordered blocks (the q and
    -q of its range read the same pairs only when both are in the range)."""
    from gb200 import solvers
    kp, _ = solvers.kq_maps((5, 5, 5))
    for r in range(8):
        q0, q1 = shard.q_shard(125, 8, r)
        ids = shard.pairs_for_q_range(kp, q0, q1)
        assert np.all(np.diff(ids) > 0)
        frac = shard.integral_blocks_held(ids, 125) / 125 ** 2
        assert 0.19 < frac < 0.27, (r, frac)
    assert shard.integral_blocks_held(shard.pairs_for_q_range(kp, 0, 125), 125) == 125 ** 2


@pytest.mark.parametrize("name,ws", [("small", 2), ("odd_mesh", 2)])
def test_sharded_sigma_sums_to_full(tmp_path, name, ws):
    import torch.multiprocessing as mp

    import gw_oracle as O
    from _systems import system

    mp.start_processes(_rank_main, args=(ws, _free_port(), name, str(tmp_path)), nprocs=ws, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / "sigma.npy")
    s = system(name)
    full = O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), s.grid.Tnt_b, s.grid.Ttn_b, s.ns, s.NQ)
    assert np.abs(got - full).max() <= 1e-12 * np.abs(full).max()


def test_batch_memory_shares_are_proportional():
    """SystemBatch.share_memory splits a byte budget over contexts by their intermediate sizes."""
    from gb200 import batch

    class Dims:
        def __init__(self, nts, ns, NQ, nao):
            self.nts, self.ns, self.NQ, self.nao = nts, ns, NQ, nao

    class Ctx:
        def __init__(self, *d):
            self.dims = Dims(*d)
            self.budget = None

        def set_memory_budget(self, b):
            self.budget = b

    ctxs = [Ctx(80, 1, 40, 8), Ctx(80, 1, 240, 48), Ctx(80, 2, 100, 20)]
    b = batch.SystemBatch(ctxs).share_memory(60e9)
    assert abs(sum(b) - 60e9) < 1.0
    sizes = [80 * 1 * 40 * 64, 80 * 1 * 240 * 48 * 48, 80 * 2 * 100 * 400]
    for c, x in zip(ctxs, sizes):
        assert abs(c.budget / 60e9 - x / sum(sizes)) < 1e-12


def test_tile_table_lookup():
    """The autotuner's table is read by nearest measured (nao, naux); without one the widest tile."""
    from gb200 import tune
    table = {"8x32": {"bn": 32}, "40x200": {"bn": 80}, "48x288": {"bn": 96}}
    assert tune.choose_tile(9, 36, table) == 32
    assert tune.choose_tile(40, 210, table) == 80
    assert tune.choose_tile(47, 280, table) == 96
    assert tune.choose_tile(20, 100, {}) == 0
    for key, entry in tune.load_table().items():
        nao, naux = (int(x) for x in key.split("x"))
        assert entry["bn"] in tune.CANDIDATES and min(entry["ms"], key=lambda k: entry["ms"][k]) == str(entry["bn"])
