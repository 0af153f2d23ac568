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
