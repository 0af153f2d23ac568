"""q-point sharding of the GW self-energy over ranks (one process per GPU).

The reference splits the irreducible q-points over nodes and sums the partial
self-energies with one allreduce (gw_cpu_kernel.cpp:45-48,53-54).  Here each
rank's context is restricted to a contiguous q range (gb200_set_q_range); the
partial Sigma of a range is already divided by nk, so the ranks' results add up
to the full self-energy.  The work per q is uniform, so ranges are balanced by
count.
"""
from __future__ import annotations


def q_shard(nq: int, world_size: int, rank: int) -> tuple[int, int]:
    """[q_begin, q_end) of `rank`: sizes differ by at most one, lower ranks take the extra q."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} of {world_size}")
    if nq < 0:
        raise ValueError("nq must be non-negative")
    base, extra = divmod(nq, world_size)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def reduce_partial_sigma(Sigma, dist, group=None):
    """Sum the ranks' partial Sigma in place (complex128 reduced as pairs of float64)."""
    import torch
    dist.all_reduce(torch.view_as_real(Sigma), op=dist.ReduceOp.SUM, group=group)
    return Sigma
