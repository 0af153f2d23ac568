"""q-point sharding of the GW self-energy over ranks (one process per GPU).

The reference splits the irreducible q-points over nodes and sums the partial
self-energies with one allreduce (gw_cpu_kernel.cpp:45-48,53-54).  Here each
rank's context is restricted to a contiguous q range (gb200_set_q_range); the
partial Sigma of a range is already divided by nk, so the ranks' results add up
to the full self-energy.  The work per q is uniform, so ranges are balanced by
count.  Each rank needs only the integral pairs its q range reads
(pairs_for_q_range, uploaded with gb200_set_integrals_pairs).
"""
from __future__ import annotations

import numpy as np


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


def pairs_for_q_range(kplus, q_begin: int, q_end: int):
    """Stored-pair indices (k1 (k1 + 1) / 2 + k2, k1 >= k2, increasing) that the q-points
    [q_begin, q_end) read: V(k, k+q) for P0 and V(k, k-q) for Sigma (gw_cpu_kernel.cpp:88-90,
    113-119).  Both are blocks of the unordered pair {k, k+q}: (k', k'-q) with k' = k + q.
    kplus[k, q] is the index of k + q (solvers.kq_maps / inputs.kq_maps_from_points)."""
    kp = np.asarray(kplus)
    nk = kp.shape[0]
    if not 0 <= q_begin <= q_end <= nk:
        raise ValueError(f"q range [{q_begin}, {q_end}) outside [0, {nk})")
    k = np.arange(nk)[:, None]
    k2 = kp[:, q_begin:q_end]
    a, b = np.maximum(k, k2), np.minimum(k, k2)
    return np.unique((a * (a + 1) // 2 + b).ravel()).astype(np.int64)


def integral_blocks_held(npairs_ids, nk: int) -> int:
    """Ordered [NQ, nao, nao] blocks a context keeps for the stored pairs `npairs_ids`."""
    ids = np.asarray(npairs_ids)
    k1 = ((np.sqrt(8.0 * ids + 1.0) - 1.0) // 2).astype(np.int64)
    k1 -= (k1 * (k1 + 1) // 2 > ids)
    k1 += ((k1 + 1) * (k1 + 2) // 2 <= ids)
    diag = (ids - k1 * (k1 + 1) // 2) == k1
    return int(2 * len(ids) - diag.sum())
