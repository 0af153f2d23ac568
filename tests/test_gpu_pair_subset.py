"""q-sharded integral storage on the GPU (gb200_set_integrals_pairs).

Two contexts stand in for two ranks: each holds only the stored pairs its q range reads
(gb200.shard.pairs_for_q_range), computes its partial self-energy and its partial Fock matrix,
and the two partial results must add up to the oracle's full ones (gw_cpu_kernel.cpp:45-48,53-54
for Sigma; for the Fock matrix the exchange splits by q = k' - k, the direct and Madelung terms
go to the range that holds q = 0).  The contexts run one after the other on one GPU; nothing
waits on another context.
"""
import numpy as np
import pytest

import gw_oracle as O
from gb200 import lib, shard, solvers
from _systems import oracle_fock, oracle_sigma, rel, system

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _subset_context(s, q0, q1, precision=lib.PREC_FP64):
    g = s.grid
    kp, km = solvers.kq_maps(s.mesh)
    ids = shard.pairs_for_q_range(kp, q0, q1)
    ctx = lib.Context(s.nk, s.nao, s.ns, s.NQ, g.nts, g.nw, g.nw_b, s.beta)
    ctx.set_kq_maps(kp, km)
    ctx.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
    ctx.set_integrals_pairs(np.ascontiguousarray(s.V_half[ids]), ids)
    ctx.set_q_range(q0, q1)
    ctx.set_precision(precision, 5)
    return ctx, ids


@pytest.mark.parametrize("name", ["small", "small_ns2", "odd_mesh"])
def test_pair_subsets_sum_to_full_sigma_and_fock(gpu, name):
    s = system(name)
    ranges = [shard.q_shard(s.nk, 2, r) for r in range(2)]
    sig = np.zeros_like(s.G)
    F = np.zeros_like(s.S)
    held = set()
    mad = 0.23
    for q0, q1 in ranges:
        ctx, ids = _subset_context(s, q0, q1)
        try:
            held |= set(ids.tolist())
            sig += ctx.gw_sigma(s.G)
            F += ctx.hf_fock(O.hf_density(s.G, s.ns), s.S, mad)
        finally:
            ctx.close()
    assert held == set(range(s.nk * (s.nk + 1) // 2))
    assert rel(sig, oracle_sigma(name)) < TOL
    assert rel(F, oracle_fock(s, mad)) < TOL


def test_pair_subset_split_precision(gpu):
    s = system("small")
    sig = np.zeros_like(s.G)
    for r in range(2):
        ctx, _ = _subset_context(s, *shard.q_shard(s.nk, 2, r), precision=lib.PREC_SPLIT)
        try:
            sig += ctx.gw_sigma(s.G)
        finally:
            ctx.close()
    ref = oracle_sigma("small")
    assert float(np.abs(sig - ref).max()) < 1e-8 * max(1.0, float(np.abs(ref).max()))


def test_pair_subset_refuses_uncovered_q_range(gpu):
    """A q range whose pairs the subset does not hold is an error, not a silent wrong result; the
    adjoint, which runs every q-point, needs the full pair set."""
    s = system("odd_mesh")
    ctx, _ = _subset_context(s, 0, 1)
    try:
        ctx.set_q_range(0, s.nk)
        with pytest.raises(RuntimeError):
            ctx.gw_sigma(s.G)
        with pytest.raises(RuntimeError):
            ctx.hf_fock(O.hf_density(s.G, s.ns), s.S, 0.0)
        ctx.set_q_range(0, 1)
        with pytest.raises(RuntimeError):
            ctx.gw_sigma_vjp(s.G, np.ones_like(s.G))
    finally:
        ctx.close()
