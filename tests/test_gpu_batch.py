"""Batched independent systems: concurrent evaluation equals one-by-one evaluation."""
import numpy as np
import pytest

from gb200 import batch, solvers, synth

pytestmark = pytest.mark.gpu


def test_batch_equals_individual(gpu):
    systems = [synth.make_system(mesh=m, nao=n, naux=a, ns=1, beta=20.0, nts=20, eps_range=2.0, seed=31 + i)
               for i, (m, n, a) in enumerate([((2, 1, 1), 6, 24), ((2, 2, 1), 9, 40), ((1, 1, 3), 7, 30)])]
    ctxs = [solvers.make_context(s) for s in systems]
    try:
        want = [c.gw_sigma(s.G) for c, s in zip(ctxs, systems)]
        b = batch.SystemBatch(ctxs)
        got = b.run_gw_host([s.G for s in systems])
        for w, g in zip(want, got):
            assert np.array_equal(w, g)
    finally:
        for c in ctxs:
            c.close()


def test_batch_device_buffers(gpu):
    import torch
    systems = [synth.make_system(mesh=(2, 1, 1), nao=n, naux=4 * n, ns=1, beta=20.0, nts=20, eps_range=2.0,
                                 seed=50 + n) for n in (5, 8)]
    ctxs = [solvers.make_context(s) for s in systems]
    try:
        G = [torch.from_numpy(s.G).cuda() for s in systems]
        Sig = [torch.empty_like(g) for g in G]
        b = batch.SystemBatch(ctxs)
        times = b.run_gw([g.data_ptr() for g in G], [x.data_ptr() for x in Sig])
        torch.cuda.synchronize()
        assert len(times) == 2 and all(t["total"] > 0 for t in times)
        for c, s, x in zip(ctxs, systems, Sig):
            assert np.array_equal(x.cpu().numpy(), c.gw_sigma(s.G))
    finally:
        for c in ctxs:
            c.close()


def _uneven(seed0=70):
    shapes = [((2, 1, 1), 6, 24), ((2, 2, 1), 9, 40), ((1, 1, 3), 7, 30), ((2, 2, 2), 5, 26)]
    return [synth.make_system(mesh=m, nao=n, naux=a, ns=1, beta=20.0, nts=20, eps_range=2.0, seed=seed0 + i)
            for i, (m, n, a) in enumerate(shapes)]


def test_grouped_batch_matches_oracle_and_individual(gpu):
    """gb200_gw_sigma_batch_device: four systems of different nk, nao and naux, split precision,
    every contraction stage one grouped launch.  Each system's self-energy is bit-identical to
    its own gb200_gw_sigma_device call and within the split-precision bound of the oracle."""
    import torch

    import gw_oracle as O
    from gb200 import lib
    systems = _uneven()
    ctxs = [solvers.make_context(s, precision=lib.PREC_SPLIT, slices=5) for s in systems]
    try:
        G = [torch.from_numpy(s.G).cuda() for s in systems]
        Sig = [torch.empty_like(g) for g in G]
        b = batch.SystemBatch(ctxs)
        b.run_gw_grouped([g.data_ptr() for g in G], [x.data_ptr() for x in Sig])
        torch.cuda.synchronize()
        for c, s, x in zip(ctxs, systems, Sig):
            got = x.cpu().numpy()
            assert np.array_equal(got, c.gw_sigma(s.G))
            ref = O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), s.grid.Tnt_b, s.grid.Ttn_b,
                             s.ns, s.NQ)
            assert np.abs(got - ref).max() < 1e-8 * max(1.0, np.abs(ref).max())
    finally:
        for c in ctxs:
            c.close()


def test_grouped_batch_fp64_and_tile_widths(gpu):
    """FP64 contexts go through the same call one contraction at a time (1e-10 against the oracle);
    a chosen tile width changes the tiling, not a bit of the split-precision result."""
    import torch

    import gw_oracle as O
    from gb200 import lib
    systems = _uneven(90)[:3]
    ctxs = [solvers.make_context(s) for s in systems]
    try:
        G = [torch.from_numpy(s.G).cuda() for s in systems]
        Sig = [torch.empty_like(g) for g in G]
        batch.SystemBatch(ctxs).run_gw_grouped([g.data_ptr() for g in G], [x.data_ptr() for x in Sig])
        torch.cuda.synchronize()
        for s, x in zip(systems, Sig):
            ref = O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), s.grid.Tnt_b, s.grid.Ttn_b,
                             s.ns, s.NQ)
            assert np.abs(x.cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()
        c, s = ctxs[1], systems[1]
        c.set_precision(lib.PREC_SPLIT, 5)
        base = c.gw_sigma(s.G)
        for bn in (16, 32, 48):
            c.set_tile_width(bn)
            assert np.array_equal(c.gw_sigma(s.G), base)
        c.set_tile_width(0)
    finally:
        for c in ctxs:
            c.close()
