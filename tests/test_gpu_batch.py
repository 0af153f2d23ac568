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
