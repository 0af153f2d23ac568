"""Many independent systems on one GPU (the batched uneven-systems workload).

Each system keeps its own context: its integrals, grid, maps and scratch buffers, and its own
CUDA stream.  `run_gw_grouped` evaluates all of them in one library call whose contraction stages
are grouped persistent launches over the tiles of every system (gb200_gw_sigma_batch_device), with
tile widths from the autotuner's table (`apply_tiles`).  `run_gw` instead issues the self-energy of
every system from a pool of host threads.  The
library calls release the interpreter lock, so the systems' kernels are queued on different
streams and overlap on the device wherever one system does not fill it: the slicing and FP64
kernels of one system run beside the contraction kernel of another.  Results are identical to
running the systems one by one: every context computes exactly what it would alone.
"""
from __future__ import annotations

import concurrent.futures as cf

import numpy as np


class SystemBatch:
    """A set of prepared contexts that are evaluated together."""

    def __init__(self, contexts, streams=None, workers: int | None = None):
        self.contexts = list(contexts)
        self.streams = list(streams) if streams is not None else [0] * len(self.contexts)
        if len(self.streams) != len(self.contexts):
            raise ValueError("one stream per context")
        self.workers = workers or len(self.contexts)

    def __len__(self):
        return len(self.contexts)

    def share_memory(self, total_bytes: float):
        """Give every context a budget for its blocked intermediates out of `total_bytes`, in
        proportion to the size of one k-point block of its self-energy intermediates
        (nts * ns * NQ * nao^2 complex values), so that all contexts fit on one GPU together."""
        sizes = []
        for c in self.contexts:
            d = c.dims
            sizes.append(float(d.nts) * d.ns * d.NQ * d.nao * d.nao * 16.0)
        tot = sum(sizes)
        budgets = [total_bytes * x / tot for x in sizes]
        for c, b in zip(self.contexts, budgets):
            c.set_memory_budget(b)
        return budgets

    def run_gw(self, G_ptrs, Sigma_ptrs):
        """gw_sigma_device for every system (device pointers), concurrently; returns the per-system
        stage timings (ms) of the calls."""
        if len(G_ptrs) != len(self) or len(Sigma_ptrs) != len(self):
            raise ValueError("one G and one Sigma buffer per system")

        def one(i):
            c = self.contexts[i]
            c.gw_sigma_device(G_ptrs[i], Sigma_ptrs[i], stream=self.streams[i])
            return c.last_timings()

        with cf.ThreadPoolExecutor(max_workers=self.workers) as ex:
            return list(ex.map(one, range(len(self))))

    def run_gw_grouped(self, G_ptrs, Sigma_ptrs, stream: int = 0):
        """gb200_gw_sigma_batch_device over all systems in one call: the systems' q-points in step,
        each contraction stage one grouped persistent tensor-core launch over the tiles of every
        system (all in split precision with the same slice count)."""
        from . import lib
        if len(G_ptrs) != len(self) or len(Sigma_ptrs) != len(self):
            raise ValueError("one G and one Sigma buffer per system")
        lib.gw_sigma_batch_device(self.contexts, G_ptrs, Sigma_ptrs, stream)

    def apply_tiles(self, table=None):
        """Tile width of every context from the autotuner's table (gb200.tune.choose_tile)."""
        from . import tune
        widths = []
        for c in self.contexts:
            d = c.dims
            bn = tune.choose_tile(d.nao, d.NQ, table)
            c.set_tile_width(bn)
            widths.append(bn)
        return widths

    def run_gw_host(self, Gs):
        """gw_sigma (host arrays in and out) for every system, concurrently."""
        def one(i):
            return self.contexts[i].gw_sigma(Gs[i])

        with cf.ThreadPoolExecutor(max_workers=self.workers) as ex:
            return list(ex.map(one, range(len(self))))

    def close(self):
        for c in self.contexts:
            c.close()
        self.contexts = []


def uneven_systems(count: int = 16, seed: int = 0, nts: int = 80, beta: float = 100.0, meshes=None,
                   with_integrals: bool = True):
    """Synthetic systems of the batched workload: nk from {8, 27, 64}, nao ~ U{8..48},
    naux ~ U{4 nao .. 6 nao}, ntau = 80, beta = 100, per-system seeds (the generator of the
    single-system configurations).  with_integrals=False leaves V out (to be generated on the
    device, synth.upload_device_integrals)."""
    from . import synth
    rng = np.random.default_rng(seed)
    meshes = meshes or [(2, 2, 2), (3, 3, 3), (4, 4, 4)]
    out = []
    for i in range(count):
        mesh = meshes[int(rng.integers(len(meshes)))]
        nao = int(rng.integers(8, 49))
        naux = int(rng.integers(4 * nao, 6 * nao + 1))
        out.append(synth.make_system(mesh=mesh, nao=nao, naux=naux, ns=1, beta=beta, nts=nts, eps_range=2.0,
                                     seed=seed * 1000 + i, with_integrals=with_integrals))
    return out
