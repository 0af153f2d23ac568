"""Seeded synthetic systems with the shapes of the benchmark configurations.

No public dataset is involved: the reference's own inputs come from PySCF
runs, which cannot be reproduced here.  The generator follows one recipe:

* Monkhorst-Pack n1 x n2 x n3 mesh, no point-group symmetry (ink = nk),
  q = k1 - k2 on the mesh.
* per spin and k: U_k Haar-random (QR of a complex Gaussian with the phase
  fix of Mezzadri 2007), eps ~ U[-E, E], F_k = U diag(eps) U^H, S_k = I, mu = 0.
* G(tau, k) = -U diag(f(eps, tau)) U^H, f = exp(-eps tau)/(1 + exp(-beta eps)),
  evaluated in the overflow-free form for eps < 0.
* V^Q_ij(k1, k2) for k1 > k2: complex Gaussian with E|V|^2 = 1/naux; for
  k1 = k2 each V^Q is made Hermitian; for k1 < k2 it is the per-Q conjugate
  transpose of the (k2, k1) block (so only k1 >= k2 is stored, in the order of
  df_integral_t.h:68).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .grids import ChebyshevGrid, cached_grid


CONFIGS = {
    # name: (mesh, nao, naux, ns, beta, nts, nw, eps range)
    "c0": ((2, 2, 2), 10, 40, 1, 100.0, 60, None, 2.0),
    "c1": ((4, 4, 4), 26, 150, 2, 100.0, 100, None, 2.0),
    "c2": ((5, 5, 5), 40, 250, 1, 200.0, 120, 120, 5.0),
    "c4": ((3, 3, 3), 20, 100, 1, 100.0, 80, None, 2.0),
    # c2's orbital, auxiliary and time shapes on a 2x1x1 mesh: the kernel-profiling case
    "c2k2": ((2, 1, 1), 40, 250, 1, 200.0, 120, 120, 5.0),
}


def haar_unitary(rng, n):
    z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diag(r)
    return q * (d / np.abs(d))[None, :]


def fermi_tau(eps, tau, beta):
    """exp(-eps tau)/(1+exp(-beta eps)) without overflow; shape [ntau, neps]."""
    eps = np.asarray(eps)[None, :]
    tau = np.asarray(tau)[:, None]
    pos = eps >= 0
    e_pos = np.where(pos, eps, 0.0)
    e_neg = np.where(pos, 0.0, eps)
    a = np.exp(-e_pos * tau) / (1.0 + np.exp(-beta * e_pos))
    b = np.exp((beta - tau) * e_neg) / (1.0 + np.exp(beta * e_neg))
    return np.where(pos, a, b)


def pair_count(nk):
    return nk * (nk + 1) // 2


@dataclass
class System:
    mesh: tuple
    nk: int
    nao: int
    NQ: int
    ns: int
    beta: float
    grid: ChebyshevGrid
    eps: np.ndarray            # [ns, nk, nao]
    U: np.ndarray              # [ns, nk, nao, nao]
    F: np.ndarray              # [ns, nk, nao, nao]
    S: np.ndarray              # [ns, nk, nao, nao]
    G: np.ndarray              # [nts, ns, nk, nao, nao]
    V_half: np.ndarray         # [nk(nk+1)/2, NQ, nao, nao]
    madelung: float = 0.0
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def nts(self):
        return self.grid.nts

    @property
    def nso(self):
        return self.nao

    def V_full(self):
        """All ordered pairs [nk, nk, NQ, nao, nao] (k1 < k2 by conjugate transpose)."""
        nk = self.nk
        out = np.empty((nk, nk) + self.V_half.shape[1:], dtype=np.complex128)
        for k1 in range(nk):
            for k2 in range(nk):
                if k1 >= k2:
                    out[k1, k2] = self.V_half[k1 * (k1 + 1) // 2 + k2]
                else:
                    out[k1, k2] = np.conj(np.swapaxes(self.V_half[k2 * (k2 + 1) // 2 + k1], -1, -2))
        return out

    def nel_from_G0(self):
        """Electron count of the generator's G0 at mu = 0 with exact Fermi occupations."""
        occ = 1.0 / (1.0 + np.exp(np.clip(self.beta * self.eps, -700, 700)))
        pref = 2.0 if self.ns == 1 else 1.0
        return float(pref * occ.sum() / self.nk)


def make_system(mesh=(2, 2, 2), nao=10, naux=40, ns=1, beta=100.0, nts=60, nw=None, eps_range=2.0,
                seed=0, madelung=0.0, grid: ChebyshevGrid | None = None, with_integrals: bool = True) -> System:
    rng = np.random.default_rng(seed)
    nk = int(np.prod(mesh))
    grid = grid if grid is not None else cached_grid(float(beta), int(nts), nw, nw)
    eps = rng.uniform(-eps_range, eps_range, size=(ns, nk, nao))
    U = np.empty((ns, nk, nao, nao), dtype=np.complex128)
    for s in range(ns):
        for k in range(nk):
            U[s, k] = haar_unitary(rng, nao)
    F = np.einsum("skia,ska,skja->skij", U, eps, np.conj(U))
    S = np.broadcast_to(np.eye(nao, dtype=np.complex128), (ns, nk, nao, nao)).copy()
    G = np.empty((grid.nts, ns, nk, nao, nao), dtype=np.complex128)
    for s in range(ns):
        for k in range(nk):
            f = fermi_tau(eps[s, k], grid.tau, beta)                    # [nts, nao]
            G[:, s, k] = -np.einsum("ia,ta,ja->tij", U[s, k], f, np.conj(U[s, k]))
    npair = pair_count(nk)
    sd = 1.0 / np.sqrt(2.0 * naux)
    if with_integrals:
        V = (rng.standard_normal((npair, naux, nao, nao)) + 1j * rng.standard_normal((npair, naux, nao, nao))) * sd
        for k in range(nk):
            idx = k * (k + 1) // 2 + k
            V[idx] = 0.5 * (V[idx] + np.conj(np.swapaxes(V[idx], -1, -2)))
    else:
        V = np.zeros((0, naux, nao, nao), dtype=np.complex128)
    return System(mesh=tuple(mesh), nk=nk, nao=nao, NQ=naux, ns=ns, beta=float(beta), grid=grid, eps=eps, U=U,
                  F=F, S=S, G=G, V_half=V, madelung=madelung, seed=seed)


def random_pair(rng, naux, nao, hermitian=False):
    """One V^Q_ij(k1,k2) block with the generator's distribution."""
    sd = 1.0 / np.sqrt(2.0 * naux)
    v = (rng.standard_normal((naux, nao, nao)) + 1j * rng.standard_normal((naux, nao, nao))) * sd
    return 0.5 * (v + np.conj(np.swapaxes(v, -1, -2))) if hermitian else v


def make_config(name: str, seed: int = 0, **over) -> System:
    mesh, nao, naux, ns, beta, nts, nw, er = CONFIGS[name]
    kw = dict(mesh=mesh, nao=nao, naux=naux, ns=ns, beta=beta, nts=nts, nw=nw, eps_range=er, seed=seed)
    kw.update(over)
    return make_system(**kw)


PAIR_BLOCK = 32  # stored pairs per seeded block of the device generator


def _device_pair_block(b: int, nk: int, naux: int, nao: int, seed: int, device: int):
    """Stored pairs [b PAIR_BLOCK, (b + 1) PAIR_BLOCK) of the device generator, each block from
    its own seed, so a pair has the same values whichever rank or chunk generates it."""
    import torch

    p0 = b * PAIR_BLOCK
    cnt = min(PAIR_BLOCK, pair_count(nk) - p0)
    gen = torch.Generator(device=f"cuda:{device}")
    gen.manual_seed(int(seed) * 1000003 + b)
    re = torch.randn((cnt, naux, nao, nao), dtype=torch.float64, device=f"cuda:{device}", generator=gen)
    im = torch.randn((cnt, naux, nao, nao), dtype=torch.float64, device=f"cuda:{device}", generator=gen)
    v = torch.complex(re, im) * (1.0 / np.sqrt(2.0 * naux))
    del re, im
    for k in range(nk):
        p = k * (k + 1) // 2 + k  # diagonal pairs are Hermitian per Q
        if p0 <= p < p0 + cnt:
            blk = v[p - p0]
            v[p - p0] = 0.5 * (blk + blk.conj().transpose(-1, -2))
    return v.contiguous()


def upload_device_integrals(ctx, nk: int, naux: int, nao: int, seed: int = 0, chunk_bytes: float = 2e9,
                            device: int = 0):
    """Generate V^Q_ij(k1,k2), k1 >= k2, on the GPU chunk by chunk and hand each chunk to the context.

    Same distribution as make_system (complex Gaussian with E|V|^2 = 1/naux, Hermitian
    diagonal pairs); the values come from torch's seeded CUDA generator (one seed per block of
    PAIR_BLOCK stored pairs), so they differ from the host generator's.  Nothing of size
    nk(nk+1)/2 * naux * nao^2 is ever held on the host or twice on the device.
    """
    import torch

    npair = pair_count(nk)
    pe = naux * nao * nao
    per_chunk = max(1, int(chunk_bytes // (pe * 16 * PAIR_BLOCK))) * PAIR_BLOCK
    for p0 in range(0, npair, per_chunk):
        cnt = min(per_chunk, npair - p0)
        v = torch.cat([_device_pair_block(b, nk, naux, nao, seed, device)
                       for b in range(p0 // PAIR_BLOCK, (p0 + cnt + PAIR_BLOCK - 1) // PAIR_BLOCK)])
        torch.cuda.synchronize(device)  # the context copies on its own stream
        ctx.set_integrals_device(v.data_ptr(), p0, cnt)
        torch.cuda.synchronize(device)
        del v


def upload_device_integral_pairs(ctx, nk: int, naux: int, nao: int, pair_ids, seed: int = 0, device: int = 0):
    """The stored pairs `pair_ids` (increasing) of upload_device_integrals' generator, and only
    those, as the context's q-sharded integral set (gb200_set_integrals_pairs)."""
    import torch

    ids = np.asarray(pair_ids, dtype=np.int64)
    pe = naux * nao * nao
    out = torch.empty((len(ids), naux, nao, nao), dtype=torch.complex128, device=f"cuda:{device}")
    blocks = ids // PAIR_BLOCK
    for b in np.unique(blocks):
        sel = np.nonzero(blocks == b)[0]
        v = _device_pair_block(int(b), nk, naux, nao, seed, device)
        out[torch.from_numpy(sel).to(out.device)] = v[torch.from_numpy(ids[sel] - b * PAIR_BLOCK).to(out.device)]
        del v
    torch.cuda.synchronize(device)
    ctx.set_integrals_pairs(out.data_ptr(), ids)
    torch.cuda.synchronize(device)
    del out
    return len(ids) * pe * 16
