"""Host-side mirror of green-mbpt's solver interface on top of the C ABI.

The reference wires its kernels as
  gw_solver(p, ft, bz, S_k).solve(G, Sigma1, Sigma_tau)   (gw_solver.h:61-72, gw_solver.cpp:30-32)
  hf_solver(p, bz, S_k).solve(G, Sigma1, Sigma_tau)       (hf_solver.h:27-43, hf_solver.cpp:9-16)
  dyson(p).solve(G, Sigma1, Sigma_tau); dyson.diff(...)   (dyson.cpp:290-317)
These classes keep the same names, call order, argument meaning and error
classes; the arrays are numpy complex128 with the reference's index order.
"""
from __future__ import annotations

import numpy as np

from . import lib
from .synth import System


def kq_maps(mesh):
    """k1_from_k2q / k2_from_k1q tables of a Monkhorst-Pack mesh without symmetry."""
    n1, n2, n3 = mesh
    nk = n1 * n2 * n3
    idx = np.arange(nk)
    f = np.stack([idx // (n2 * n3), (idx // n3) % n2, idx % n3], axis=1)

    def index(v):
        v = np.mod(v, (n1, n2, n3))
        return v[..., 0] * n2 * n3 + v[..., 1] * n3 + v[..., 2]

    kplus = index(f[:, None, :] + f[None, :, :]).astype(np.int32)   # [k, q] -> k + q
    kminus = index(f[:, None, :] - f[None, :, :]).astype(np.int32)  # [k, q] -> k - q
    return kplus, kminus


def make_context(system: System, device: int = 0, precision: int = lib.PREC_FP64, slices: int = 4,
                 hf_integrals=None) -> lib.Context:
    """Context with maps, grid, integrals and Hamiltonian of a synthetic system uploaded."""
    g = system.grid
    ctx = lib.Context(system.nk, system.nao, system.ns, system.NQ, g.nts, g.nw, g.nw_b, system.beta, device=device)
    kp, km = kq_maps(system.mesh)
    ctx.set_kq_maps(kp, km)
    ctx.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
    ctx.set_integrals(system.V_half, lib.INTEGRALS_GW)
    if hf_integrals is not None:
        ctx.set_integrals(hf_integrals, lib.INTEGRALS_HF)
    ctx.set_hamiltonian(system.F, system.S)
    ctx.set_precision(precision, slices)
    return ctx


def context_from_files(input_path: str, hf_integrals: str | None = None, gw_integrals: str | None = None,
                       grid=None, beta: float | None = None, device: int = 0, q0_file: str | None = None):
    """A context for a system written in green-mbpt's file format.

    input_path: input.h5 (parameters, Hamiltonian blocks, k-point symmetry); hf_integrals /
    gw_integrals: the integral directories (meta.h5 + VQ_<c>.h5) of the HF and GW kernels.
    Objects at irreducible k-points and irreducible k-pair integrals are expanded to the full
    zone on the host (inputs.KSymmetry).  `grid` (a grids.ChebyshevGrid or any object with
    Tnt_f, Ttn_f, Tnt_b, Ttn_b, wsample_f, nts, nw, nw_b) is needed for GW and the Dyson step.
    q0_file: an AqQ.h5 switches on the "extrapolate" q -> 0 correction (irreducible q-points
    of the input's q symmetry; the Madelung constant of the input).
    Returns (context, input dictionary).
    """
    from . import inputs
    inp = inputs.read_input(input_path)
    npairs = len(inp["symmetry"].kpair_irre)
    hf = inputs.read_integrals(hf_integrals, npairs)[0] if hf_integrals else None
    gw = inputs.read_integrals(gw_integrals, npairs)[0] if gw_integrals else None
    q0 = None
    if q0_file:
        from .h5lite import H5File
        A, q_abs, _ = inputs.read_q0(q0_file)
        q0 = (A, q_abs, np.asarray(H5File(input_path).read("symmetry/q/ibz2bz")))
    return context_from_arrays(inp, hf, gw, grid, beta, device, q0)


def context_from_arrays(inp: dict, hf_store=None, gw_store=None, grid=None, beta: float | None = None,
                        device: int = 0, q0=None):
    """The context of context_from_files from arrays already in memory.

    inp: the dictionary of inputs.read_input (nk, nao, nso, ns, NQ, symmetry as an
    inputs.KSymmetry, and optionally k_frac, S_ibz, H_ibz, madelung); hf_store / gw_store: the
    irreducible k-pair blocks [npairs, NQ, nao, nao] of the integral files; q0: (AqQ, q_abs,
    q_ibz2bz) at the irreducible q-points for the "extrapolate" q -> 0 correction.
    Returns (context, inp) with the full-zone S and H added to inp.
    """
    from . import inputs
    sym = inp["symmetry"]
    nk, nao, nso, ns, NQ = inp["nk"], inp["nao"], inp["nso"], inp["ns"], inp["NQ"]
    if grid is not None:
        ctx = lib.Context(nk, nao, ns, NQ, grid.nts, grid.nw, grid.nw_b, float(beta if beta is not None else grid.beta),
                          nso=nso, device=device)
        ctx.set_grid(grid.Tnt_f, grid.Ttn_f, grid.Tnt_b, grid.Ttn_b, grid.wsample_f)
    else:
        ctx = lib.Context(nk, nao, ns, NQ, 2, 2, 3, float(beta or 1.0), nso=nso, device=device)
    try:
        if inp.get("k_frac") is not None:
            kp, km = inputs.kq_maps_from_points(inp["k_frac"])
            ctx.set_kq_maps(kp, km)
        if hf_store is not None:
            ctx.set_integrals(sym.half_storage(hf_store), lib.INTEGRALS_HF)
        if gw_store is not None:
            ctx.set_integrals(sym.half_storage(gw_store), lib.INTEGRALS_GW)
        if q0 is not None:
            A, q_abs, ibz2bz_q = q0
            Af, qf = inputs.q0_full_zone(A, q_abs, ibz2bz_q, nk)
            ctx.set_q0_correction(Af, qf, inp.get("madelung", 0.0))
        if "S_ibz" in inp:
            inp["S"] = sym.full_from_ibz(inp["S_ibz"])
        if "H_ibz" in inp:
            inp["H"] = sym.full_from_ibz(inp["H_ibz"])
            if "S" in inp:
                ctx.set_hamiltonian(inp["H"], inp["S"])
    except BaseException:
        ctx.close()
        raise
    return ctx, inp


class gw_solver:
    """GW self-energy through the B200 kernel (custom_gw_kernel callback)."""

    def __init__(self, ctx: lib.Context):
        self.ctx = ctx

    def solve(self, G, Sigma1, Sigma_tau):
        Sigma_tau[...] = self.ctx.gw_sigma(G)


class hf_solver:
    """Hartree-Fock through the B200 kernel (custom_hf_kernel callback)."""

    def __init__(self, ctx: lib.Context, S, madelung: float, ns: int, X2C: bool = False):
        if ns != 1 and X2C:
            raise ValueError('For GSCF methods, "ns" has to be 1.')
        self.ctx = ctx
        self.S = np.ascontiguousarray(S, dtype=np.complex128)
        self.madelung = float(madelung)
        self.spin_prefactor = -1.0 if (ns == 2 or X2C) else -2.0   # hf_solver.h:38

    def solve(self, G, Sigma1, Sigma_tau):
        dm = self.spin_prefactor * np.ascontiguousarray(G[-1])
        Sigma1[...] = self.ctx.hf_fock(dm, self.S, self.madelung)


class dyson:
    """Dyson step: find_mu (if const_density) then compute_G; diff() returns |dE|."""

    def __init__(self, ctx: lib.Context, nel: float, mu: float = 0.0, tol: float = 1e-9, const_density: bool = True):
        self.ctx = ctx
        self.nel = float(nel)
        self.mu = float(mu)
        self.tol = float(tol)
        self.const_density = const_density
        self.E = (0.0, 0.0, 0.0)

    def solve(self, G, Sigma1, Sigma_tau):
        if self.const_density:
            _, self.mu = self.ctx.find_mu(Sigma1, Sigma_tau, self.mu, self.nel, self.tol)
        Gn, S1h, Sth = self.ctx.compute_G(Sigma1, Sigma_tau, self.mu)
        G[...] = Gn
        Sigma1[...] = S1h
        Sigma_tau[...] = Sth

    def diff(self, G, Sigma1, Sigma_tau):
        e = self.ctx.energy(G, Sigma1, Sigma_tau)
        d = sum(abs(a - b) for a, b in zip(e, self.E))
        self.E = e
        return d
