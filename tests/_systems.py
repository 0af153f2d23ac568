"""Shared small systems for the parity tests (seeded, built once per process)."""
import functools

import numpy as np

import gw_oracle as O
from gb200 import synth

SMALL = dict(mesh=(2, 2, 1), nao=6, naux=20, ns=1, beta=20.0, nts=20, eps_range=2.0)
SMALL_NS2 = dict(mesh=(2, 1, 2), nao=5, naux=16, ns=2, beta=20.0, nts=24, eps_range=2.0)


@functools.lru_cache(maxsize=None)
def system(name, seed=0):
    if name == "small":
        return synth.make_system(seed=seed, **SMALL)
    if name == "small_ns2":
        return synth.make_system(seed=seed, **SMALL_NS2)
    if name == "odd_mesh":
        return synth.make_system(mesh=(3, 1, 1), nao=7, naux=18, ns=1, beta=15.0, nts=16, eps_range=1.5, seed=seed)
    return synth.make_config(name, seed=seed)


@functools.lru_cache(maxsize=None)
def oracle_sigma(name, seed=0):
    s = system(name, seed)
    bz = O.NoSymBZ(s.mesh)
    return O.gw_solve(s.G, O.HalfStoredIntegrals(s.V_half), bz, s.grid.Tnt_b, s.grid.Ttn_b, s.ns, s.NQ)


def oracle_fock(s, madelung=0.0):
    dm = O.hf_density(s.G, s.ns)
    integ = O.HalfStoredIntegrals(s.V_half)
    return O.hf_scalar(dm, s.S, madelung, integ.pair, lambda X, k: X[k], s.nk, lambda ik: ik, s.NQ)


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
