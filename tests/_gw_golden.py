"""The reference's GW fixtures (tests/golden/gw.npz, written by tests/golden/make_golden.py).

Three cases of the reference's GW self-energy test (test/solvers_test.cpp:80-135,389-391):
``gw`` (H2 chain, 3x3x3 mesh with full point-group symmetry: 4 irreducible k-points, ns = 2,
nao = 2, NQ = 36), ``gw_c`` (the same system with time-reversal symmetry only, 14 irreducible
points, and the "extrapolate" q -> 0 correction) and ``gw_x2c`` (a two-component molecule,
nso = 20, NQ = 154).  All run on the 110 tau points of the green-grids IR file ``ir/1e4.h5`` at
beta = 100, for which the transforms come from gb200.grids.SampledGrid.
"""
from __future__ import annotations

import functools
import os

import numpy as np

import gw_oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("gw", "gw_c", "gw_x2c")
REF_TOL = 1e-6  # IsCloseTo(..., 1e-6): absolute, elementwise (solvers_test.cpp:134, tensor_test.h)


@functools.lru_cache(maxsize=None)
def _npz():
    return dict(np.load(os.path.join(HERE, "gw.npz")))


@functools.lru_cache(maxsize=None)
def grid():
    from gb200 import grids
    z = _npz()
    return grids.SampledGrid(z["tau"], float(z["beta"]), float(z["wmax"]))


def case(name: str) -> dict:
    z = _npz()
    p = name + "/"
    d = {k[len(p):]: v for k, v in z.items() if k.startswith(p)}
    ns, nk, nao, nso, NQ = (int(x) for x in d["dims"])
    d.update(ns=ns, nk=nk, nao=nao, nso=nso, NQ=NQ, X2C=(nso == 2 * nao), beta=float(z["beta"]))
    return d


def ref_symmetry(d) -> O.RefSymmetry:
    return O.RefSymmetry(d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
                         d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])


def oracle_full_from_ibz(sym: O.RefSymmetry, X):
    """[..., ink, n, n] -> [..., nk, n, n] through the oracle's value_AO."""
    lead = X.shape[:-3]
    flat = X.reshape((-1,) + X.shape[-3:])
    out = np.stack([np.stack([sym.value_AO(flat[b], k) for k in range(sym.nk)]) for b in range(flat.shape[0])])
    return out.reshape(lead + out.shape[1:])


@functools.lru_cache(maxsize=None)
def oracle_sigma(name: str):
    """The oracle's Sigma_tau at the irreducible points for the fixture's G_tau."""
    d = case(name)
    g = grid()
    sym = ref_symmetry(d)
    G = oracle_full_from_ibz(sym, d["G_tau"])

    class Ints:
        def pair(self, k1, k2):
            return sym.integral(d["V_chunk"], k1, k2)

    q0 = None
    if "AqQ" in d:
        A = np.zeros((d["nk"], d["NQ"]), dtype=np.complex128)
        qa = np.zeros(d["nk"])
        A[d["q_ibz2bz"]] = d["AqQ"]
        qa[d["q_ibz2bz"]] = d["q_abs"]
        q0 = (A, qa, float(d["madelung"]), oracle_full_from_ibz(sym, d["S_ibz"]))
    S = O.gw_solve(G, Ints(), O.PointsBZ(d["k_frac"]), g.Tnt_b, g.Ttn_b, d["ns"], d["NQ"], X2C=d["X2C"], q0=q0)
    return S[:, :, d["ibz2bz"]]


def product_inputs(d):
    """The dictionary of gb200.inputs.read_input for a fixture case (for solvers.context_from_arrays)."""
    from gb200 import inputs
    sym = inputs.KSymmetry(d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
                           d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])
    return dict(nk=d["nk"], nao=d["nao"], nso=d["nso"], ns=d["ns"], NQ=d["NQ"], symmetry=sym, k_frac=d["k_frac"],
                S_ibz=d["S_ibz"], H_ibz=d["H_ibz"], madelung=float(d["madelung"]))
