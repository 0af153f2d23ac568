"""The CPU oracle against the reference's own HF golden fixtures.

The fixtures were extracted from green-mbpt test/data/{HF,HF_X2C} by
tests/golden/make_golden.py; the reference test compares Sigma1 at 1e-10
(test/solvers_test.cpp:27-78,387-388, tensor_test.h:41).
"""
import os

import numpy as np
import pytest

import gw_oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = dict(np.load(os.path.join(HERE, name + ".npz")))
    sym = O.RefSymmetry(d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
                        d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])
    return d, sym


def test_hf_scalar_golden():
    d, sym = load("hf")
    ns, nk, NQ = int(d["ns"]), int(d["nk"]), int(d["NQ"])
    dm = O.hf_density(d["G_beta"][None], ns)
    F = O.hf_scalar(dm, d["S_ibz"], float(d["madelung"]), lambda a, b: sym.integral(d["V_chunk"], a, b),
                    sym.value_AO, nk, sym.full_point, NQ)
    np.testing.assert_allclose(F, d["Sigma1"], rtol=0, atol=1e-10)


def test_hf_x2c_golden():
    d, sym = load("hf_x2c")
    nk, NQ, nao = int(d["nk"]), int(d["NQ"]), int(d["nao"])
    dm = O.hf_density(d["G_beta"][None], int(d["ns"]), X2C=True)
    F = O.hf_x2c(dm, d["S_ibz"], float(d["madelung"]), lambda a, b: sym.integral(d["V_chunk"], a, b),
                 sym.value_AO, nk, sym.full_point, NQ, nao)
    np.testing.assert_allclose(F, d["Sigma1"], rtol=0, atol=1e-10 * max(1.0, np.abs(d["Sigma1"]).max()))


def test_golden_integral_version():
    for name in ("hf", "hf_x2c"):
        d, _ = load(name)
        assert bytes(d["version"]).decode() == "1.0.0"


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's input must break the golden match."""
    d, sym = load("hf")
    ns, nk, NQ = int(d["ns"]), int(d["nk"]), int(d["NQ"])
    dm = O.hf_density(d["G_beta"][None], ns)
    dm[0, 1, 0, 1] += 1e-6
    F = O.hf_scalar(dm, d["S_ibz"], float(d["madelung"]), lambda a, b: sym.integral(d["V_chunk"], a, b),
                    sym.value_AO, nk, sym.full_point, NQ)
    assert np.abs(F - d["Sigma1"]).max() > 1e-10


ORTH_BASES = ("none", "lowdin", "mo", "natural")


def orth_case(d, basis):
    ns, nk, nao, nso, NQ = (int(x) for x in d[f"{basis}/dims"])
    V = d[f"{basis}/V_chunk"].reshape(-1, NQ, nso, nso)
    return ns, nk, NQ, V


def test_hf_orth_invariance_golden():
    """HF part of the reference's orth-invariance test (test/solvers_test.cpp:296-430) on one H2
    molecule written in four orbital bases: from each basis's G(beta), the oracle's Fock matrix
    equals the reference run's iter1/Sigma1, E_1b and E_HF + E_nuc equal the energies it wrote
    (dyson.cpp:325-326), and both energies agree across the bases, all to 1e-10."""
    d = dict(np.load(os.path.join(HERE, "hf_orth.npz")))
    E = {}
    for basis in ORTH_BASES:
        ns, nk, NQ, V = orth_case(d, basis)
        dm = O.hf_density(d[f"{basis}/G_beta"][None], ns)
        F = O.hf_scalar(dm, d[f"{basis}/S"], float(d[f"{basis}/madelung"]), lambda a, b: V[0], lambda X, k: X[k],
                        nk, lambda ik: ik, NQ)
        np.testing.assert_allclose(F, d[f"{basis}/Sigma1"], rtol=0, atol=1e-10)
        G = d[f"{basis}/G_beta"][None]
        e1, ehf, ec = O.compute_energy(G, F, np.zeros_like(G), d[f"{basis}/H"], np.ones((1, 1)), np.ones(1), 1.0 / nk)
        assert ec == 0.0
        assert abs(e1 - float(d[f"{basis}/Energy_1b"])) < 1e-10
        assert abs(ehf + float(d[f"{basis}/E_nuc"]) - float(d[f"{basis}/Energy_HF"])) < 1e-10
        E[basis] = (e1, ehf)
    for basis in ORTH_BASES[1:]:
        assert abs(E[basis][0] - E["none"][0]) < 1e-10
        assert abs(E[basis][1] - E["none"][1]) < 1e-10
