"""The adjoint of Sigma[G] in the oracle against central finite differences (CPU).

Sigma[G] has no derivative in the reference; its adjoint is checked against finite differences
of the forward restatement, and the GPU adjoint (test_gpu_adjoint.py) against this one.
"""
import numpy as np
import pytest

import gw_oracle as O
from _systems import system


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_oracle_vjp_matches_finite_differences(name):
    s = system(name)
    g = s.grid
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)
    rng = np.random.default_rng(1)
    Sb = rng.standard_normal(s.G.shape) + 1j * rng.standard_normal(s.G.shape)
    Gb = O.gw_vjp_G(s.G, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ, Sb)

    def loss(G):
        return np.real(np.sum(np.conj(Sb) * O.gw_solve(G, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)))

    h = 1e-6
    for _ in range(2):
        E = rng.standard_normal(s.G.shape) + 1j * rng.standard_normal(s.G.shape)
        fd = (loss(s.G + h * E) - loss(s.G - h * E)) / (2 * h)
        an = np.real(np.sum(np.conj(Gb) * E))
        assert abs(fd - an) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_oracle_vjp_V_matches_finite_differences(name):
    s = system(name)
    g = s.grid
    bz = O.NoSymBZ(s.mesh)
    rng = np.random.default_rng(5)
    Sb = rng.standard_normal(s.G.shape) + 1j * rng.standard_normal(s.G.shape)
    Gb, Vb = O.gw_vjp(s.G, O.HalfStoredIntegrals(s.V_half), bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ, Sb)
    assert Vb.shape == s.V_half.shape

    def loss(V):
        Sig = O.gw_solve(s.G, O.HalfStoredIntegrals(V), bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
        return np.real(np.sum(np.conj(Sb) * Sig))

    h = 1e-6
    for _ in range(2):
        E = rng.standard_normal(s.V_half.shape) + 1j * rng.standard_normal(s.V_half.shape)
        fd = (loss(s.V_half + h * E) - loss(s.V_half - h * E)) / (2 * h)
        an = np.real(np.sum(np.conj(Vb) * E))
        assert abs(fd - an) <= 1e-6 * abs(fd)

