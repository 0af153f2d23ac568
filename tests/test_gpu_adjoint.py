"""The GPU vector-Jacobian product of Sigma[G] against the oracle's adjoint (itself checked
against finite differences of the forward in test_adjoint_cpu.py), and the torch autograd
binding built on it.

Tolerance: 1e-10 relative to the largest element, the FP64 parity bar of the forward.
"""
import numpy as np
import pytest

import gw_oracle as O
from gb200 import lib, solvers
from _systems import rel, system

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _cotangent(shape, seed=1):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_gw_vjp_matches_oracle(gpu, name):
    s = system(name)
    g = s.grid
    Sb = _cotangent(s.G.shape)
    ref = O.gw_vjp_G(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), g.Tnt_b, g.Ttn_b, s.ns, s.NQ, Sb)
    with solvers.make_context(s) as c:
        Gb = c.gw_sigma_vjp(s.G, Sb)
    assert rel(Gb, ref) < TOL


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_gw_vjp_V_matches_oracle(gpu, name):
    s = system(name)
    g = s.grid
    Sb = _cotangent(s.G.shape, 6)
    Gref, Vref = O.gw_vjp(s.G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), g.Tnt_b, g.Ttn_b, s.ns, s.NQ, Sb)
    with solvers.make_context(s) as c:
        Gb, Vb = c.gw_sigma_vjp(s.G, Sb, with_V=True)
    assert rel(Gb, Gref) < TOL
    assert rel(Vb, Vref) < TOL


def test_gw_vjp_c4_finite_differences(gpu):
    """At the differentiable-step size (nk=27, nao=20, naux=100, ntau=80) the adjoint against central
    finite differences of the GPU forward (step 1e-6) along random directions in G and in V."""
    s = system("c4")
    Sb = _cotangent(s.G.shape, 7)
    rng = np.random.default_rng(8)
    h = 1e-6
    with solvers.make_context(s) as c:
        Gb, Vb = c.gw_sigma_vjp(s.G, Sb, with_V=True)

        def loss_G(G):
            return np.real(np.vdot(Sb, c.gw_sigma(G)))

        E = _cotangent(s.G.shape, 9)
        fd = (loss_G(s.G + h * E) - loss_G(s.G - h * E)) / (2 * h)
        an = np.real(np.vdot(Gb, E))
        assert abs(fd - an) <= 1e-6 * abs(fd)

        def loss_V(V):
            c.set_integrals(V, lib.INTEGRALS_GW)
            return np.real(np.vdot(Sb, c.gw_sigma(s.G)))

        EV = rng.standard_normal(s.V_half.shape) + 1j * rng.standard_normal(s.V_half.shape)
        fd = (loss_V(s.V_half + h * EV) - loss_V(s.V_half - h * EV)) / (2 * h)
        an = np.real(np.vdot(Vb, EV))
        assert abs(fd - an) <= 1e-6 * abs(fd)


def test_gw_vjp_c4_matches_cpu_directional_derivatives(gpu):
    """At the differentiable-step size, the adjoint against central differences (step 1e-6) of the
    FP64 CPU oracle along fixed directions in G and V (tests/golden/make_c4_directional.py)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "c4_directional.json")) as f:
        d = json.load(f)
    s = system(d["config"], d["generator_seed"])
    Sb = _cotangent(s.G.shape, d["seed_cotangent"])
    EG = _cotangent(s.G.shape, d["seed_dir_G"])
    EV = _cotangent(s.V_half.shape, d["seed_dir_V"])
    with solvers.make_context(s) as c:
        Gb, Vb = c.gw_sigma_vjp(s.G, Sb, with_V=True)
    assert abs(np.real(np.vdot(Gb, EG)) - d["fd_G"]) <= 1e-6 * abs(d["fd_G"])
    assert abs(np.real(np.vdot(Vb, EV)) - d["fd_V"]) <= 1e-6 * abs(d["fd_V"])


def test_gw_vjp_linearity(gpu):
    """Sigma[G] is not complex-analytic (P0 is hermitized), so its adjoint is linear in the
    cotangent over the reals: Gb(a Sb1 + Sb2) = a Gb(Sb1) + Gb(Sb2) for real a."""
    s = system("small")
    Sb1, Sb2 = _cotangent(s.G.shape, 2), _cotangent(s.G.shape, 3)
    a = 0.7
    with solvers.make_context(s) as c:
        g1 = c.gw_sigma_vjp(s.G, Sb1)
        g2 = c.gw_sigma_vjp(s.G, Sb2)
        g12 = c.gw_sigma_vjp(s.G, a * Sb1 + Sb2)
    assert rel(g12, a * g1 + g2) < 1e-12


def test_autograd_gradient(gpu):
    torch = pytest.importorskip("torch")
    from gb200 import autograd
    s = system("small")
    Sb = _cotangent(s.G.shape, 4)
    with solvers.make_context(s) as c:
        G = torch.tensor(s.G, dtype=torch.complex128, device="cuda", requires_grad=True)
        Sigma = autograd.gw_sigma(c, G)
        loss = torch.real(torch.sum(torch.conj(torch.tensor(Sb, device="cuda")) * Sigma))
        loss.backward()
        torch.cuda.synchronize()
        assert rel(Sigma.detach().cpu().numpy(), c.gw_sigma(s.G)) < 1e-13
        assert rel(G.grad.cpu().numpy(), c.gw_sigma_vjp(s.G, Sb)) < 1e-13


def test_vjp_rejects_q0_correction(gpu):
    s = system("small")
    with solvers.make_context(s) as c:
        c.set_q0_correction(np.ones((s.nk, s.NQ), dtype=np.complex128), np.linspace(0.1, 1.0, s.nk), 0.1)
        with pytest.raises(lib.mbpt_kernel_error):
            c.gw_sigma_vjp(s.G, _cotangent(s.G.shape))


def test_autograd_gradient_V(gpu):
    torch = pytest.importorskip("torch")
    from gb200 import autograd
    s = system("small_ns2")
    Sb = _cotangent(s.G.shape, 10)
    with solvers.make_context(s) as c:
        G = torch.tensor(s.G, dtype=torch.complex128, device="cuda", requires_grad=True)
        V = torch.tensor(s.V_half, dtype=torch.complex128, device="cuda", requires_grad=True)
        Sigma = autograd.gw_sigma(c, G, V)
        loss = torch.real(torch.sum(torch.conj(torch.tensor(Sb, device="cuda")) * Sigma))
        loss.backward()
        torch.cuda.synchronize()
        Gb, Vb = c.gw_sigma_vjp(s.G, Sb, with_V=True)
        assert rel(G.grad.cpu().numpy(), Gb) < 1e-13
        assert rel(V.grad.cpu().numpy(), Vb) < 1e-13
