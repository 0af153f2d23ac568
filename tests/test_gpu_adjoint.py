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
