"""Newton-Krylov self-consistency (gb200.newton) on the CPU: GMRES on a real-linear operator, and
Newton-Krylov against the plain iteration on the oracle's iteration map (HF, GW, Dyson at fixed mu)."""
import numpy as np
import pytest
import torch

import gw_oracle as O
from gb200 import newton
from _systems import system


def test_gmres_real_linear_operator():
    rng = np.random.default_rng(0)
    n = 40
    M = torch.from_numpy(np.eye(n) * 3 + 0.2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))))
    N = torch.from_numpy(0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))))

    def A(x):  # real-linear, not complex-linear
        return M @ x + N @ torch.conj(x)

    xt = torch.from_numpy(rng.standard_normal(n) + 1j * rng.standard_normal(n))
    b = A(xt)
    x, res, used = newton.gmres(A, b, rtol=1e-12, restart=25, maxiter=200)
    assert torch.linalg.norm(x - xt) <= 1e-9 * torch.linalg.norm(xt)
    assert used <= 200


def _oracle_phi(s, mu=0.0):
    g = s.grid
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)

    def phi(G):
        Gn = G.numpy()
        dm = O.hf_density(Gn, s.ns)
        F = O.hf_scalar(dm, s.S, 0.0, integ.pair, lambda X, k: X[k], s.nk, lambda ik: ik, s.NQ)
        sig = O.gw_solve(Gn, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
        return torch.from_numpy(O.compute_G(F, sig, s.F, s.S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f))
    return phi


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_newton_krylov_converges_quadratically(name):
    s = system(name)
    phi = _oracle_phi(s)
    G0 = torch.from_numpy(s.G.copy())
    Gn, hist = newton.newton_krylov(phi, G0, steps=6, atol=1e-12)
    r = hist.residual
    assert r[-1] < 1e-11
    # superlinear: once below 1e-2 each Newton step at least squares the relative reduction
    big = [x for x in r[1:] if 1e-9 < x < 1e-2]
    for a, b in zip(big, big[1:]):
        assert b < 10 * a * a + 1e-12
    # the plain iteration reaches the same fixed point, with more steps
    Gp, hp = newton.plain_iteration(phi, G0, 60)
    assert hp.residual[-1] < 1e-10
    assert float(torch.abs(Gn - Gp).max()) < 1e-9
    # and, with the same number of map evaluations, is still far from it
    _, hq = newton.plain_iteration(phi, G0, 8)
    assert hq.residual[-1] > 1e3 * r[-1]


def test_newton_krylov_with_mu_search_where_plain_iteration_cycles():
    """The oracle's iteration with the mu search (find_mu every iteration) on the small system: the
    plain iteration settles into a two-cycle of mu, Newton-Krylov converges."""
    s = system("small")
    g = s.grid
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)
    target = s.nel_from_G0()

    def phi(G):
        Gn = G.numpy()
        dm = O.hf_density(Gn, s.ns)
        F = O.hf_scalar(dm, s.S, 0.0, integ.pair, lambda X, k: X[k], s.nk, lambda ik: ik, s.NQ)
        sig = O.gw_solve(Gn, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
        ev = O.selfenergy_eigenspectra(F, sig, s.F, s.S, g.Tnt_f)
        _, mu = O.find_mu(0.0, target, ev, g.Ttn_beta, g.wsample_f, s.ns, 1.0 / s.nk, 1e-12)
        return torch.from_numpy(O.compute_G(F, sig, s.F, s.S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f))

    G0 = torch.from_numpy(s.G.copy())
    _, hist = newton.newton_krylov(phi, G0, steps=10, atol=1e-10)
    assert hist.residual[-1] < 1e-9
    _, hp = newton.plain_iteration(phi, G0, 30)
    assert min(hp.residual[-6:]) > 1.0
    # damped G mixing (weight 0.5) breaks the cycle and converges linearly, more slowly than Newton
    _, hm = newton.plain_iteration(phi, G0, 30, mixing=0.5)
    assert hm.residual[-1] < 1e-5
    assert hm.residual[-1] > 100 * hist.residual[-1]


def test_autograd_rejects_wrong_inputs_without_gpu():
    """gb200.autograd.gw_sigma validates dtype, device and shape before any library call."""
    from gb200 import autograd

    class FakeDims:
        nk, NQ, nao = 2, 3, 4

    class FakeContext:
        shape_G = (4, 1, 2, 4, 4)
        dims = FakeDims()

    c = FakeContext()
    with pytest.raises(TypeError):
        autograd.gw_sigma(c, torch.zeros(c.shape_G, dtype=torch.complex128))          # not on a GPU
    with pytest.raises(TypeError):
        autograd.gw_sigma(c, torch.zeros(c.shape_G, dtype=torch.complex64))


def test_newton_krylov_rejects_steps_the_map_cannot_take():
    """A map that fails (raises) outside |x| <= 1.5, and whose full Newton step from x0 lands there
    (R(x) = -atan(x), the classic overshoot): the line search halves the step instead of aborting,
    and the solve converges."""
    raised = []

    def phi(x):
        if float(torch.abs(x).max()) > 1.5:
            raised.append(1)
            raise RuntimeError("outside the admissible region")
        return x - torch.atan(x)

    x0 = torch.tensor([1.45 + 0.0j, -1.45 + 0.0j], dtype=torch.complex128)
    x, hist = newton.newton_krylov(phi, x0, steps=12, atol=1e-12, presteps=0)
    assert raised
    assert hist.residual[-1] < 1e-10
    assert float(torch.abs(x).max()) < 1e-9
