"""Newton-Krylov self-consistency with the iteration map on the GPU (gb200_iteration_device: HF,
GW, mu search, Dyson), beside the plain iteration from the same start."""
import numpy as np
import pytest
import torch

import gw_oracle as O
from gb200 import newton, solvers
from _systems import system

pytestmark = pytest.mark.gpu


def _oracle_phi(s, G, mu):
    g = s.grid
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)
    dm = O.hf_density(G, s.ns)
    F = O.hf_scalar(dm, s.S, 0.0, integ.pair, lambda X, k: X[k], s.nk, lambda ik: ik, s.NQ)
    sig = O.gw_solve(G, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
    return O.compute_G(F, sig, s.F, s.S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f)


def test_newton_krylov_fixed_mu_matches_plain_and_oracle(gpu):
    s = system("small")
    with solvers.make_context(s) as c:
        G0 = torch.tensor(s.G, dtype=torch.complex128, device="cuda")
        it = newton.DeviceIteration(c, G0, nel=None, mu=0.0)
        atol = 1e-11 * (1.0 + float(torch.linalg.norm(G0)))
        Gn, hist = newton.newton_krylov(it, G0, steps=8, atol=atol)
        Gp, hp = newton.plain_iteration(it, G0, 60)
    assert hist.residual[-1] < 1e-9
    assert hp.residual[-1] < 1e-9
    assert float(torch.abs(Gn - Gp).max()) < 1e-8
    Gh = Gn.cpu().numpy()
    assert np.abs(_oracle_phi(s, Gh, 0.0) - Gh).max() < 1e-8


def test_newton_krylov_with_mu_search(gpu):
    """With the electron count held by the mu search the plain iteration of this system falls into
    a two-cycle (mu alternating near -2.40 and -2.33, as the oracle's iteration does too); Newton-Krylov
    converges, to a fixed point of the oracle's map at the chemical potential it finds."""
    s = system("small")
    with solvers.make_context(s) as c:
        G0 = torch.tensor(s.G, dtype=torch.complex128, device="cuda")
        it = newton.DeviceIteration(c, G0, nel=s.nel_from_G0(), mu=0.0, tol=1e-12)
        atol = 1e-11 * (1.0 + float(torch.linalg.norm(G0)))
        Gn, hist = newton.newton_krylov(it, G0, steps=10, atol=atol)
        _, hp = newton.plain_iteration(it, G0, 40)
        it(Gn)
        mu = it.last_mu
    assert hist.residual[-1] < 1e-9
    assert hp.residual[-1] > 1e6 * hist.residual[-1]
    assert -2.40 < mu < -2.33
    Gh = Gn.cpu().numpy()
    assert np.abs(_oracle_phi(s, Gh, mu) - Gh).max() < 1e-8
