"""Newton-Krylov self-consistency with the iteration map on the GPU (gb200_iteration_device: HF,
GW, mu search, Dyson), beside the plain iteration from the same start."""
import numpy as np
import pytest
import torch

import gw_oracle as O
from gb200 import newton, solvers
from _systems import system

pytestmark = pytest.mark.gpu


def test_newton_krylov_with_mu_search(gpu):
    s = system("small")
    g = s.grid
    with solvers.make_context(s) as c:
        G0 = torch.tensor(s.G, dtype=torch.complex128, device="cuda")
        it = newton.DeviceIteration(c, G0, nel=s.nel_from_G0(), mu=0.0, tol=1e-12)
        Gn, hist = newton.newton_krylov(it, G0, steps=8, atol=1e-11 * (1.0 + float(torch.linalg.norm(G0))))
        assert hist.residual[-1] < 1e-9
        Gp, hp = newton.plain_iteration(it, G0, 80)
        assert hp.residual[-1] < 1e-9
        assert float(torch.abs(Gn - Gp).max()) < 1e-8
        it(Gn)
        mu = it.last_mu
    # the GPU fixed point is one of the oracle's iteration map at the same chemical potential
    Gh = Gn.cpu().numpy()
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)
    dm = O.hf_density(Gh, s.ns)
    F = O.hf_scalar(dm, s.S, 0.0, integ.pair, lambda X, k: X[k], s.nk, lambda ik: ik, s.NQ)
    sig = O.gw_solve(Gh, integ, bz, g.Tnt_b, g.Ttn_b, s.ns, s.NQ)
    G1 = O.compute_G(F, sig, s.F, s.S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f)
    assert np.abs(G1 - Gh).max() < 1e-8
