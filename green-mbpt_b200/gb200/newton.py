"""Newton-Krylov solution of the GW self-consistency, beside the plain iteration.

The self-consistency of green-mbpt is the fixed point G = Phi(G) of one iteration
(mbpt_run.h:199-209, dyson.cpp:290-317): Sigma1 = HF(dm(G)), Sigma = GW(G), mu from the electron
count, G <- Dyson(Sigma1, Sigma, mu).  The reference iterates Phi (with optional mixing).  Here the
residual R(G) = Phi(G) - G is driven to zero by Newton's method, each step solving
(I - J) d = R(G) with restarted GMRES; J, the Jacobian of Phi, enters only through products J v,
taken as directional differences of Phi (Phi is evaluated entirely on the GPU through
gb200_iteration_device).  Phi is not complex-analytic (hermitization, conjugated integrals), so
the Krylov solve works on the real and imaginary parts as one real vector and the inner product
is Re<a, b>.  A backtracking line search on |R| keeps the steps safe far from the solution.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


def _rdot(a: torch.Tensor, b: torch.Tensor) -> float:
    """Re <a, b> of two complex (or real) tensors."""
    if a.is_complex():
        return float(torch.sum(torch.view_as_real(a) * torch.view_as_real(b)).item())
    return float(torch.sum(a * b).item())


def _norm(a: torch.Tensor) -> float:
    return math.sqrt(max(_rdot(a, a), 0.0))


def gmres(matvec, b: torch.Tensor, rtol: float = 1e-6, restart: int = 30, maxiter: int = 60):
    """Solve A x = b for a real-linear operator A (x0 = 0) by restarted GMRES with modified
    Gram-Schmidt and Givens rotations (Saad and Schultz 1986).  Returns (x, residual norm, matvecs);
    the residual is the true one after a restart and the recurrence estimate at the exit."""
    x = torch.zeros_like(b)
    bnorm = _norm(b)
    if bnorm == 0.0:
        return x, 0.0, 0
    used = 0
    r, rnorm = b, bnorm
    while True:
        m = min(restart, maxiter - used)
        V = [r / rnorm]
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = rnorm
        n = 0
        for j in range(m):
            w = matvec(V[j])
            used += 1
            for i in range(j + 1):
                H[i, j] = _rdot(V[i], w)
                w = w - H[i, j] * V[i]
            hn = _norm(w)
            H[j + 1, j] = hn
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            d = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if d == 0.0 else (H[j, j] / d, H[j + 1, j] / d)
            H[j, j] = d
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            n = j + 1
            if abs(g[j + 1]) <= rtol * bnorm or hn == 0.0:
                break
            V.append(w / hn)
        y = np.linalg.lstsq(np.triu(H[:n, :n]), g[:n], rcond=None)[0]
        for i in range(n):
            x = x + float(y[i]) * V[i]
        est = abs(g[n])
        if est <= rtol * bnorm or used >= maxiter or m == 0:
            return x, est, used
        r = b - matvec(x)
        used += 1
        rnorm = _norm(r)
        if rnorm <= rtol * bnorm or used >= maxiter:
            return x, rnorm, used


@dataclass
class History:
    """Residual norms |Phi(G) - G| after each step and the Phi evaluations spent to reach them."""
    residual: list = field(default_factory=list)
    evaluations: list = field(default_factory=list)
    krylov: list = field(default_factory=list)


def plain_iteration(phi, G0: torch.Tensor, steps: int, mixing: float = 1.0):
    """G <- (1 - w) G + w Phi(G), `steps` times (w = `mixing`; 1 is the bare iteration, w < 1 the
    damped G mixing of green-sc's G_MIXING with weight w); the residual of step i is |Phi(G_i) - G_i|."""
    G = G0.clone()
    hist = History()
    evals = 0
    for _ in range(steps):
        G1 = phi(G)
        evals += 1
        hist.residual.append(_norm(G1 - G))
        hist.evaluations.append(evals)
        G = G1 if mixing == 1.0 else (1.0 - mixing) * G + mixing * G1
    return G, hist


def newton_krylov(phi, G0: torch.Tensor, steps: int, rtol: float = 1e-3, restart: int = 30, maxiter: int = 40,
                  fd_rel: float = 1e-7, max_backtracks: int = 6, presteps: int = 1, atol: float = 0.0):
    """Newton steps on R(G) = Phi(G) - G, after `presteps` plain steps G <- Phi(G) (the non-interacting
    start lies outside the region where Newton converges fast; one plain step brings the iterate
    into it).  Each Newton step solves (I - J) d = R(G) by GMRES to the relative tolerance `rtol`
    (tightened as the residual falls, Eisenstat-Walker choice 2), with
    J v = (Phi(G + h v) - Phi(G)) / h, h = fd_rel (1 + |G|) / |v|; then G <- G + lam d with lam halved
    until |R| decreases.  Stops early once |R| <= atol.  Returns (G, History); History.residual[i]
    is |Phi(G_i) - G_i| for the iterate after i steps (plain and Newton steps counted alike)."""
    G = G0.clone()
    hist = History()
    evals = 0
    PG = phi(G)
    evals += 1
    for _ in range(presteps):
        hist.residual.append(_norm(PG - G))
        hist.evaluations.append(evals)
        hist.krylov.append(0)
        G = PG
        PG = phi(G)
        evals += 1
    R = PG - G
    rn = _norm(R)
    eta = rtol
    rn_prev = None
    for _ in range(steps):
        hist.residual.append(rn)
        hist.evaluations.append(evals)
        if rn <= atol:
            break
        gnorm = _norm(G)

        def matvec(v, G=G, PG=PG, gnorm=gnorm):
            nonlocal evals
            vn = _norm(v)
            if vn == 0.0:
                return torch.zeros_like(v)
            h = fd_rel * (1.0 + gnorm) / vn
            Jv = (phi(G + h * v) - PG) / h
            evals += 1
            return v - Jv

        if rn_prev is not None:
            eta = min(rtol, max(0.9 * (rn / rn_prev) ** 2, 1e-10))
        d, _, used = gmres(matvec, R, rtol=eta, restart=restart, maxiter=maxiter)
        hist.krylov.append(used)
        lam = 1.0
        Gt = PGt = Rt = None
        rt = math.inf
        for _ in range(max_backtracks + 1):
            Gt = G + lam * d
            try:
                PGt = phi(Gt)
            except RuntimeError:
                # a trial point the iteration cannot take (e.g. the chemical-potential search fails
                # for an unphysical G far from the solution) counts as a rejected step
                PGt = None
            evals += 1
            if PGt is not None:
                Rt = PGt - Gt
                rt = _norm(Rt)
                if rt < (1.0 - 1e-4 * lam) * rn:
                    break
            lam *= 0.5
        if PGt is None:
            raise RuntimeError("newton_krylov: no admissible step along the Newton direction")
        rn_prev = rn
        G, PG, R, rn = Gt, PGt, Rt, rt
    else:
        hist.residual.append(rn)
        hist.evaluations.append(evals)
    return G, hist


class DeviceIteration:
    """Phi(G) on the GPU: one gb200_iteration_device call (HF, GW, mu search, Dyson) on a copy of G.

    context: a prepared lib.Context (maps, grid, integrals, Hamiltonian); nel: the electron count
    (None keeps mu fixed at `mu`).  Every evaluation starts the mu search from the same `mu`, so that
    directional differences of nearby points see the same bisection; the mu found last is `last_mu`."""

    def __init__(self, context, G_like: torch.Tensor, madelung: float = 0.0, nel: float | None = None,
                 mu: float = 0.0, tol: float = 1e-12):
        self.c = context
        self.madelung = float(madelung)
        self.nel = -1.0 if nel is None else float(nel)
        self.mu = float(mu)
        self.tol = float(tol)
        d = context.dims
        self.Sigma1 = torch.empty((d.ns, d.nk, d.nso, d.nso), dtype=torch.complex128, device=G_like.device)
        self.Sigma = torch.empty_like(G_like)
        self.last_mu = self.mu
        self.calls = 0

    def __call__(self, G: torch.Tensor) -> torch.Tensor:
        out = G.contiguous().clone()
        stream = torch.cuda.current_stream().cuda_stream or 0x1
        mu, _ = self.c.iteration_device(out.data_ptr(), self.Sigma1.data_ptr(), self.Sigma.data_ptr(),
                                        self.madelung, self.nel, self.tol, self.mu, stream=stream, energies=False)
        self.last_mu = mu
        self.calls += 1
        return out
