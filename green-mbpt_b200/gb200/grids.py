"""Imaginary-time / Matsubara grids and the dense transforms the kernels use.

The reference obtains every tau <-> i omega operation from green-grids'
``transformer_t`` (an external package; call sites gw_cpu_kernel.cpp:234,264,
dyson.cpp:61,76,205,213,219, common_utils.cpp:22,31-32).  The library takes
those operations as dense FP64 matrices, so any grid works; this module builds
one for synthetic workloads:

* tau nodes: the ``ncheb = nts - 2`` Chebyshev roots mapped to (0, beta) plus
  the two endpoints 0 and beta (nts = ncoeff + 2 as in the reference tests,
  solvers_test.cpp:56-59).  The grid is mirror symmetric, tau[nts-1-t] =
  beta - tau[t], which the polarization needs (gw_cpu_kernel.cpp:171,223).
* functions of tau are represented by their Chebyshev interpolant through the
  interior nodes.
* the Matsubara sampling frequencies are chosen by column-pivoted QR of the
  exact Fourier transforms of the Chebyshev basis over a large candidate set
  (the sparse-sampling idea), which keeps the fitting matrix well conditioned
  (cond ~ 1e2-1e3) instead of the ~1e9-1e16 of the lowest frequencies.

Matrices (row-major, complex128):
  Tnt_f [nw, nts]   tau -> fermionic i omega_n   (tau_to_omega)
  Ttn_f [nts, nw]   fermionic i omega_n -> tau   (omega_to_tau, Ttn())
  Tnt_b [nwb, nts]  tau -> bosonic i Omega_m     (tau_f_to_w_b); nwb is odd
  Ttn_b [nts, nwb]  bosonic i Omega_m -> tau     (w_b_to_tau_f)
"""
from __future__ import annotations

import functools

import numpy as np


def _chebyshev_nodes(nts: int, beta: float):
    n = nts - 2
    j = np.arange(n)
    x = np.cos(np.pi * (j + 0.5) / n)[::-1]
    x = 0.5 * (x - x[::-1])  # exact antisymmetry of the roots
    tau = np.concatenate([[0.0], beta * (x + 1.0) / 2.0, [beta]])
    half = nts // 2
    tau[nts - half:] = beta - tau[:half][::-1]
    return x, tau


def _composite_gauss(nseg: int, p: int = 64):
    g, w = np.polynomial.legendre.leggauss(p)
    e = np.linspace(-1.0, 1.0, nseg + 1)
    X = ((e[:-1, None] + e[1:, None]) / 2 + (e[1:, None] - e[:-1, None]) / 2 * g).ravel()
    W = ((e[1:, None] - e[:-1, None]) / 2 * w).ravel()
    return X, W


def chebyshev_fourier(omega: np.ndarray, ncheb: int, beta: float) -> np.ndarray:
    """M[n, l] = int_0^beta exp(i omega_n tau) T_l(2 tau/beta - 1) d tau (composite Gauss-Legendre)."""
    zmax = float(np.max(np.abs(omega))) * beta / 2 if len(omega) else 0.0
    nseg = max(64, int(np.ceil(zmax / 16.0)))
    X, W = _composite_gauss(nseg)
    T = np.polynomial.chebyshev.chebvander(X, ncheb - 1) * W[:, None]
    out = np.empty((len(omega), ncheb), dtype=np.complex128)
    step = max(1, int(4e7 // len(X)))
    for i in range(0, len(omega), step):
        ph = np.exp(1j * np.outer(omega[i:i + step] * beta / 2, X + 1.0))
        out[i:i + step] = (beta / 2) * (ph @ T)
    return out


def _select_frequencies(ncheb, beta, count, bosonic, candidates):
    """Pick sampling frequencies in conjugate pairs (+w, -w) by pivoted QR.

    Functions of tau here are Hermitian-matrix valued, so F(-i w) = F(i w)^H;
    sampling in conjugate pairs keeps every transformed quantity Hermitian in
    tau.  Pivoting runs on the real/imaginary rows of the non-negative
    frequencies; the bosonic set always contains Omega = 0 and therefore has
    an odd size.
    """
    m = np.arange(0, candidates)
    omega_pos = (2 * m + (0 if bosonic else 1)) * np.pi / beta
    Mpos = chebyshev_fourier(omega_pos, ncheb, beta)
    # each candidate frequency contributes two real rows (Re, Im); greedy block
    # selection maximizes the residual norm of those rows against the span of
    # the rows already chosen (a block version of column-pivoted QR)
    rows = np.stack([Mpos.real, Mpos.imag], axis=1)             # [cand, 2, L]
    Q = np.zeros((ncheb, 0))
    if bosonic:
        q0 = rows[0, 0] / np.linalg.norm(rows[0, 0])
        Q = q0[:, None]
    avail = np.ones(len(m), dtype=bool)
    avail[0] = not bosonic
    chosen = []
    half = count // 2
    for _ in range(half):
        res = rows - np.einsum("fri,ij,kj->frk", rows, Q, Q, optimize=True)
        score = np.where(avail, np.einsum("fri,fri->f", res, res), -1.0)
        f = int(np.argmax(score))
        chosen.append(f)
        avail[f] = False
        for r in res[f]:
            r = r - Q @ (Q.T @ r)
            nr = np.linalg.norm(r)
            if nr > 1e-12 * np.linalg.norm(rows[f]) and Q.shape[1] < ncheb:
                Q = np.concatenate([Q, (r / nr)[:, None]], axis=1)
    pos = np.sort(np.array(chosen, dtype=int))
    if bosonic:
        n = np.concatenate([-pos[::-1], [0], pos])
        omega = 2 * n * np.pi / beta
    else:
        n = np.concatenate([-pos[::-1] - 1, pos])
        omega = (2 * n + 1) * np.pi / beta
    return n, omega, chebyshev_fourier(omega, ncheb, beta)


class ChebyshevGrid:
    """Chebyshev tau grid with pivoted sparse Matsubara sampling for both statistics."""

    def __init__(self, beta: float, nts: int, nw: int | None = None, nw_b: int | None = None, candidates: int | None = None):
        if nts % 2 != 0:
            raise ValueError("Number of tau points should be even")
        self.beta = float(beta)
        self.nts = int(nts)
        self.ncheb = nts - 2
        nw = int(nw if nw is not None else nts)
        nw_b = int(nw_b if nw_b is not None else nw)
        if nw % 2 != 0:
            raise ValueError("the fermionic sample count must be even (conjugate pairs)")
        if nw < self.ncheb or nw_b < self.ncheb:
            raise ValueError("need at least ncheb Matsubara samples")
        cand = int(candidates if candidates is not None else max(512, self.ncheb ** 2 // 3))
        x, self.tau = _chebyshev_nodes(nts, beta)
        L = self.ncheb
        # Chebyshev coefficients from the interior nodes: c = Cint @ f_interior
        Tx = np.polynomial.chebyshev.chebvander(x, L - 1)          # [L nodes, L polys]
        Cint = (2.0 / L) * Tx.T
        Cint[0] *= 0.5
        self.C = np.zeros((L, nts))
        self.C[:, 1:nts - 1] = Cint
        self.T_tau = np.polynomial.chebyshev.chebvander(2 * self.tau / beta - 1, L - 1)  # [nts, L]
        self.n_f, self.wsample_f, Mf = _select_frequencies(L, beta, nw, False, cand)
        self.n_b, self.wsample_b, Mb = _select_frequencies(L, beta, nw_b, True, cand)
        self.nw = len(self.n_f)
        self.nw_b = len(self.n_b)
        self.Tnt_f = Mf @ self.C
        self.Ttn_f = self.T_tau @ np.linalg.pinv(Mf)
        self.Tnt_b = Mb @ self.C
        self.Ttn_b = self.T_tau @ np.linalg.pinv(Mb)
        self.cond_f = float(np.linalg.cond(Mf))
        self.cond_b = float(np.linalg.cond(Mb))

    @property
    def Ttn_beta(self):
        """Row of Ttn at tau = beta (dyson.cpp:76, common_utils.cpp:16)."""
        return self.Ttn_f[-1]

    def chebyshev_coefficients(self, F_tau):
        nts = F_tau.shape[0]
        return (self.C @ F_tau.reshape(nts, -1)).reshape((self.ncheb,) + F_tau.shape[1:])

    def leakage(self, F_tau) -> float:
        """max|c_last| / max|c_first|: the resolution diagnostic of transformer_t::check_chebyshev."""
        c = self.chebyshev_coefficients(F_tau)
        first = np.abs(c[0]).max()
        return float(np.abs(c[-1]).max() / first) if first > 0 else 0.0


def _omega_quadrature(wmax: float, beta: float, p: int = 64):
    """Composite Gauss-Legendre nodes and weights on [-wmax, wmax], segments doubling in length from
    |omega| = 1/(8 beta) outward (the kernels vary on the scale 1/beta near 0 and 1/tau_min far out)."""
    edges = [0.0, 1.0 / (8.0 * beta)]
    while edges[-1] < wmax:
        edges.append(min(2.0 * edges[-1], wmax))
    e = np.array(edges)
    g, w = np.polynomial.legendre.leggauss(p)
    X = ((e[:-1, None] + e[1:, None]) / 2 + (e[1:, None] - e[:-1, None]) / 2 * g).ravel()
    W = ((e[1:, None] - e[:-1, None]) / 2 * w).ravel()
    return np.concatenate([-X[::-1], X]), np.concatenate([W[::-1], W])


def fermi_kernel_tau(tau, omega, beta):
    """exp(-tau w) / (1 + exp(-beta w)) without overflow: [len(tau), len(omega)]."""
    t, w = np.asarray(tau)[:, None], np.asarray(omega)[None, :]
    pos = w >= 0
    a = np.exp(-t * np.where(pos, w, 0.0)) / (1.0 + np.exp(-beta * np.where(pos, w, 0.0)))
    wn = np.where(pos, 0.0, w)
    b = np.exp((beta - t) * wn) / (1.0 + np.exp(beta * wn))
    return np.where(pos, a, b)


def bose_kernel_tau(tau, omega, beta):
    """w exp(-tau w) / (1 - exp(-beta w)) (finite, 1/beta at w = 0) without overflow."""
    t, w = np.asarray(tau)[:, None], np.asarray(omega)[None, :]
    aw = np.abs(w)
    small = aw * beta < 1e-12
    wsafe = np.where(small, 1.0, w)
    # w > 0: w e^{-t w} / (1 - e^{-beta w});  w < 0: |w| e^{(beta - t) w} / (1 - e^{beta w})
    num = np.where(w > 0, np.exp(-t * np.where(w > 0, w, 0.0)), np.exp((beta - t) * np.where(w < 0, w, 0.0)))
    den = -np.expm1(-beta * np.abs(wsafe))
    out = np.abs(wsafe) * num / den
    return np.where(small, 1.0 / beta, out)


class SampledGrid:
    """Transforms for given imaginary-time sampling points (for example the points of a green-grids
    IR grid file, which green-mbpt's own result files record as the mesh of G_tau).

    A function of tau is represented by its spectral form F(tau) = int K(tau, w) rho(w) dw over
    |w| <= wmax, with the fermionic kernel exp(-tau w)/(1 + exp(-beta w)) or the bosonic one
    w exp(-tau w)/(1 - exp(-beta w)) on a composite Gauss-Legendre w grid.  The Matsubara transform
    of a kernel column is known in closed form (int_0^beta e^{i w_n tau} K dtau = 1/(w - i w_n), and
    w/(w - i W_n) for bosons), so tau -> i w_n is (K_iw pinv(K_tau)) and i w_n -> tau is
    (K_tau pinv(K_iw)), both pseudo-inverses truncated at `rcut` of the largest singular value and
    applied through the singular vectors (never formed as matrices of size 1/s_min).
    Functions whose spectra lie in the window are reproduced whatever frequencies are sampled, which
    is what makes results on these points comparable with a calculation that used the IR basis of
    the same window.  Sampling frequencies: every Matsubara index up to `ndense`, then geometrically
    spaced ones up to about wmax * `wfac`, in conjugate pairs."""

    def __init__(self, tau, beta: float, wmax: float, ndense: int = 128, ngeo: int = 64, wfac: float = 20.0,
                 rcut: float = 1e-15):
        tau = np.asarray(tau, dtype=np.float64)
        if len(tau) % 2 != 0:
            raise ValueError("Number of tau points should be even")
        self.tau, self.beta, self.wmax = tau, float(beta), float(wmax)
        self.nts = len(tau)
        X, W = _omega_quadrature(self.wmax, self.beta)
        sw = np.sqrt(W)
        nmax = max(ndense + 1, int(np.ceil(self.wmax * wfac * self.beta / (2 * np.pi))))
        geo = np.unique(np.round(np.geomspace(ndense + 1, nmax, ngeo)).astype(int))
        pos = np.concatenate([np.arange(ndense + 1), geo[geo > ndense]])
        # bosonic: 0 and +-n; fermionic: n >= 0 and their partners -n-1
        self.n_b = np.concatenate([-pos[:0:-1], pos])
        self.n_f = np.concatenate([-pos[::-1] - 1, pos])
        self.wsample_b = 2 * np.pi * self.n_b / self.beta
        self.wsample_f = (2 * self.n_f + 1) * np.pi / self.beta
        self.nw, self.nw_b = len(self.n_f), len(self.n_b)

        def apply_pinv(L, K):
            # L pinv(K) grouped as ((L V) / s) U^H: L V ~ s (the transform's own basis) stays moderate,
            # while pinv(K) alone has entries ~ 1 / s_min and would cancel catastrophically
            U, S, Vh = np.linalg.svd(K, full_matrices=False)
            r = int((S > rcut * S[0]).sum())
            return ((L @ np.conj(Vh[:r]).T) / S[:r]) @ np.conj(U[:, :r]).T

        def transforms(Ktau, Kiw):
            Ktau, Kiw = Ktau * sw, Kiw * sw
            return apply_pinv(Kiw, Ktau), apply_pinv(Ktau, Kiw)

        Kf_iw = 1.0 / (X[None, :] - 1j * self.wsample_f[:, None])
        self.Tnt_f, self.Ttn_f = transforms(fermi_kernel_tau(tau, X, self.beta), Kf_iw)
        Wb = self.wsample_b[:, None]
        Kb_iw = np.where(np.abs(X[None, :]) + np.abs(Wb) > 0, X[None, :] / (X[None, :] - 1j * Wb + (X[None, :] == 0) * (Wb == 0)), 1.0)
        self.Tnt_b, self.Ttn_b = transforms(bose_kernel_tau(tau, X, self.beta), Kb_iw)

    @property
    def Ttn_beta(self):
        """Row of Ttn at tau = beta (dyson.cpp:76, common_utils.cpp:16)."""
        return self.Ttn_f[-1]


@functools.lru_cache(maxsize=8)
def cached_grid(beta: float, nts: int, nw: int | None = None, nw_b: int | None = None) -> ChebyshevGrid:
    return ChebyshevGrid(beta, nts, nw, nw_b)
