"""FP64 CPU oracle for the density-fitted GW / HF / Dyson path of green-mbpt.

TEST INFRASTRUCTURE ONLY.  The CUDA library's results are compared against this
module; only tests, the smoke check and the CPU-baseline leg of the benchmark
may import it.  The library never calls it.

It restates, in numpy (complex128, BLAS zgemm through ``@``), the reference's
algorithm with the same contraction order, prefactors, signs and loop
structure.  Each function cites the reference file:line it follows
(paths relative to the green-mbpt project root).

Parity status
-------------
* HF (``hf_scalar``/``hf_x2c``) and the DF integral access with full k-point
  symmetry (``RefSymmetry``) are pinned against the reference's own golden
  fixtures (test/data/HF, HF_X2C, HF_orth_invariance) at 1e-10 — see
  tests/test_oracle_golden.py.
* The GW self-energy (P0 -> W -> Sigma, with and without the "extrapolate"
  q -> 0 correction, scalar and two-component) is pinned against the
  reference's three GW fixtures (test/data/GW data.h5 and data_c.h5,
  test/data/GW_X2C): the fixture's G_tau, replayed on transforms built for the
  fixture's own IR tau points (gb200.grids.SampledGrid; the green-grids file
  ``ir/1e4.h5`` itself is external), reproduces ``result/Sigma_tau`` within
  the reference test's absolute 1e-6 (measured 8.9e-9, 2.8e-11, 1.2e-11) —
  see tests/test_gw_golden.py.
* The Dyson step follows the same reference code and is pinned by identities
  (G0 reproduction, the chemical-potential search's electron count).

Array conventions (row-major, as the reference):
  G, Sigma : [nts, ns, nk, nso, nso]            (mbpt_run.h:260-263)
  V pair   : [NQ, nao, nao] for an ordered k-pair (k1, k2)
  dm, F, S : [ns, nk, nso, nso]
  transforms are dense matrices (the green-grids transformer is external):
    Tnt_f [nw, nts], Ttn_f [nts, nw]   fermionic tau <-> i omega
    Tnt_b [nwb, nts], Ttn_b [nts, nwb] tau -> bosonic i Omega and back
"""
from __future__ import annotations

import numpy as np


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------
def make_hermitian(X):
    """X = (X + X^H)/2 over the two innermost dims (common_defs.h:104-115)."""
    return 0.5 * (X + np.conj(np.swapaxes(X, -1, -2)))


class NoSymBZ:
    """Monkhorst-Pack mesh without point-group symmetry.

    Mirrors the parts of green-symmetry's brillouin_zone_utils used on the hot
    path when every k is irreducible (ink = nk, value_AO = identity, star(q) =
    {q}).  k_q_map semantics: k1_from_k2q(k2, q) = k2 + q, k2_from_k1q(k1, q)
    = k1 - q, q_from_k1k2(k1, k2) = k1 - k2 (all modulo the mesh).
    """

    def __init__(self, mesh):
        self.mesh = tuple(int(m) for m in mesh)
        n1, n2, n3 = self.mesh
        self.nk = n1 * n2 * n3
        idx = np.arange(self.nk)
        self.frac = np.stack([idx // (n2 * n3), (idx // n3) % n2, idx % n3], axis=1)

    def _index(self, f):
        n1, n2, n3 = self.mesh
        f = np.mod(f, self.mesh)
        return int(f[0] * n2 * n3 + f[1] * n3 + f[2])

    def k1_from_k2q(self, k2, q):
        return self._index(self.frac[k2] + self.frac[q])

    def k2_from_k1q(self, k1, q):
        return self._index(self.frac[k1] - self.frac[q])

    def q_from_k1k2(self, k1, k2):
        return self._index(self.frac[k1] - self.frac[k2])

    def kplus_table(self):
        """table[k, q] = k1_from_k2q(k, q)."""
        return np.array([[self.k1_from_k2q(k, q) for q in range(self.nk)] for k in range(self.nk)], dtype=np.int32)

    def kminus_table(self):
        """table[k, q] = k2_from_k1q(k, q)."""
        return np.array([[self.k2_from_k1q(k, q) for q in range(self.nk)] for k in range(self.nk)], dtype=np.int32)


class PointsBZ(NoSymBZ):
    """The k_q_map of a mesh given by the fractional coordinates of its points (an input file's
    symmetry/k/mesh_scaled), in the file's own point order: k + q and k - q are looked up modulo
    reciprocal lattice vectors (the same semantics as NoSymBZ)."""

    def __init__(self, frac):
        self.f = np.asarray(frac, dtype=np.float64).reshape(-1, 3)
        self.nk = len(self.f)

    def _lookup(self, v):
        d = self.f - v
        d = np.abs(d - np.round(d)).max(axis=1)
        i = int(np.argmin(d))
        if d[i] > 1e-6:
            raise ValueError("k-point set is not closed under addition")
        return i

    def k1_from_k2q(self, k2, q):
        return self._lookup(self.f[k2] + self.f[q])

    def k2_from_k1q(self, k1, q):
        return self._lookup(self.f[k1] - self.f[q])

    def q_from_k1k2(self, k1, k2):
        return self._lookup(self.f[k1] - self.f[k2])


def pair_index(k1, k2):
    """Stored k-pair index, k1 >= k2 only (df_integral_t.h:68)."""
    return k1 * (k1 + 1) // 2 + k2 if k1 >= k2 else k2 * (k2 + 1) // 2 + k1


class HalfStoredIntegrals:
    """V^Q_ij(k1,k2) stored only for k1 >= k2, no k-pair symmetry lists.

    ``store`` has shape [nk(nk+1)/2, NQ, nao, nao].  For k1 < k2 the block is
    the per-Q conjugate transpose of the stored (k2, k1) block
    (df_integral_t.h:162-177 with v_type sign < 0 and symmetry type 'direct').
    """

    def __init__(self, store):
        self.store = store

    def pair(self, k1, k2):
        v = self.store[pair_index(k1, k2)]
        if k1 >= k2:
            return v.copy()
        return np.conj(np.swapaxes(v, -1, -2))


class RefSymmetry:
    """k-point and k-pair symmetry as stored in green-mbpt input files.

    Used to replay the reference's golden fixtures.  Reproduces
    ``k_symmetry().value_AO`` and ``df_integral_t::read_integrals`` /
    ``symmetrize`` / ``wrap`` / ``v_type`` (df_integral_t.h:64-84,140-203).
    """

    def __init__(self, bz2ibz, ibz2bz, tr_conj, transform_ao, conj_pairs, trans_pairs, kpair_irre, weight_ibz):
        self.bz2ibz = np.asarray(bz2ibz)
        self.ibz2bz = np.asarray(ibz2bz)
        self.tr_conj = np.asarray(tr_conj)
        self.U = np.asarray(transform_ao)
        self.conj_pairs = np.asarray(conj_pairs)
        self.trans_pairs = np.asarray(trans_pairs)
        self.irre_pos = {int(v): i for i, v in enumerate(np.asarray(kpair_irre))}
        self.weight = np.asarray(weight_ibz)
        self.nk = len(self.bz2ibz)
        self.ink = len(self.ibz2bz)
        self._ibz_pos = {int(v): i for i, v in enumerate(self.ibz2bz)}

    def full_point(self, ik):
        return int(self.ibz2bz[ik])

    def reduced_point(self, k):
        return self._ibz_pos[int(self.bz2ibz[k])]

    def value_AO(self, X_ibz, k):
        """Object at full-BZ point k from its irreducible image: U X U^H, conj if TR."""
        Y = X_ibz[self.reduced_point(k)]
        U = self.U[k]
        Y = U @ Y @ np.conj(U.T)
        if self.tr_conj[k]:
            Y = np.conj(Y)
        return Y

    def _resolved(self, k1, k2):
        idx = pair_index(k1, k2)
        if self.conj_pairs[idx] != idx:
            return int(self.conj_pairs[idx]), "conj", idx
        if self.trans_pairs[idx] != idx:
            return int(self.trans_pairs[idx]), "trans", idx
        return idx, "direct", idx

    def integral(self, store, k1, k2):
        """df_integral_t::symmetrize for one (k1, k2) from the irreducible chunk."""
        red, kind, _ = self._resolved(k1, k2)
        v = store[self.irre_pos[red]]
        v = np.conj(np.swapaxes(v, -1, -2)) if k1 < k2 else v.copy()
        if kind == "conj":
            v = np.conj(v)
        elif kind == "trans":
            v = np.swapaxes(v, -1, -2).copy()
        return v


# ----------------------------------------------------------------------------
# GW self-energy (gw_cpu_kernel.cpp)
# ----------------------------------------------------------------------------
def p0_contraction(Gb, Gq, v, P0, prefactor):
    """One (q, k, tau, spin) term of the polarization (gw_cpu_kernel.cpp:200-215).

    X1[t,(m,Q)] = Gb[t,p] V^Q[p,m];  X2[(Q',t),m] = conj(V^{Q'}[t,n]) Gq[m,n];
    P0^T -= pref * X2mm @ X1mm.
    """
    NQ, nao, _ = v.shape
    VVm = v.reshape(NQ, nao * nao).T.copy()            # (pm, Q)
    X1 = Gb @ VVm.reshape(nao, nao * NQ)               # (t, mQ)
    X2 = np.conj(v.reshape(NQ * nao, nao)) @ Gq.T      # (Q't, m)
    P0 -= prefactor * (X2.reshape(NQ, nao * nao) @ X1.reshape(nao * nao, NQ)).T


def eval_P0_tilde(G, v, k1, k1q, P0, ns, X2C=False):
    """Loop over the first half of the tau grid (gw_cpu_kernel.cpp:143-190)."""
    nts = G.shape[0]
    nso = G.shape[-1]
    nao = v.shape[-1]
    pns = nso // nao
    prefactor = 1.0 if (ns == 2 or X2C) else 2.0
    pseudo_ns = ns if not X2C else 4
    for t in range(nts // 2):
        tt = nts - t - 1
        for s in range(pseudo_ns):
            is_ = s // (pns * pns)
            a = (s // pns) % pns
            b = s % pns
            Gb = G[tt, is_, k1][b * nao:(b + 1) * nao, a * nao:(a + 1) * nao]
            Gq = G[t, is_, k1q][a * nao:(a + 1) * nao, b * nao:(b + 1) * nao]
            p0_contraction(Gb, Gq, v, P0[t], prefactor)


def hermitian_from_lower(A):
    """Hermitian matrix defined by the strict lower triangle and the real diagonal of A."""
    L = np.tril(A, -1)
    return L + np.conj(L.T) + np.diag(np.real(np.diag(A)))


def symmetrize_P0(P0, nk):
    """P0/=nk, hermitize, P0(beta-tau)=P0(tau) (gw_cpu_kernel.cpp:217-225)."""
    nts = P0.shape[0]
    for it in range(nts // 2):
        P0[it] = make_hermitian(P0[it] / nk)
        P0[nts - it - 1] = P0[it]


def eval_P_tilde(P0, Tnt_b, Ttn_b, return_w=False):
    """tau -> i Omega, (I - P0)^-1 P0 per frequency, back to tau (gw_cpu_kernel.cpp:227-279).

    The reference inverts with Eigen's LDLT (:245-249), which reads only the
    lower triangle and the real part of the diagonal of (I - P0(i Omega)); the
    same Hermitian matrix is formed here (``hermitian_from_lower``) and
    inverted, then the inverse is hermitized (:250) and multiplied (:251).
    """
    nts, NQ, _ = P0.shape
    Pw = (Tnt_b @ P0.reshape(nts, NQ * NQ)).reshape(-1, NQ, NQ)
    I = np.eye(NQ, dtype=np.complex128)
    for n in range(Pw.shape[0]):
        temp = np.linalg.solve(hermitian_from_lower(I - Pw[n]), I)
        temp = 0.5 * (temp + np.conj(temp.T))
        Pw[n] = temp @ Pw[n]
    Pt = (Ttn_b @ Pw.reshape(Pw.shape[0], NQ * NQ)).reshape(nts, NQ, NQ)
    return (Pt, Pw) if return_w else Pt


# ----------------------------------------------------------------------------
# q -> 0 correction (mbpt_q0_utils_t.cpp, "extrapolate" treatment)
# ----------------------------------------------------------------------------
def q0_head(Pw, Aq):
    """eps_inv[n] = conj(Aq) . P(i Omega_n) . Aq (aux_to_PW_00, mbpt_q0_utils_t.cpp:11-20)."""
    return np.array([np.conj(Aq) @ Pw[n] @ Aq for n in range(Pw.shape[0])])


def extrapolate_q0(X, q_abs, fit_order=2, q_max=1.0):
    """q -> 0 limit of Re X(q): quadratic least-squares fit over the first occurrences of the
    distinct |q| in (0, q_max], normal equations (extrapolate_q0 / filter_q_abs / polyfit,
    mbpt_q0_utils_t.cpp:30-86)."""
    seen, idx = set(), []
    for i, qa in enumerate(q_abs):
        if 0.0 < qa <= q_max and qa not in seen:
            seen.add(qa)
            idx.append(i)
    x = np.array([q_abs[i] for i in idx])
    y = np.array([np.real(X[i]) for i in idx])
    A = np.vander(x, fit_order + 1, increasing=True)
    c = np.linalg.solve(A.T @ A, A.T @ y)
    return c[0]


def q0_correction(eps_inv_wq, q_abs, Ttn_b, G, S, madelung, X2C=False):
    """Delta Sigma(t) = -madelung eps_inv_q0(t) S G(t) S (GW_q0_correction / apply_q0_correction
    and apply_q0_correction_2C, mbpt_q0_utils_t.cpp:88-178).  eps_inv_wq: [nw_b, nq]; the
    extrapolated head is taken to tau with the bosonic-to-fermionic-tau transform."""
    e_w = np.array([extrapolate_q0(eps_inv_wq[n], q_abs) for n in range(eps_inv_wq.shape[0])], dtype=np.complex128)
    e_t = Ttn_b @ e_w
    nts, ns, nk, nso, _ = G.shape
    D = np.zeros_like(G)
    if not X2C:
        for t in range(nts):
            for s in range(ns):
                for k in range(nk):
                    D[t, s, k] = -madelung * e_t[t] * (S[s, k] @ G[t, s, k] @ S[s, k])
        return D
    nao = nso // 2
    for t in range(nts):
        for k in range(nk):
            Sa = S[0, k, :nao, :nao]
            Gm = G[t, 0, k]
            D[t, 0, k, :nao, :nao] = -madelung * e_t[t] * (Sa @ Gm[:nao, :nao] @ Sa)
            D[t, 0, k, nao:, nao:] = -madelung * e_t[t] * (Sa @ Gm[nao:, nao:] @ Sa)
            off = madelung * e_t[t] * (Sa @ Gm[:nao, nao:] @ Sa)
            D[t, 0, k, :nao, nao:] = -off
            D[t, 0, k, nao:, :nao] = -np.conj(off.T)
    return D


def selfenergy_contraction(Gq, v, P):
    """Sigma_ij = sum V^Q_im G_mn P_QQ' conj(V^Q'_jn) (gw_cpu_kernel.cpp:359-373)."""
    NQ, nao, _ = v.shape
    vm = v.reshape(NQ * nao, nao)
    Y1 = vm @ Gq                                       # (Qi, n)
    Y2 = Y1.reshape(NQ, nao * nao).T @ P               # (in, Q')
    X2 = np.conj(vm.T)                                 # (n, Q'j)
    return Y2.reshape(nao, nao * NQ) @ X2.reshape(nao * NQ, nao)


def eval_selfenergy(G, v, k1, k1mq, P, Sigma, ns, X2C=False):
    """Loop over all tau (gw_cpu_kernel.cpp:295-354); Sigma block -= contraction."""
    nts = G.shape[0]
    nso = G.shape[-1]
    nao = v.shape[-1]
    pns = nso // nao
    pseudo_ns = ns if not X2C else 4
    for t in range(nts):
        for s in range(pseudo_ns):
            is_ = s // (pns * pns)
            a = (s // pns) % pns
            b = s % pns
            Gq = G[t, is_, k1mq][a * nao:(a + 1) * nao, b * nao:(b + 1) * nao]
            Sigma[t, is_, k1, a * nao:(a + 1) * nao, b * nao:(b + 1) * nao] -= selfenergy_contraction(Gq, v, P[t])


def gw_solve(G, integrals, bz, Tnt_b, Ttn_b, ns, NQ, X2C=False, q_list=None, k_list=None, return_P=False,
             q0=None):
    """gw_cpu_kernel::solve for the no-symmetry case (gw_cpu_kernel.cpp:31-72,74-134).

    ``integrals.pair(k1, k2)`` returns V(k1,k2) [NQ, nao, nao].
    ``q_list``/``k_list`` restrict the work to a sample (CPU-baseline timing);
    with the defaults the full self-energy is returned, already divided by nk.
    ``q0 = (AqQ [nq, NQ], q_abs [nq], madelung, S [ns, nk, nso, nso])`` adds the
    "extrapolate" q -> 0 correction (gw_cpu_kernel.cpp:58-64,267-270).
    """
    nts = G.shape[0]
    if nts % 2 != 0:
        raise ValueError("Number of tau points should be even!!!")
    nk = bz.nk
    Sigma = np.zeros_like(G)
    Ps = {}
    eps_cols = {}
    qs = range(nk) if q_list is None else q_list
    ks = range(nk) if k_list is None else k_list
    for q in qs:
        P0 = np.zeros((nts, NQ, NQ), dtype=np.complex128)
        for k1 in ks:
            k1q = bz.k1_from_k2q(k1, q)
            eval_P0_tilde(G, integrals.pair(k1, k1q), k1, k1q, P0, ns, X2C)
        symmetrize_P0(P0, nk)
        if q0 is not None:
            P, Pw = eval_P_tilde(P0, Tnt_b, Ttn_b, return_w=True)
            eps_cols[q] = q0_head(Pw, q0[0][q])
        else:
            P = eval_P_tilde(P0, Tnt_b, Ttn_b)
        if return_P:
            Ps[q] = P
        for k1 in ks:
            k1mq = bz.k2_from_k1q(k1, q)
            eval_selfenergy(G, integrals.pair(k1, k1mq), k1, k1mq, P, Sigma, ns, X2C)
    Sigma /= nk
    if q0 is not None:
        AqQ, q_abs, madelung, S = q0
        eps = np.stack([eps_cols[q] for q in range(nk)], axis=1)  # [nw_b, nq]
        Sigma += q0_correction(eps, q_abs, Ttn_b, G, S, madelung, X2C)
    return (Sigma, Ps) if return_P else Sigma


def herm(X):
    return 0.5 * (X + np.conj(np.swapaxes(X, -1, -2)))


def hermitian_from_lower_adjoint(Ab):
    """Adjoint (real inner product Re<a, b>) of X -> hermitian_from_lower(X)."""
    n = Ab.shape[-1]
    Xb = np.zeros_like(Ab)
    low = np.tril_indices(n, -1)
    Xb[low] = Ab[low] + np.conj(Ab.T[low])
    Xb[np.diag_indices(n)] = np.real(np.diag(Ab))
    return Xb


def gw_vjp_G(G, integrals, bz, Tnt_b, Ttn_b, ns, NQ, Sigma_bar):
    """Vector-Jacobian product of the GW self-energy (gw_solve, no X2C, no q0) with respect to G.

    With L = Re sum conj(Sigma_bar) Sigma(G), returns Gbar such that dL = Re sum conj(Gbar) dG
    for every complex perturbation dG (real and imaginary parts independent).  This is not a
    restatement of the reference (which has no derivatives); it is the adjoint of the forward
    restatement above, step by step, and is checked against central finite differences.
    """
    return gw_vjp(G, integrals, bz, Tnt_b, Ttn_b, ns, NQ, Sigma_bar, with_V=False)[0]


def fold_pair_gradient(Vbar_full):
    """Gradient with respect to the half-stored integrals [nk(nk+1)/2, NQ, nao, nao] from the one of
    the full pair set [nk, nk, NQ, nao, nao]: the (k2, k1) block, k1 > k2, is the per-Q conjugate
    transpose of the stored (k1, k2) block (HalfStoredIntegrals.pair), so its gradient enters the
    stored block conjugate-transposed."""
    nk = Vbar_full.shape[0]
    out = np.zeros((nk * (nk + 1) // 2,) + Vbar_full.shape[2:], dtype=np.complex128)
    for k1 in range(nk):
        for k2 in range(k1 + 1):
            g = Vbar_full[k1, k2].copy()
            if k1 != k2:
                g += np.conj(np.swapaxes(Vbar_full[k2, k1], -1, -2))
            out[pair_index(k1, k2)] = g
    return out


def gw_vjp(G, integrals, bz, Tnt_b, Ttn_b, ns, NQ, Sigma_bar, with_V=True):
    """Vector-Jacobian product of the GW self-energy with respect to G and to the half-stored
    integrals: returns (Gbar, Vbar_half or None), dL = Re sum conj(Gbar) dG + Re sum conj(Vbar) dV
    for L = Re sum conj(Sigma_bar) Sigma(G, V).  V enters Sigma through the pair V(k, k - q) twice
    (V^Q and conj(V^Q')) and P0 through the pair V(k, k + q) twice, each one a term below."""
    nts = G.shape[0]
    nth = nts // 2
    nk = bz.nk
    pref = 1.0 if ns == 2 else 2.0
    Gbar = np.zeros_like(G)
    Vbar = None
    if with_V:
        nao = G.shape[-1]
        Vbar = np.zeros((nk, nk, NQ, nao, nao), dtype=np.complex128)
    I = np.eye(NQ, dtype=np.complex128)
    for q in range(nk):
        # ---- forward of this q (recomputed) ----
        P0 = np.zeros((nts, NQ, NQ), dtype=np.complex128)
        for k1 in range(nk):
            k1q = bz.k1_from_k2q(k1, q)
            eval_P0_tilde(G, integrals.pair(k1, k1q), k1, k1q, P0, ns)
        symmetrize_P0(P0, nk)
        nwb = Tnt_b.shape[0]
        Pw = (Tnt_b @ P0.reshape(nts, NQ * NQ)).reshape(nwb, NQ, NQ)
        T = np.empty_like(Pw)
        Th = np.empty_like(Pw)
        Ptw = np.empty_like(Pw)
        for n in range(nwb):
            T[n] = np.linalg.solve(hermitian_from_lower(I - Pw[n]), I)
            Th[n] = herm(T[n])
            Ptw[n] = Th[n] @ Pw[n]
        W = (Ttn_b @ Ptw.reshape(nwb, NQ * NQ)).reshape(nts, NQ, NQ)
        # ---- Sigma = -(1/nk) sum_QQ' W_QQ' V^Q G V^Q'^H ----
        Wbar = np.zeros_like(W)
        for k1 in range(nk):
            k1mq = bz.k2_from_k1q(k1, q)
            v = integrals.pair(k1, k1mq)
            vh = np.conj(np.swapaxes(v, -1, -2))
            for t in range(nts):
                for s_ in range(ns):
                    Gq = G[t, s_, k1mq]
                    Sb = Sigma_bar[t, s_, k1]
                    # Gbar += -(1/nk) sum_QQ' conj(W_QQ') V^Q^H Sb V^Q'
                    A = np.einsum("qim,ij->qmj", np.conj(v), Sb)           # (V^Q^H Sb)[m][j]
                    Y = np.einsum("Qjn,qmj->qQmn", v, A)                   # (V^Q^H Sb V^Q')[m][n]
                    Gbar[t, s_, k1mq] += -(1.0 / nk) * np.einsum("qQ,qQmn->mn", np.conj(W[t]), Y)
                    # Wbar_QQ' += -(1/nk) tr(V^Q^H Sb V^Q' G^H)
                    Wbar[t] += -(1.0 / nk) * np.einsum("qQmn,mn->qQ", Y, np.conj(Gq))
                    if with_V:
                        # Vbar^Q += -(1/nk) Sb sum_Q' conj(W_QQ') V^Q' G^H
                        F = np.einsum("qQ,Qjn,mn->qjm", np.conj(W[t]), v, np.conj(Gq))
                        Vbar[k1, k1mq] += -(1.0 / nk) * np.einsum("ij,qjm->qim", Sb, F)
                        # Vbar^Q' += -(1/nk) sum_Q W_QQ' Sb^H V^Q G
                        H = np.einsum("ij,qim,mn->qjn", np.conj(Sb), v, Gq)
                        Vbar[k1, k1mq] += -(1.0 / nk) * np.einsum("qQ,qjn->Qjn", W[t], H)
        # ---- W = Ttn_b Ptw ----
        Ptw_bar = (np.conj(Ttn_b).T @ Wbar.reshape(nts, NQ * NQ)).reshape(nwb, NQ, NQ)
        Pw_bar = np.zeros_like(Pw)
        for n in range(nwb):
            Th_bar = Ptw_bar[n] @ np.conj(Pw[n].T)
            Pw_bar[n] = np.conj(Th[n].T) @ Ptw_bar[n]
            T_bar = herm(Th_bar)
            TH = np.conj(T[n].T)
            A_bar = -TH @ T_bar @ TH
            Pw_bar[n] += -hermitian_from_lower_adjoint(A_bar)
        # ---- Pw = Tnt_b P0;  P0 = symmetrize(P0h) ----
        P0_bar = (np.conj(Tnt_b).T @ Pw_bar.reshape(nwb, NQ * NQ)).reshape(nts, NQ, NQ)
        P0h_bar = np.zeros_like(P0_bar)
        for t in range(nth):
            P0h_bar[t] = herm(P0_bar[t] + P0_bar[nts - 1 - t]) / nk
        # ---- P0h_QQ' = -pref sum_{k,s} tr(V^Q'^H Gb V^Q G1), Gb = G(beta - t, k), G1 = G(t, k + q) ----
        for k1 in range(nk):
            k1q = bz.k1_from_k2q(k1, q)
            v = integrals.pair(k1, k1q)
            vh = np.conj(np.swapaxes(v, -1, -2))
            for t in range(nth):
                tt = nts - 1 - t
                for s_ in range(ns):
                    Gb = G[tt, s_, k1]
                    G1 = G[t, s_, k1q]
                    Pb = P0h_bar[t]
                    # Gb_bar = -pref sum_QQ' Pb_QQ' V^Q' G1^H V^Q^H
                    X = np.einsum("Qrn,mn->Qrm", v, np.conj(G1))            # V^Q' G1^H
                    Gbar[tt, s_, k1] += -pref * np.einsum("qQ,Qrm,qmp->rp", Pb, X, vh)
                    # G1_bar = -pref sum_QQ' Pb_QQ' V^Q^H Gb^H V^Q'
                    Z = np.einsum("qmp,rp->qmr", vh, np.conj(Gb))           # V^Q^H Gb^H
                    Gbar[t, s_, k1q] += -pref * np.einsum("qQ,qmr,Qrn->mn", Pb, Z, v)
                    if with_V:
                        # Vbar^Q += -pref Gb^H R^Q G1^H, R^Q = sum_Q' Pb_QQ' V^Q'
                        R = np.einsum("qQ,Qrn->qrn", Pb, v)
                        Vbar[k1, k1q] += -pref * np.einsum("rp,qrn,mn->qpm", np.conj(Gb), R, np.conj(G1))
                        # Vbar^Q' += -pref sum_Q conj(Pb_QQ') Gb V^Q G1
                        Bt = np.einsum("rp,qpm,mn->qrn", Gb, v, G1)
                        Vbar[k1, k1q] += -pref * np.einsum("qQ,qrn->Qrn", np.conj(Pb), Bt)
    return Gbar, (fold_pair_gradient(Vbar) if with_V else None)


# ----------------------------------------------------------------------------
# Hartree-Fock (hf_solver.cpp, hf_cpu_kernels.cpp)
# ----------------------------------------------------------------------------
def hf_density(G, ns, X2C=False):
    """dm = spin_prefactor * G(tau=beta) (hf_solver.cpp:9-16, hf_solver.h:38)."""
    return (-1.0 if (ns == 2 or X2C) else -2.0) * G[-1].copy()


def hf_scalar(dm, S, madelung, integral, value_AO, nk, full_point, NQ):
    """hf_scalar_cpu_kernel::solve (hf_cpu_kernels.cpp:25-146), single rank.

    integral(k1, k2) -> V [NQ, nao, nao]; value_AO(X_ibz, k) -> X at full k;
    full_point(ik) -> full-BZ index of irreducible point ik.
    dm, S: [ns, ink, nao, nao].  Returns F [ns, ink, nao, nao].
    """
    ns, ink, nao, _ = dm.shape
    F = np.zeros_like(dm)
    upper = np.zeros(NQ, dtype=np.complex128)
    for ikps in range(nk * ns):                        # :47-59
        is_ = ikps % ns
        ikp = ikps // ns
        v = integral(ikp, ikp).reshape(NQ, nao * nao)
        X1 = value_AO(dm[is_], ikp).T
        upper += v @ X1.reshape(nao * nao)
    upper /= nk                                        # :65
    for ii in range(ink * ns):                         # :67-80
        is_ = ii // ink
        ik = ii % ink
        k_ir = full_point(ik)
        v = integral(k_ir, k_ir).reshape(NQ, nao * nao)
        F[is_, ik] += (upper @ v).reshape(nao, nao)
    prefactor = 1.0 if ns == 2 else 0.5                # :98
    for ii in range(ink * ns):                         # :101-124
        is_ = ii // ink
        ik = ii % ink
        k_ir = full_point(ik)
        for ikp in range(nk):
            dmm = value_AO(dm[is_], ikp)
            v = integral(k_ir, ikp)
            vmm = v.reshape(NQ * nao, nao)
            Y = (vmm @ dmm).reshape(NQ, nao * nao)     # (Q, ia)
            Y1 = Y.T.copy().reshape(nao, nao * NQ)     # (i, aQ)
            v2 = np.conj(vmm).T.copy().reshape(nao * NQ, nao)  # (aQ, j)
            F[is_, ik] -= prefactor * (Y1 @ v2) / nk
    for ii in range(ns * ink):                         # :128-137
        is_ = ii // ink
        ik = ii % ink
        F[is_, ik] -= prefactor * madelung * S[is_, ik] @ dm[is_, ik] @ S[is_, ik]
    return F


def hf_x2c(dm, S, madelung, integral, value_AO, nk, full_point, NQ, nao):
    """hf_x2c_cpu_kernel::solve (hf_cpu_kernels.cpp:148-279), single rank, ns = 1."""
    _, ink, nso, _ = dm.shape
    F = np.zeros((1, ink, nso, nso), dtype=np.complex128)
    upper = np.zeros(NQ, dtype=np.complex128)
    for ikp in range(nk):
        v = integral(ikp, ikp).reshape(NQ, nao * nao)
        d = value_AO(dm[0], ikp)
        X1 = (d[:nao, :nao] + d[nao:, nao:]).T
        upper += v @ X1.reshape(nao * nao)
    upper /= nk
    for ik in range(ink):
        k_ir = full_point(ik)
        v = integral(k_ir, k_ir).reshape(NQ, nao * nao)
        Fm = (upper @ v).reshape(nao, nao)
        F[0, ik, :nao, :nao] += Fm
        F[0, ik, nao:, nao:] += Fm
    for ik in range(ink):
        k_ir = full_point(ik)
        Saa = S[0, ik, :nao, :nao]
        dm_nso = dm[0, ik]
        Faa = np.zeros((nao, nao), dtype=np.complex128)
        Fbb = np.zeros_like(Faa)
        Fab = np.zeros_like(Faa)
        for ikp in range(nk):
            v = integral(k_ir, ikp)
            vmm = v.reshape(NQ * nao, nao)
            dmk = value_AO(dm[0], ikp)
            v2 = np.conj(vmm).T.copy().reshape(nao * NQ, nao)
            for blk, acc in (((0, 0), Faa), ((1, 1), Fbb), ((0, 1), Fab)):
                d = dmk[blk[0] * nao:(blk[0] + 1) * nao, blk[1] * nao:(blk[1] + 1) * nao]
                Y = (vmm @ d).reshape(NQ, nao * nao)
                acc -= (Y.T.copy().reshape(nao, nao * NQ) @ v2) / nk
        F[0, ik, :nao, :nao] += Faa - madelung * Saa @ dm_nso[:nao, :nao] @ Saa
        F[0, ik, nao:, nao:] += Fbb - madelung * Saa @ dm_nso[nao:, nao:] @ Saa
        Fab = Fab - madelung * Saa @ dm_nso[:nao, nao:] @ Saa
        F[0, ik, :nao, nao:] += Fab
        F[0, ik, nao:, :nao] = np.conj(F[0, ik, :nao, nao:].T)
    return F


# ----------------------------------------------------------------------------
# Dyson step, chemical potential, energies (dyson.cpp, common_utils.cpp)
# ----------------------------------------------------------------------------
def compute_G(Sigma1, Sigma_tau, H, S, mu, Tnt_f, Ttn_f, wsample_f):
    """dyson::compute_G (dyson.cpp:238-288): hermitize, tau->iw, invert, iw->tau.

    Returns (G_tau, leakage-free) ; Sigma1/H/S: [ns, nk, nso, nso].
    """
    Sigma1 = make_hermitian(Sigma1)
    Sigma_tau = make_hermitian(Sigma_tau)
    nts, ns, nk, nso, _ = Sigma_tau.shape
    nw = Tnt_f.shape[0]
    G = np.zeros_like(Sigma_tau)
    for is_ in range(ns):
        for ik in range(nk):
            Sw = (Tnt_f @ Sigma_tau[:, is_, ik].reshape(nts, nso * nso)).reshape(nw, nso, nso)
            z = 1j * wsample_f + mu
            A = z[:, None, None] * S[is_, ik][None] - H[is_, ik][None] - Sigma1[is_, ik][None] - Sw
            Gw = np.linalg.inv(A)
            G[:, is_, ik] = (Ttn_f @ Gw.reshape(nw, nso * nso)).reshape(nts, nso, nso)
    return G


def selfenergy_eigenspectra(Sigma1, Sigma_tau, H, S, Tnt_f):
    """Eigenvalues of S^-1 (H + Sigma1 + Sigma(iw)) for all (w, s, k) (dyson.cpp:48-70).

    Returned with shape [nw, ns, nk, nso] (iwsk order of the reference loop).
    """
    nts, ns, nk, nso, _ = Sigma_tau.shape
    nw = Tnt_f.shape[0]
    ev = np.zeros((nw, ns, nk, nso), dtype=np.complex128)
    for is_ in range(ns):
        for ik in range(nk):
            Sw = (Tnt_f @ Sigma_tau[:, is_, ik].reshape(nts, nso * nso)).reshape(nw, nso, nso)
            Sinv = np.linalg.inv(S[is_, ik])
            X = H[is_, ik][None] + Sigma1[is_, ik][None] + Sw
            ev[:, is_, ik] = np.linalg.eigvals(Sinv[None] @ X)
    return ev


def number_of_electrons(mu, ev, Ttn_beta, wsample_f, ns, nkpw, weight=None, X2C=False):
    """dyson::compute_number_of_electrons (dyson.cpp:72-99)."""
    nw, _, nk, _ = ev.shape
    w = np.ones(nk) if weight is None else np.asarray(weight, dtype=float)
    z = (1j * wsample_f + mu)[:, None, None, None]
    trace_w = (nkpw * w[None, None, :, None] / (z - ev)).sum(axis=(1, 2, 3))
    trace_t = Ttn_beta @ trace_w
    prefactor = 1 if (ns == 2 or X2C) else 2
    return prefactor * -trace_t.real


class ChemicalPotentialSearchFailure(RuntimeError):
    pass


def find_mu(mu0, nel_target, ev, Ttn_beta, wsample_f, ns, nkpw, tol, weight=None, X2C=False):
    """dyson::find_mu (dyson.cpp:101-174): bracket with step 0.5, then bisection."""
    nel_of = lambda m: number_of_electrons(m, ev, Ttn_beta, wsample_f, ns, nkpw, weight, X2C)
    mu = mu0
    delta = 0.5
    nel = nel_of(mu)
    if abs((nel - nel_target) / nel_target) > tol:
        if nel > nel_target:
            mu1 = mu - delta
            while True:
                nel1 = nel_of(mu1)
                mu1 -= delta
                if not nel1 > nel_target:
                    break
            mu2, nel2 = mu, nel
        else:
            mu2 = mu + delta
            while True:
                nel2 = nel_of(mu2)
                mu2 += delta
                if not nel2 < nel_target:
                    break
            mu1, nel1 = mu, nel
        while abs((nel - nel_target) / nel_target) > tol and abs(mu2 - mu1) > 0.01 * tol:
            mu = 0.5 * (mu1 + mu2)
            nel_old = nel_of(mu)
            if abs((nel_old - nel_target) / nel_target) > tol and abs(nel - nel_old) < 0.001 * tol:
                raise ChemicalPotentialSearchFailure("Chemical potential search failed.")
            nel = nel_old
            if nel > nel_target:
                mu2 = mu
            else:
                mu1 = mu
    return nel, mu


def compute_energy(G, Sigma1, Sigma_tau, H, Tnt_f, Ttn_beta, nkpw, weight=None, X2C=False):
    """(E_1b, E_HF, E_corr) of common_utils.cpp:5-55."""
    nts, ns, nk, nso, _ = G.shape
    w = np.ones(nk) if weight is None else np.asarray(weight, dtype=float)
    dmr = G[-1] * (-1.0 if (ns == 2 or X2C) else -2.0)
    nw = Tnt_f.shape[0]
    Gw = (Tnt_f @ G.reshape(nts, -1)).reshape(nw, ns, nk, nso, nso)
    Sw = (Tnt_f @ Sigma_tau.reshape(nts, -1)).reshape(nw, ns, nk, nso, nso)
    tr = np.einsum("wskij,wskji->wsk", Gw, Sw)
    GS_w = (tr * w[None, None, :]).sum(axis=(1, 2))
    energy = -(Ttn_beta @ GS_w).real * (1.0 if (ns == 1 and not X2C) else 0.5)
    ehf = 0.0
    e1e = 0.0
    for is_ in range(ns):
        for ik in range(nk):
            ehf += 0.5 * np.trace(dmr[is_, ik] @ (Sigma1[is_, ik] + 2.0 * H[is_, ik])).real * w[ik]
            e1e += np.trace(dmr[is_, ik] @ H[is_, ik]).real * w[ik]
    return e1e * nkpw, ehf * nkpw, energy * nkpw
