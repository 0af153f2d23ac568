"""CPU model of the split-precision (Ozaki INT8) contractions, for error budgets.

Test infrastructure, like gw_oracle.py: nothing in the product imports it.  It restates the
arithmetic of the library's split engine in numpy:
- a per-row exponent for the left operand and a per-column exponent for the right one, taken
  over the contraction range, with one bit of headroom (max of |Re| and |Im| < 2^(e-1));
- rounding X = rint(a 2^(7S - e)) and its S balanced base-128 digits;
- the digit products of the diagonals i + j <= S - 1, summed exactly.
The engine's first form (truncation toward zero, sign-magnitude digits) is kept as
digits="truncated" for comparison.
`gw_split_model` runs the six contractions of the GPU's GW pipeline with the same operand roles:
P0 (a) T1^T = G^T V^T, (b) Bt = Gbar T1, (c) P0^T = conj(V) Bt^T; Sigma (d) Y1^T = G^T V^T,
(e) Y2^T = W^T Y1, (f) Sigma^T = conj(V) Y2^T.  Each takes its own slice count, or FP64.  The W
solve and the transforms are FP64, as on the GPU.

For one iteration from G0 on a c2-shaped system (nao=40, naux=250, ntau=120, nw=120, beta=200,
eps ~ U[-5,5], 2x1x1 mesh, seed 0), five slices everywhere: the truncated form gives
max|dSigma| = 1.0344e-7, as the GPU measured with it (1.0344e-7); the balanced form gives 3.1e-9.
Truncation toward zero biases every digit product the same way, so its errors add in phase along
each contraction and across the six of them.

    python oracle/split_model.py [2x1x1] [balanced|truncated]     (error table; about 25 minutes)
"""
import json
import os
import sys
import time

import numpy as np

import gw_oracle as O

CONTRACTIONS = "abcdef"


def split_mm(A, B, S, digits="balanced"):
    """A (M,K) @ B (K,N), complex, as the split engine forms it.  Exponents: per row of A and per
    column of B, over K, of max(|Re|, |Im|).
    - "balanced" (the engine): e = frexp exponent + 1, X = rint(a 2^(7S-e)), balanced base-128 digits
      (lower ones in [-64, 63], the top one the remaining quotient);
    - "truncated" (the engine's first form): e = frexp exponent, X = trunc(a 2^(7S-e)), digits of |X|
      carrying the sign of a.
    Digit products of the diagonals i + j <= S - 1 are kept; S = None is the FP64 product."""
    if S is None:
        return A @ B
    bal = digits == "balanced"

    def expo(X, axis):
        m = np.maximum(np.abs(X.real), np.abs(X.imag)).max(axis=axis)
        _, e = np.frexp(m)
        return np.where(m > 0, e + (1 if bal else 0), 0)

    def planes_of(X, e, rows):
        sc = np.ldexp(1.0, 7 * S - e)
        sc = sc[:, None] if rows else sc[None, :]
        out = []
        for part in (X.real, X.imag):
            if bal:
                Xi = np.rint(part * sc)
                planes = [None] * S
                for i in range(S - 1, 0, -1):
                    d = np.mod(Xi + 64, 128) - 64
                    planes[i] = d
                    Xi = (Xi - d) / 128
                planes[0] = Xi
            else:
                Xi = np.trunc(part * sc)
                mag, sg = np.abs(Xi), np.sign(Xi)
                planes = [sg * (np.floor(mag / 2.0 ** (7 * (S - 1 - i))) % 128) for i in range(S)]
            out.append(planes)
        return [out[0][i] + 1j * out[1][i] for i in range(S)]

    eA, eB = expo(A, 1), expo(B, 0)
    dA, dB = planes_of(A, eA, True), planes_of(B, eB, False)
    C = np.zeros((A.shape[0], B.shape[1]), dtype=np.complex128)
    for d in range(S):
        acc = np.zeros_like(C)
        for i in range(d + 1):
            acc += dA[i] @ dB[d - i]
        C += np.ldexp(1.0, -7 * (d + 2)) * acc
    return C * np.ldexp(1.0, eA)[:, None] * np.ldexp(1.0, eB)[None, :]


def gw_split_model(s, Sc, digits="balanced"):
    """Sigma(tau, k) of the synthetic system `s` with contraction c in 'abcdef' run at Sc[c] slices
    (None: FP64), digits as in split_mm."""
    g = s.grid
    integ, bz = O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh)
    G = s.G
    nts, ns, nk, nao, _ = G.shape
    nth, NQ = nts // 2, s.NQ
    pref = 1.0 if ns == 2 else 2.0
    Sig = np.zeros_like(G)
    I = np.eye(NQ)
    for q in range(nk):
        P0T = np.zeros((nth, NQ, NQ), dtype=np.complex128)   # P0^T[t][Q'][Q]
        Bts = []
        Vs = []
        for k in range(nk):
            kq = bz.k1_from_k2q(k, q)
            V = integ.pair(k, kq)                            # [Q][p][m]
            G1 = G[:nth, :, kq]                              # [t][s][m][n]
            # (a) T1^T[(t,s,n)][(Q,p)] = sum_m G1[t,s][m][n] V[Q][p][m]
            A = np.transpose(G1, (0, 1, 3, 2)).reshape(nth * ns * nao, nao)
            B = np.transpose(V, (2, 0, 1)).reshape(nao, NQ * nao)
            T1T = split_mm(A, B, Sc["a"], digits).reshape(nth, ns, nao, NQ, nao)   # [t][s][n][Q][p]
            T1 = np.transpose(T1T, (0, 1, 3, 4, 2))                       # [t][s][Q][p][n]
            # (b) Bt[t,s][r][(Q,n)] = sum_p Gbar[t,s][r][p] T1[t,s][Q][p][n]
            Bt = np.empty((nth, ns, NQ, nao, nao), dtype=np.complex128)    # [t][s][Q][r][n]
            for t in range(nth):
                for s_ in range(ns):
                    Gb = G[nts - 1 - t, s_, k]
                    Bm = np.transpose(T1[t, s_], (1, 0, 2)).reshape(nao, NQ * nao)  # [p][(Q,n)]
                    R = split_mm(Gb, Bm, Sc["b"], digits).reshape(nao, NQ, nao)            # [r][Q][n]
                    Bt[t, s_] = np.transpose(R, (1, 0, 2))
            Bts.append(Bt)
            Vs.append(V)
        # (c) P0^T[t][Q'][Q] = -pref sum_{(k,s),(r,n)} conj(V_k[Q'][r][n]) Bt_k[t,s][Q][(r,n)]
        for t in range(nth):
            A = np.concatenate([np.conj(Vs[k]).reshape(NQ, nao * nao) for k in range(nk) for s_ in range(ns)], axis=1)
            B = np.concatenate([Bts[k][t, s_].reshape(NQ, nao * nao).T for k in range(nk) for s_ in range(ns)], axis=0)
            P0T[t] = -pref * split_mm(A, B, Sc["c"], digits)
        P0 = np.zeros((nts, NQ, NQ), dtype=np.complex128)
        for t in range(nth):
            M = P0T[t].T / nk
            h = 0.5 * (M + M.conj().T)
            P0[t] = h
            P0[nts - 1 - t] = h
        nwb = g.Tnt_b.shape[0]
        Pw = (g.Tnt_b @ P0.reshape(nts, NQ * NQ)).reshape(nwb, NQ, NQ)
        Ptw = np.empty_like(Pw)
        for n in range(nwb):
            T = np.linalg.solve(O.hermitian_from_lower(I - Pw[n]), I)
            Ptw[n] = O.herm(T) @ Pw[n]
        W = (g.Ttn_b @ Ptw.reshape(nwb, NQ * NQ)).reshape(nts, NQ, NQ)
        for k in range(nk):
            kmq = bz.k2_from_k1q(k, q)
            V = integ.pair(k, kmq)                          # [Q][i][m]
            Gm = G[:, :, kmq]                               # [t][s][m][n]
            # (d) Y1^T[(t,s,n)][(Q,i)] = sum_m Gm[t,s][m][n] V[Q][i][m]
            A = np.transpose(Gm, (0, 1, 3, 2)).reshape(nts * ns * nao, nao)
            B = np.transpose(V, (2, 0, 1)).reshape(nao, NQ * nao)
            Y1T = split_mm(A, B, Sc["d"], digits).reshape(nts, ns, nao, NQ, nao)     # [t][s][n][Q][i]
            Y1 = np.transpose(Y1T, (0, 1, 3, 4, 2))                        # [t][s][Q][i][n]
            Y2 = np.empty((nts, ns, nao, nao, NQ), dtype=np.complex128)     # [t][s][i][n][Q']
            for t in range(nts):
                for s_ in range(ns):
                    # (e) Y2^T[Q'][(i,n)] = sum_Q W[t][Q][Q'] Y1[t,s][Q][(i,n)]
                    R = split_mm(W[t].T, Y1[t, s_].reshape(NQ, nao * nao), Sc["e"], digits)   # [Q'][(i,n)]
                    Y2[t, s_] = R.T.reshape(nao, nao, NQ)
            # (f) Sigma^T[j][((t,s),i)] = -sum_{(n,Q')} conj(V[Q'][j][n]) Y2[t,s][i][(n,Q')]
            A = np.transpose(np.conj(V), (1, 2, 0)).reshape(nao, nao * NQ)            # [j][(n,Q')]
            B = np.transpose(Y2.reshape(nts * ns, nao, nao * NQ), (2, 0, 1)).reshape(nao * NQ, nts * ns * nao)
            ST = -split_mm(A, B, Sc["f"], digits).reshape(nao, nts, ns, nao)               # [j][t][s][i]
            Sig[:, :, k] += np.transpose(ST, (1, 2, 3, 0))
    return Sig / nk


def main(argv):
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "..", "green-mbpt_b200"))
    from gb200 import synth
    mesh = tuple(int(x) for x in argv[1].split("x")) if len(argv) > 1 else (2, 1, 1)
    s = synth.make_system(mesh=mesh, nao=40, naux=250, ns=1, beta=200.0, nts=120, nw=120, eps_range=5.0, seed=0)
    ref = gw_split_model(s, {c: None for c in CONTRACTIONS})
    print("max|Sigma|", float(np.abs(ref).max()), flush=True)
    configs = [("all5", {c: 5 for c in CONTRACTIONS}), ("all4", {c: 4 for c in CONTRACTIONS})]
    for c in CONTRACTIONS:
        d = {x: None for x in CONTRACTIONS}
        d[c] = 5
        configs.append((f"only_{c}5", d))
    digits = argv[2] if len(argv) > 2 else "balanced"
    for name, Sc in configs:
        t0 = time.time()
        sig = gw_split_model(s, Sc, digits)
        print(json.dumps({"config": name, "digits": digits, "max_dSigma": float(np.abs(sig - ref).max()),
                          "seconds": time.time() - t0}), flush=True)


if __name__ == "__main__":
    main(sys.argv)
