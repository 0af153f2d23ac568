// Vector-Jacobian product of the GW self-energy with respect to G (FP64).
//
// The reference has no derivatives; this is the adjoint of the forward pipeline of gw.cu
// (gw_cpu_kernel.cpp:74-373), for the real inner product Re<a, b>: with L = Re sum conj(Sb) Sigma,
// the result Gb satisfies dL = Re sum conj(Gb) dG for every complex dG.  Per q-point the
// forward is recomputed in FP64 (P0, the W solve) and the backward runs through
//   Sigma = -(1/nk) sum_QQ' W_QQ' V^Q G V^Q'^H       -> Gb, Wbar
//   W = Ttn_b herm(T) Pw,  T = hfl(I - Pw)^-1        -> Pw_bar (hfl: lower triangle + real diagonal)
//   Pw = Tnt_b P0,  P0 = symmetrize(P0h)              -> P0h_bar
//   P0h_QQ' = -pref sum tr(V^Q'^H Gbar V^Q G1)          -> Gb at G(beta - tau, k) and G(tau, k + q)
// with the contractions ordered so that no NQ x NQ x nao^2 intermediate appears.  With Vb the
// gradient with respect to the full pair set [nk][nk][NQ][nao][nao] is accumulated as well: V enters
// Sigma through V(k, k - q) and P0 through V(k, k + q), each twice (V^Q and conj(V^Q')).
#include <algorithm>
#include <vector>

#include "context.cuh"

namespace gb200 {
namespace {

inline unsigned grid_for(int64_t n, int nt) {
  int64_t g = (n + nt - 1) / nt;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

ZOperand dense(const cplx* p, int64_t ld) {
  ZOperand o;
  o.ptr = p;
  o.row = lin(ld);
  o.col = lin(1);
  return o;
}

// P0(t) = herm(P0(t)/nk), P0(nts-1-t) = P0(t) for t < nts/2 (the forward's symmetrize_P0)
__global__ void adj_symmetrize_p0_kernel(cplx* P0, int nts, int NQ, double inv_nk) {
  const int nth = nts / 2;
  const int64_t nq2 = (int64_t)NQ * NQ, total = (int64_t)nth * nq2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / nq2);
    const int64_t r = e % nq2, i = r / NQ, j = r % NQ;
    if (j > i) continue;
    cplx* M = P0 + (int64_t)t * nq2;
    cplx* Mm = P0 + (int64_t)(nts - 1 - t) * nq2;
    const cplx h = cscale(cadd(cscale(M[i * NQ + j], inv_nk), cconj(cscale(M[j * NQ + i], inv_nk))), 0.5);
    M[i * NQ + j] = h;
    M[j * NQ + i] = cconj(h);
    Mm[i * NQ + j] = h;
    Mm[j * NQ + i] = cconj(h);
  }
}

// adjoint of symmetrize_P0: P0h_bar(t) = herm(P0_bar(t) + P0_bar(nts-1-t)) / nk for t < nts/2
__global__ void adj_symmetrize_p0_back_kernel(const cplx* P0b, cplx* P0hb, int nts, int NQ, double inv_nk) {
  const int nth = nts / 2;
  const int64_t nq2 = (int64_t)NQ * NQ, total = (int64_t)nth * nq2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int t = (int)(e / nq2);
    const int64_t r = e % nq2, i = r / NQ, j = r % NQ;
    const cplx* A = P0b + (int64_t)t * nq2;
    const cplx* B = P0b + (int64_t)(nts - 1 - t) * nq2;
    const cplx sij = cadd(A[i * NQ + j], B[i * NQ + j]);
    const cplx sji = cadd(A[j * NQ + i], B[j * NQ + i]);
    P0hb[e] = cscale(cadd(sij, cconj(sji)), 0.5 * inv_nk);
  }
}

// Pw_bar -= hfl^T(A_bar): X_bar_ij = A_bar_ij + conj(A_bar_ji) (i > j), Re A_bar_ii (i = j), 0 (i < j)
__global__ void adj_hfl_back_kernel(const cplx* Ab, cplx* Pwb, int64_t nmat, int NQ) {
  const int64_t nq2 = (int64_t)NQ * NQ, total = nmat * nq2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = e / nq2, r = e % nq2, i = r / NQ, j = r % NQ;
    const cplx* A = Ab + m * nq2;
    cplx x;
    if (i > j) x = cadd(A[i * NQ + j], cconj(A[j * NQ + i]));
    else if (i == j) x = cmk(A[i * NQ + i].x, 0.0);
    else continue;
    Pwb[e] = csub(Pwb[e], x);
  }
}

// offsets of the (kk, s) blocks of a [kk][t][s][...] intermediate: tab[kk*ns + s] = kk*blk + s*pe
__global__ void ks_table_kernel(int64_t* tab, int kbk, int ns, int64_t blk, int64_t pe) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kbk * ns) tab[i] = (int64_t)(i / ns) * blk + (int64_t)(i % ns) * pe;
}

// Vb_half[p(k1,k2)] = Vb[k1][k2] + (k1 > k2 ? Vb[k2][k1]^H per Q : 0): the (k2, k1) block of the full
// pair set is the per-Q conjugate transpose of the stored (k1, k2) block (scatter_pairs_kernel)
__global__ void fold_pair_gradient_kernel(const cplx* full, cplx* half, int nk, int NQ, int nao) {
  const int64_t m2 = (int64_t)nao * nao, pe = (int64_t)NQ * m2;
  const int64_t total = (int64_t)nk * (nk + 1) / 2 * pe;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t idx = e / pe, r = e - idx * pe;
    int64_t k1 = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (k1 * (k1 + 1) / 2 > idx) --k1;
    while ((k1 + 1) * (k1 + 2) / 2 <= idx) ++k1;
    const int64_t k2 = idx - k1 * (k1 + 1) / 2;
    const int64_t Q = r / m2, ij = r - Q * m2, i = ij / nao, j = ij % nao;
    cplx g = full[(k1 * nk + k2) * pe + r];
    if (k1 != k2) g = cadd(g, cconj(full[(k2 * nk + k1) * pe + Q * m2 + j * nao + i]));
    half[e] = g;
  }
}
}  // namespace

void fold_pair_gradient(Context& c, const cplx* full, cplx* half, cudaStream_t st) {
  const int64_t total = (int64_t)c.d.nk * (c.d.nk + 1) / 2 * c.pair_elems();
  fold_pair_gradient_kernel<<<grid_for(total, 256), 256, 0, st>>>(full, half, c.d.nk, c.d.NQ, c.d.nao);
  GB_CHECK_LAUNCH();
}

void gw_sigma_vjp(Context& c, const cplx* G, const cplx* Sb, cplx* Gb, cplx* Vb, cudaStream_t st) {
  const gb200_dims& d = c.d;
  require(d.nts % 2 == 0, GB200_ERR_WRONG_GRID, "Number of tau points should be even!!!");
  require(c.have_kq && c.have_grid && c.have_V, GB200_ERR_STATE, "gw_sigma_vjp: k/q maps, grid and integrals must be set");
  require(!c.x2c(), GB200_ERR_INVALID, "gw_sigma_vjp: two-component input is not supported by the adjoint");
  require(!c.q0_on, GB200_ERR_INVALID, "gw_sigma_vjp: the q->0 correction is not supported by the adjoint");
  require(!c.v_subset(), GB200_ERR_INVALID, "gw_sigma_vjp: needs all integral pairs (the adjoint runs every q-point)");
  const int nk = d.nk, ns = d.ns, nts = d.nts, nth = nts / 2, NQ = d.NQ, nw_b = d.nw_b;
  const int64_t nao = d.nao, nao2 = nao * nao, pe = c.pair_elems(), nq2 = (int64_t)NQ * NQ;
  const int64_t ge = nao2, g_s = (int64_t)nk * ge, g_t = (int64_t)ns * g_s;
  const double pref = (ns == 2) ? 1.0 : 2.0;
  const cplx* V = c.V.get();
  GB_CUDA(cudaMemsetAsync(Gb, 0, c.g_elems() * sizeof(cplx), st));

  auto buf = [&](int slot, int64_t n) { return (cplx*)c.scratch.get(slot, (size_t)n * sizeof(cplx)); };
  cplx* P0 = buf(SL_P0, nts * nq2);
  cplx* Pw = buf(SL_PW, nw_b * nq2);
  cplx* T = buf(SL_PINV, nw_b * nq2);
  cplx* aug = buf(SL_AUG, nw_b * 2 * nq2);
  cplx* Th = buf(SL_ADJ_TH, nw_b * nq2);
  cplx* Ptw = buf(SL_ADJ_PTW, nw_b * nq2);
  cplx* W = buf(SL_ADJ_W, nts * nq2);
  cplx* Wb = buf(SL_ADJ_WB, nts * nq2);
  cplx* Ptwb = buf(SL_ADJ_PTWB, nw_b * nq2);
  cplx* Pwb = buf(SL_ADJ_PWB, nw_b * nq2);
  cplx* Thb = buf(SL_ADJ_THB, nw_b * nq2);
  cplx* Xb = buf(SL_ADJ_XB, nw_b * nq2);
  cplx* Ab = buf(SL_ADJ_AB, nw_b * nq2);
  cplx* P0b = buf(SL_ADJ_P0B, nts * nq2);
  cplx* P0hb = buf(SL_ADJ_P0HB, nth * nq2);
  // k-block: three intermediates of nts*ns*pe per k-point
  const int64_t blk = (int64_t)nts * ns * pe;
  const double budget = c.budget_or(24e9, 0.6);
  int kb = (int)std::max(1.0, std::floor(budget / (3.0 * (double)blk * sizeof(cplx))));
  kb = std::min(kb, nk);
  cplx* X1 = buf(SL_Y1, kb * blk);
  cplx* X2 = buf(SL_Y2, kb * blk);
  cplx* X3 = buf(SL_ADJ_X3, kb * blk);
  int64_t* tab_ks = (int64_t*)c.scratch.get(SL_ADJ_TAB, (size_t)kb * ns * sizeof(int64_t));
  // tab_tq[t*ns + s] = t*NQ^2: the (tau, spin) blocks of an [nts][NQ][NQ] matrix set
  int64_t* tab_tq = (int64_t*)c.scratch.get(SL_ADJ_TQ, (size_t)nts * ns * sizeof(int64_t));
  if (Vb) {
    ks_table_kernel<<<(unsigned)((nts * ns + 255) / 256), 256, 0, st>>>(tab_tq, nts, ns, nq2, 0);
    GB_CHECK_LAUNCH();
    GB_CUDA(cudaMemsetAsync(Vb, 0, (size_t)nk * nk * pe * sizeof(cplx), st));
  }

  for (int q = 0; q < nk; ++q) {
    // ---------------- forward P0(tau, q), FP64 (the contractions (a)-(c) of gw.cu) ----------
    GB_CUDA(cudaMemsetAsync(P0, 0, (size_t)nts * nq2 * sizeof(cplx), st));
    for (int k0 = 0; k0 < nk; k0 += kb) {
      const int kbk = std::min(kb, nk - k0);
      const int64_t* tVp = c.tab_pair_plus.get() + (int64_t)q * nk + k0;
      const int64_t* tGp = c.tab_g_plus.get() + (int64_t)q * nk + k0;
      const int64_t blkT1 = (int64_t)nth * ns * pe;
      ZGemm a;  // T1^T = G(t,s,k+q)^T V(k,k+q)^T
      a.M = (int64_t)nth * ns * nao; a.N = (int64_t)NQ * nao; a.K = nao;
      a.nb0 = kbk;
      a.A.ptr = G; a.A.row = two(nao, 1, g_s); a.A.col = lin(nao); a.A.bat.tab0 = tGp;
      a.B.ptr = V; a.B.row = lin(1); a.B.col = lin(nao); a.B.bat.tab0 = tVp;
      a.C.ptr = X1; a.C.row = two(nao, 1, pe); a.C.col = lin(nao); a.C.bat.s0 = blkT1;
      zgemm_fp64(a, st);
      ZGemm b;  // Bt = Gbar(nts-1-t, s, k) T1
      b.M = nao; b.N = (int64_t)NQ * nao; b.K = nao;
      b.nb0 = kbk; b.nb1 = nth; b.nb2 = ns;
      b.A = dense(G + (int64_t)(nts - 1) * g_t + (int64_t)k0 * ge, nao);
      b.A.bat.s0 = ge; b.A.bat.s1 = -g_t; b.A.bat.s2 = g_s;
      b.B.ptr = X1; b.B.row = lin(nao); b.B.col = two(nao, 1, nao2);
      b.B.bat.s0 = blkT1; b.B.bat.s1 = (int64_t)ns * pe; b.B.bat.s2 = pe;
      b.C.ptr = X2; b.C.row = lin(nao); b.C.col = two(nao, 1, nao2);
      b.C.bat.s0 = (int64_t)ns * pe; b.C.bat.s1 = (int64_t)kbk * ns * pe; b.C.bat.s2 = pe;
      zgemm_fp64(b, st);
      ZGemm cc;  // P0^T -= pref conj(V) Bt^T
      cc.M = NQ; cc.N = NQ; cc.K = (int64_t)kbk * ns * nao2;
      cc.nb2 = nth;
      cc.A.ptr = V; cc.A.row = lin(nao2); cc.A.conj = true;
      cc.A.col = twotab(nao2, 1, c.tab_pair_plus_ns.get() + ((int64_t)q * nk + k0) * ns);
      cc.B.ptr = X2; cc.B.col = lin(nao2); cc.B.row = two(nao2, 1, (int64_t)NQ * nao2);
      cc.B.bat.s2 = (int64_t)kbk * ns * pe;
      cc.C.ptr = P0; cc.C.row = lin(1); cc.C.col = lin(NQ); cc.C.bat.s2 = nq2;
      cc.alpha = cmk(-pref, 0.0); cc.beta = cmk(1.0, 0.0);
      zgemm_fp64(cc, st);
    }
    adj_symmetrize_p0_kernel<<<grid_for((int64_t)nth * nq2, 256), 256, 0, st>>>(P0, nts, NQ, 1.0 / nk);
    GB_CHECK_LAUNCH();
    // ---------------- forward W phase ----------------------------------------------------------
    {
      ZGemm f;  // Pw = Tnt_b P0
      f.M = nw_b; f.N = nq2; f.K = nts;
      f.A = dense(c.Tnt_b.get(), nts);
      f.B = dense(P0, nq2);
      f.C.ptr = Pw; f.C.row = lin(nq2); f.C.col = lin(1);
      zgemm_fp64(f, st);
      invert_large_batched(Pw, T, aug, nw_b, NQ, true, true, st);
      GB_CUDA(cudaMemcpyAsync(Th, T, (size_t)nw_b * nq2 * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
      hermitize_batched(Th, nw_b, NQ, 1.0, st);
      ZGemm m;  // Ptw = Th Pw
      m.M = NQ; m.N = NQ; m.K = NQ; m.nb2 = nw_b;
      m.A = dense(Th, NQ); m.A.bat.s2 = nq2;
      m.B = dense(Pw, NQ); m.B.bat.s2 = nq2;
      m.C.ptr = Ptw; m.C.row = lin(NQ); m.C.col = lin(1); m.C.bat.s2 = nq2;
      zgemm_fp64(m, st);
      ZGemm w;  // W = Ttn_b Ptw
      w.M = nts; w.N = nq2; w.K = nw_b;
      w.A = dense(c.Ttn_b.get(), nw_b);
      w.B = dense(Ptw, nq2);
      w.C.ptr = W; w.C.row = lin(nq2); w.C.col = lin(1);
      zgemm_fp64(w, st);
    }
    // ---------------- Sigma = -(1/nk) sum_QQ' W_QQ' V^Q G V^Q'^H: Gb and Wbar -------------------
    GB_CUDA(cudaMemsetAsync(Wb, 0, (size_t)nts * nq2 * sizeof(cplx), st));
    for (int k0 = 0; k0 < nk; k0 += kb) {
      const int kbk = std::min(kb, nk - k0);
      const int64_t* tVm = c.tab_pair_minus.get() + (int64_t)q * nk + k0;
      const int64_t* tGm = c.tab_g_minus.get() + (int64_t)q * nk + k0;
      ZGemm a1;  // A1[kk][t][s][(Q,m)][j] = sum_i conj(V(k,k-q)[Q][i][m]) Sb(t,s,k)[i][j]
      a1.M = (int64_t)NQ * nao; a1.N = nao; a1.K = nao;
      a1.nb0 = kbk; a1.nb1 = nts; a1.nb2 = ns;
      a1.A.ptr = V; a1.A.row = two(nao, 1, nao2); a1.A.col = lin(nao); a1.A.conj = true; a1.A.bat.tab0 = tVm;
      a1.B = dense(Sb + (int64_t)k0 * ge, nao); a1.B.bat.s0 = ge; a1.B.bat.s1 = g_t; a1.B.bat.s2 = g_s;
      a1.C.ptr = X1; a1.C.row = lin(nao); a1.C.col = lin(1);
      a1.C.bat.s0 = blk; a1.C.bat.s1 = (int64_t)ns * pe; a1.C.bat.s2 = pe;
      zgemm_fp64(a1, st);
      ZGemm z;  // Z[kk][t][Q][(j,n)] = sum_Q' conj(W(t)[Q][Q']) V(k,k-q)[Q'][(j,n)]
      z.M = NQ; z.N = nao2; z.K = NQ;
      z.nb0 = kbk; z.nb1 = nts;
      z.A = dense(W, NQ); z.A.conj = true; z.A.bat.s1 = nq2;
      z.B.ptr = V; z.B.row = lin(nao2); z.B.col = lin(1); z.B.bat.tab0 = tVm;
      z.C.ptr = X2; z.C.row = lin(nao2); z.C.col = lin(1); z.C.bat.s0 = (int64_t)nts * pe; z.C.bat.s1 = pe;
      zgemm_fp64(z, st);
      ZGemm gs;  // Gb(t,s,k-q)[m][n] -= (1/nk) sum_{(Q,j)} A1[..][Q][m][j] Z[..][Q][j][n]
      gs.M = nao; gs.N = nao; gs.K = (int64_t)NQ * nao;
      gs.nb0 = kbk; gs.nb1 = nts; gs.nb2 = ns;
      gs.A.ptr = X1; gs.A.row = lin(nao); gs.A.col = two(nao, 1, nao2);
      gs.A.bat.s0 = blk; gs.A.bat.s1 = (int64_t)ns * pe; gs.A.bat.s2 = pe;
      gs.B.ptr = X2; gs.B.row = lin(nao); gs.B.col = lin(1); gs.B.bat.s0 = (int64_t)nts * pe; gs.B.bat.s1 = pe;
      gs.C.ptr = Gb; gs.C.row = lin(nao); gs.C.col = lin(1);
      gs.C.bat.tab0 = tGm; gs.C.bat.s1 = g_t; gs.C.bat.s2 = g_s;
      gs.alpha = cmk(-1.0 / nk, 0.0); gs.beta = cmk(1.0, 0.0);
      zgemm_fp64(gs, st);
      if (Vb) {
        ZGemm f;  // F[kk][t][s][Q][j][m] = sum_n Z[kk][t][Q][j][n] conj(G(t,s,k-q)[m][n])
        f.M = (int64_t)NQ * nao; f.N = nao; f.K = nao;
        f.nb0 = kbk; f.nb1 = nts; f.nb2 = ns;
        f.A.ptr = X2; f.A.row = lin(nao); f.A.col = lin(1); f.A.bat.s0 = (int64_t)nts * pe; f.A.bat.s1 = pe;
        f.B.ptr = G; f.B.row = lin(1); f.B.col = lin(nao); f.B.conj = true;
        f.B.bat.tab0 = tGm; f.B.bat.s1 = g_t; f.B.bat.s2 = g_s;
        f.C.ptr = X3; f.C.row = lin(nao); f.C.col = lin(1);
        f.C.bat.s0 = blk; f.C.bat.s1 = (int64_t)ns * pe; f.C.bat.s2 = pe;
        zgemm_fp64(f, st);
        ZGemm v1;  // Vb(k,k-q)[Q][i][m] -= (1/nk) sum_{(t,s),j} Sb(t,s,k)[i][j] F[kk][t][s][Q][j][m]
        v1.M = nao; v1.N = nao; v1.K = (int64_t)nts * ns * nao;
        v1.nb0 = kbk; v1.nb1 = NQ;
        v1.A.ptr = Sb + (int64_t)k0 * ge; v1.A.row = lin(nao); v1.A.col = two(nao, 1, g_s); v1.A.bat.s0 = ge;
        v1.B.ptr = X3; v1.B.row = two(nao, nao, pe); v1.B.col = lin(1); v1.B.bat.s0 = blk; v1.B.bat.s1 = nao2;
        v1.C.ptr = Vb; v1.C.row = lin(nao); v1.C.col = lin(1); v1.C.bat.tab0 = tVm; v1.C.bat.s1 = nao2;
        v1.alpha = cmk(-1.0 / nk, 0.0); v1.beta = cmk(1.0, 0.0);
        zgemm_fp64(v1, st);
        ZGemm h;  // H[kk][t][s][Q][j][n] = sum_m conj(A1[kk][t][s][Q][m][j]) G(t,s,k-q)[m][n]
        h.M = (int64_t)NQ * nao; h.N = nao; h.K = nao;
        h.nb0 = kbk; h.nb1 = nts; h.nb2 = ns;
        h.A.ptr = X1; h.A.row = two(nao, 1, nao2); h.A.col = lin(nao); h.A.conj = true;
        h.A.bat.s0 = blk; h.A.bat.s1 = (int64_t)ns * pe; h.A.bat.s2 = pe;
        h.B.ptr = G; h.B.row = lin(nao); h.B.col = lin(1); h.B.bat.tab0 = tGm; h.B.bat.s1 = g_t; h.B.bat.s2 = g_s;
        h.C.ptr = X3; h.C.row = lin(nao); h.C.col = lin(1);
        h.C.bat.s0 = blk; h.C.bat.s1 = (int64_t)ns * pe; h.C.bat.s2 = pe;
        zgemm_fp64(h, st);
        ZGemm v2;  // Vb(k,k-q)[Q'][(j,n)] -= (1/nk) sum_{(t,s),Q} W(t)[Q][Q'] H[kk][t][s][Q][(j,n)]
        v2.M = NQ; v2.N = nao2; v2.K = (int64_t)nts * ns * NQ;
        v2.nb0 = kbk;
        v2.A.ptr = W; v2.A.row = lin(1); v2.A.col = twotab(NQ, NQ, tab_tq);
        v2.B.ptr = X3; v2.B.row = lin(nao2); v2.B.col = lin(1); v2.B.bat.s0 = blk;
        v2.C.ptr = Vb; v2.C.row = lin(nao2); v2.C.col = lin(1); v2.C.bat.tab0 = tVm;
        v2.alpha = cmk(-1.0 / nk, 0.0); v2.beta = cmk(1.0, 0.0);
        zgemm_fp64(v2, st);
      }
      ZGemm ut;  // Ut[kk][t][s][Q'][m][j] = sum_n conj(G(t,s,k-q)[m][n]) V(k,k-q)[Q'][j][n]
      ut.M = nao; ut.N = (int64_t)NQ * nao; ut.K = nao;
      ut.nb0 = kbk; ut.nb1 = nts; ut.nb2 = ns;
      ut.A.ptr = G; ut.A.row = lin(nao); ut.A.col = lin(1); ut.A.conj = true;
      ut.A.bat.tab0 = tGm; ut.A.bat.s1 = g_t; ut.A.bat.s2 = g_s;
      ut.B.ptr = V; ut.B.row = lin(1); ut.B.col = lin(nao); ut.B.bat.tab0 = tVm;
      ut.C.ptr = X2; ut.C.row = lin(nao); ut.C.col = two(nao, 1, nao2);
      ut.C.bat.s0 = blk; ut.C.bat.s1 = (int64_t)ns * pe; ut.C.bat.s2 = pe;
      zgemm_fp64(ut, st);
      ks_table_kernel<<<(unsigned)((kbk * ns + 255) / 256), 256, 0, st>>>(tab_ks, kbk, ns, blk, pe);
      GB_CHECK_LAUNCH();
      ZGemm wb;  // Wb(t)[Q][Q'] -= (1/nk) sum_{(kk,s),(m,j)} A1[..][Q][m][j] Ut[..][Q'][m][j]
      wb.M = NQ; wb.N = NQ; wb.K = (int64_t)kbk * ns * nao2;
      wb.nb2 = nts;
      wb.A.ptr = X1; wb.A.row = lin(nao2); wb.A.col = twotab(nao2, 1, tab_ks); wb.A.bat.s2 = (int64_t)ns * pe;
      wb.B.ptr = X2; wb.B.row = twotab(nao2, 1, tab_ks); wb.B.col = lin(nao2); wb.B.bat.s2 = (int64_t)ns * pe;
      wb.C.ptr = Wb; wb.C.row = lin(NQ); wb.C.col = lin(1); wb.C.bat.s2 = nq2;
      wb.alpha = cmk(-1.0 / nk, 0.0); wb.beta = cmk(1.0, 0.0);
      zgemm_fp64(wb, st);
    }
    // ---------------- W = Ttn_b herm(T) Pw, T = hfl(I - Pw)^-1: Pw_bar ------------------------
    {
      ZGemm g1;  // Ptwb[n] = sum_t conj(Ttn_b[t][n]) Wb[t]
      g1.M = nw_b; g1.N = nq2; g1.K = nts;
      g1.A.ptr = c.Ttn_b.get(); g1.A.row = lin(1); g1.A.col = lin(nw_b); g1.A.conj = true;
      g1.B = dense(Wb, nq2);
      g1.C.ptr = Ptwb; g1.C.row = lin(nq2); g1.C.col = lin(1);
      zgemm_fp64(g1, st);
      ZGemm g2;  // Thb[n] = Ptwb[n] Pw[n]^H
      g2.M = NQ; g2.N = NQ; g2.K = NQ; g2.nb2 = nw_b;
      g2.A = dense(Ptwb, NQ); g2.A.bat.s2 = nq2;
      g2.B.ptr = Pw; g2.B.row = lin(1); g2.B.col = lin(NQ); g2.B.conj = true; g2.B.bat.s2 = nq2;
      g2.C.ptr = Thb; g2.C.row = lin(NQ); g2.C.col = lin(1); g2.C.bat.s2 = nq2;
      zgemm_fp64(g2, st);
      ZGemm g3;  // Pwb[n] = Th[n]^H Ptwb[n]
      g3.M = NQ; g3.N = NQ; g3.K = NQ; g3.nb2 = nw_b;
      g3.A.ptr = Th; g3.A.row = lin(1); g3.A.col = lin(NQ); g3.A.conj = true; g3.A.bat.s2 = nq2;
      g3.B = dense(Ptwb, NQ); g3.B.bat.s2 = nq2;
      g3.C.ptr = Pwb; g3.C.row = lin(NQ); g3.C.col = lin(1); g3.C.bat.s2 = nq2;
      zgemm_fp64(g3, st);
      hermitize_batched(Thb, nw_b, NQ, 1.0, st);  // T_bar = herm(Th_bar)
      ZGemm g4;  // Xb = T^H T_bar
      g4.M = NQ; g4.N = NQ; g4.K = NQ; g4.nb2 = nw_b;
      g4.A.ptr = T; g4.A.row = lin(1); g4.A.col = lin(NQ); g4.A.conj = true; g4.A.bat.s2 = nq2;
      g4.B = dense(Thb, NQ); g4.B.bat.s2 = nq2;
      g4.C.ptr = Xb; g4.C.row = lin(NQ); g4.C.col = lin(1); g4.C.bat.s2 = nq2;
      zgemm_fp64(g4, st);
      ZGemm g5;  // Ab = -Xb T^H
      g5.M = NQ; g5.N = NQ; g5.K = NQ; g5.nb2 = nw_b;
      g5.A = dense(Xb, NQ); g5.A.bat.s2 = nq2;
      g5.B.ptr = T; g5.B.row = lin(1); g5.B.col = lin(NQ); g5.B.conj = true; g5.B.bat.s2 = nq2;
      g5.C.ptr = Ab; g5.C.row = lin(NQ); g5.C.col = lin(1); g5.C.bat.s2 = nq2;
      g5.alpha = cmk(-1.0, 0.0);
      zgemm_fp64(g5, st);
      adj_hfl_back_kernel<<<grid_for((int64_t)nw_b * nq2, 256), 256, 0, st>>>(Ab, Pwb, nw_b, NQ);
      GB_CHECK_LAUNCH();
      ZGemm g6;  // P0b[t] = sum_n conj(Tnt_b[n][t]) Pwb[n]
      g6.M = nts; g6.N = nq2; g6.K = nw_b;
      g6.A.ptr = c.Tnt_b.get(); g6.A.row = lin(1); g6.A.col = lin(nts); g6.A.conj = true;
      g6.B = dense(Pwb, nq2);
      g6.C.ptr = P0b; g6.C.row = lin(nq2); g6.C.col = lin(1);
      zgemm_fp64(g6, st);
      adj_symmetrize_p0_back_kernel<<<grid_for((int64_t)nth * nq2, 256), 256, 0, st>>>(P0b, P0hb, nts, NQ, 1.0 / nk);
      GB_CHECK_LAUNCH();
    }
    // ---------------- P0h_QQ' = -pref sum tr(V^Q'^H Gbar V^Q G1): Gb ---------------------------
    for (int k0 = 0; k0 < nk; k0 += kb) {
      const int kbk = std::min(kb, nk - k0);
      const int64_t* tVp = c.tab_pair_plus.get() + (int64_t)q * nk + k0;
      const int64_t* tGp = c.tab_g_plus.get() + (int64_t)q * nk + k0;
      const int64_t rblk = (int64_t)nth * pe, cblk = (int64_t)nth * ns * pe;
      ZGemm r;  // R[kk][t][Q][(r,n)] = sum_Q' P0hb(t)[Q][Q'] V(k,k+q)[Q'][(r,n)]
      r.M = NQ; r.N = nao2; r.K = NQ;
      r.nb0 = kbk; r.nb1 = nth;
      r.A = dense(P0hb, NQ); r.A.bat.s1 = nq2;
      r.B.ptr = V; r.B.row = lin(nao2); r.B.col = lin(1); r.B.bat.tab0 = tVp;
      r.C.ptr = X1; r.C.row = lin(nao2); r.C.col = lin(1); r.C.bat.s0 = rblk; r.C.bat.s1 = pe;
      zgemm_fp64(r, st);
      ZGemm cm;  // Cm[kk][t][s][(Q,r)][m] = sum_n R[kk][t][Q][r][n] conj(G(t,s,k+q)[m][n])
      cm.M = (int64_t)NQ * nao; cm.N = nao; cm.K = nao;
      cm.nb0 = kbk; cm.nb1 = nth; cm.nb2 = ns;
      cm.A.ptr = X1; cm.A.row = lin(nao); cm.A.col = lin(1); cm.A.bat.s0 = rblk; cm.A.bat.s1 = pe;
      cm.B.ptr = G; cm.B.row = lin(1); cm.B.col = lin(nao); cm.B.conj = true;
      cm.B.bat.tab0 = tGp; cm.B.bat.s1 = g_t; cm.B.bat.s2 = g_s;
      cm.C.ptr = X2; cm.C.row = lin(nao); cm.C.col = lin(1);
      cm.C.bat.s0 = cblk; cm.C.bat.s1 = (int64_t)ns * pe; cm.C.bat.s2 = pe;
      zgemm_fp64(cm, st);
      ZGemm gb;  // Gb(nts-1-t,s,k)[r][p] -= pref sum_{(Q,m)} Cm[..][Q][r][m] conj(V(k,k+q)[Q][p][m])
      gb.M = nao; gb.N = nao; gb.K = (int64_t)NQ * nao;
      gb.nb0 = kbk; gb.nb1 = nth; gb.nb2 = ns;
      gb.A.ptr = X2; gb.A.row = lin(nao); gb.A.col = two(nao, 1, nao2);
      gb.A.bat.s0 = cblk; gb.A.bat.s1 = (int64_t)ns * pe; gb.A.bat.s2 = pe;
      gb.B.ptr = V; gb.B.row = two(nao, 1, nao2); gb.B.col = lin(nao); gb.B.conj = true; gb.B.bat.tab0 = tVp;
      gb.C.ptr = Gb + (int64_t)(nts - 1) * g_t + (int64_t)k0 * ge; gb.C.row = lin(nao); gb.C.col = lin(1);
      gb.C.bat.s0 = ge; gb.C.bat.s1 = -g_t; gb.C.bat.s2 = g_s;
      gb.alpha = cmk(-pref, 0.0); gb.beta = cmk(1.0, 0.0);
      zgemm_fp64(gb, st);
      ZGemm dd;  // D[kk][t][s][Q][p][n] = sum_r conj(G(nts-1-t,s,k)[r][p]) R[kk][t][Q][r][n]
      dd.M = nao; dd.N = (int64_t)NQ * nao; dd.K = nao;
      dd.nb0 = kbk; dd.nb1 = nth; dd.nb2 = ns;
      dd.A.ptr = G + (int64_t)(nts - 1) * g_t + (int64_t)k0 * ge; dd.A.row = lin(1); dd.A.col = lin(nao);
      dd.A.conj = true; dd.A.bat.s0 = ge; dd.A.bat.s1 = -g_t; dd.A.bat.s2 = g_s;
      dd.B.ptr = X1; dd.B.row = lin(nao); dd.B.col = two(nao, 1, nao2); dd.B.bat.s0 = rblk; dd.B.bat.s1 = pe;
      dd.C.ptr = X3; dd.C.row = lin(nao); dd.C.col = two(nao, 1, nao2);
      dd.C.bat.s0 = cblk; dd.C.bat.s1 = (int64_t)ns * pe; dd.C.bat.s2 = pe;
      zgemm_fp64(dd, st);
      ZGemm g1b;  // Gb(t,s,k+q)[m][n] -= pref sum_{(Q,p)} conj(V(k,k+q)[Q][p][m]) D[..][Q][p][n]
      g1b.M = nao; g1b.N = nao; g1b.K = (int64_t)NQ * nao;
      g1b.nb0 = kbk; g1b.nb1 = nth; g1b.nb2 = ns;
      g1b.A.ptr = V; g1b.A.row = lin(1); g1b.A.col = two(nao, nao, nao2); g1b.A.conj = true; g1b.A.bat.tab0 = tVp;
      g1b.B.ptr = X3; g1b.B.row = lin(nao); g1b.B.col = lin(1);
      g1b.B.bat.s0 = cblk; g1b.B.bat.s1 = (int64_t)ns * pe; g1b.B.bat.s2 = pe;
      g1b.C.ptr = Gb; g1b.C.row = lin(nao); g1b.C.col = lin(1);
      g1b.C.bat.tab0 = tGp; g1b.C.bat.s1 = g_t; g1b.C.bat.s2 = g_s;
      g1b.alpha = cmk(-pref, 0.0); g1b.beta = cmk(1.0, 0.0);
      zgemm_fp64(g1b, st);
      if (Vb) {
        ZGemm v3;  // Vb(k,k+q)[Q][p][m] -= pref sum_{(t,s),n} D[kk][t][s][Q][p][n] conj(G(t,s,k+q)[m][n])
        v3.M = nao; v3.N = nao; v3.K = (int64_t)nth * ns * nao;
        v3.nb0 = kbk; v3.nb1 = NQ;
        v3.A.ptr = X3; v3.A.row = lin(nao); v3.A.col = two(nao, 1, pe); v3.A.bat.s0 = cblk; v3.A.bat.s1 = nao2;
        v3.B.ptr = G; v3.B.row = two(nao, 1, g_s); v3.B.col = lin(nao); v3.B.conj = true; v3.B.bat.tab0 = tGp;
        v3.C.ptr = Vb; v3.C.row = lin(nao); v3.C.col = lin(1); v3.C.bat.tab0 = tVp; v3.C.bat.s1 = nao2;
        v3.alpha = cmk(-pref, 0.0); v3.beta = cmk(1.0, 0.0);
        zgemm_fp64(v3, st);
        ZGemm a;  // T1 recomputed: X1[kk][t][s][Q][p][n] = (V(k,k+q)^Q G(t,s,k+q))[p][n]
        a.M = (int64_t)nth * ns * nao; a.N = (int64_t)NQ * nao; a.K = nao;
        a.nb0 = kbk;
        a.A.ptr = G; a.A.row = two(nao, 1, g_s); a.A.col = lin(nao); a.A.bat.tab0 = tGp;
        a.B.ptr = V; a.B.row = lin(1); a.B.col = lin(nao); a.B.bat.tab0 = tVp;
        a.C.ptr = X1; a.C.row = two(nao, 1, pe); a.C.col = lin(nao); a.C.bat.s0 = cblk;
        zgemm_fp64(a, st);
        ZGemm b;  // Bt recomputed: X2[kk][t][s][Q][r][n] = sum_p Gbar(nts-1-t,s,k)[r][p] T1[..][Q][p][n]
        b.M = nao; b.N = (int64_t)NQ * nao; b.K = nao;
        b.nb0 = kbk; b.nb1 = nth; b.nb2 = ns;
        b.A = dense(G + (int64_t)(nts - 1) * g_t + (int64_t)k0 * ge, nao);
        b.A.bat.s0 = ge; b.A.bat.s1 = -g_t; b.A.bat.s2 = g_s;
        b.B.ptr = X1; b.B.row = lin(nao); b.B.col = two(nao, 1, nao2);
        b.B.bat.s0 = cblk; b.B.bat.s1 = (int64_t)ns * pe; b.B.bat.s2 = pe;
        b.C.ptr = X2; b.C.row = lin(nao); b.C.col = two(nao, 1, nao2);
        b.C.bat.s0 = cblk; b.C.bat.s1 = (int64_t)ns * pe; b.C.bat.s2 = pe;
        zgemm_fp64(b, st);
        ZGemm v4;  // Vb(k,k+q)[Q'][(r,n)] -= pref sum_{(t,s),Q} conj(P0hb(t)[Q][Q']) Bt[kk][t][s][Q][(r,n)]
        v4.M = NQ; v4.N = nao2; v4.K = (int64_t)nth * ns * NQ;
        v4.nb0 = kbk;
        v4.A.ptr = P0hb; v4.A.row = lin(1); v4.A.col = twotab(NQ, NQ, tab_tq); v4.A.conj = true;
        v4.B.ptr = X2; v4.B.row = lin(nao2); v4.B.col = lin(1); v4.B.bat.s0 = cblk;
        v4.C.ptr = Vb; v4.C.row = lin(nao2); v4.C.col = lin(1); v4.C.bat.tab0 = tVp;
        v4.alpha = cmk(-pref, 0.0); v4.beta = cmk(1.0, 0.0);
        zgemm_fp64(v4, st);
      }
    }
  }
}

}  // namespace gb200
