// Hartree-Fock Fock matrix on one GPU (hf_scalar_cpu_kernel::solve,
// green-mbpt src/hf_cpu_kernels.cpp:25-146, and hf_x2c_cpu_kernel::solve, :148-279) for the
// no-symmetry case.
//
//   J: u_Q = (1/nk) sum_{k,s} sum_ab V^Q_ab(k,k) dm_ba(k,s);  F_ij(k,s) = sum_Q u_Q V^Q_ij(k,k)
//   K: F_ij(k,s) -= (c/nk) sum_{k'} sum_{Q,a} Y^Q_ia conj(V^Q_ja(k,k')),
//      Y^Q = V^Q(k,k') dm(k',s), c = 0.5 (ns = 1) or 1
//   Madelung: F -= c * madelung * S dm S
#include <algorithm>

#include "context.cuh"

namespace gb200 {
namespace {

// dmT[k][s][a][b] = dm[s][k][b][a]
__global__ void dm_transpose_kernel(const cplx* dm, cplx* dmT, int ns, int nk, int n) {
  const int64_t total = (int64_t)ns * nk * n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t m = e / ((int64_t)n * n);
    int r = (int)(e % ((int64_t)n * n));
    int a = r / n, b = r % n;
    int s = (int)(m / nk), k = (int)(m % nk);
    dmT[(((int64_t)k * ns + s) * n + a) * n + b] = dm[e - r + (int64_t)b * n + a];
  }
}

// F[s][k0+kk][ij] += scale * sum_{k'} P[kk][s][k'][ij], summed in k' order
__global__ void exchange_reduce_kernel(const cplx* P, cplx* F, int kbk, int ns, int nk, int k0, int64_t nao2,
                                       double scale) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)kbk * ns * nao2) return;
  const int64_t ij = e % nao2;
  const int64_t ks = e / nao2;  // kk * ns + s
  const int s = (int)(ks % ns), kk = (int)(ks / ns);
  const cplx* p = P + ks * nk * nao2 + ij;
  double re = 0.0, im = 0.0;
  for (int kp = 0; kp < nk; ++kp) {
    re += p[(int64_t)kp * nao2].x;
    im += p[(int64_t)kp * nao2].y;
  }
  cplx* f = F + ((int64_t)s * nk + k0 + kk) * nao2 + ij;
  f->x += scale * re;
  f->y += scale * im;
}

// offset of the diagonal pair (k,k) for the block index k*nb + b
__global__ void diag_pair_table_kernel(int64_t* tab, int nk, int nb, int64_t pe) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nk * nb) tab[i] = ((int64_t)(i / nb) * nk + i / nb) * pe;
}

// the same from the per-k offsets of the diagonal blocks of a pair subset
__global__ void diag_slot_table_kernel(int64_t* tab, const int64_t* vdiag, int nk, int nb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nk * nb) tab[i] = vdiag[i / nb];
}

// two-component dm [nk][2n][2n] -> blocks aa, bb, ab [3][nk][n][n]; S -> S_aa [nk][n][n]
__global__ void x2c_split_kernel(const cplx* dm, const cplx* S, cplx* blk, cplx* Saa, int nk, int n) {
  const int64_t n2 = (int64_t)n * n, total = (int64_t)nk * n2;
  const int64_t so = 2 * (int64_t)n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / n2, r = e % n2, i = r / n, j = r % n;
    const cplx* D = dm + k * so * so;
    blk[e] = D[i * so + j];                        // aa
    blk[total + e] = D[(i + n) * so + (j + n)];    // bb
    blk[2 * total + e] = D[i * so + (j + n)];      // ab
    Saa[e] = S[k * so * so + i * so + j];
  }
}

// blocks aa, bb, ab [3][nk][n][n] -> F [nk][2n][2n] with F_ba = F_ab^H
__global__ void x2c_assemble_kernel(const cplx* Fb, cplx* F, int nk, int n) {
  const int64_t n2 = (int64_t)n * n, total = (int64_t)nk * n2;
  const int64_t so = 2 * (int64_t)n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / n2, r = e % n2, i = r / n, j = r % n;
    cplx* O = F + k * so * so;
    O[i * so + j] = Fb[e];
    O[(i + n) * so + (j + n)] = Fb[total + e];
    const cplx ab = Fb[2 * total + e];
    O[i * so + (j + n)] = ab;
    O[(j + n) * so + i] = cconj(ab);
  }
}

ZOperand dense(const cplx* p, int64_t ld) {
  ZOperand o;
  o.ptr = p;
  o.row = lin(ld);
  o.col = lin(1);
  return o;
}

}  // namespace

// The Fock build of `nsp` blocks dm[b][k] (nao x nao) into F[b][k]:
//   direct   F[b] += sum_Q u_Q V^Q(k,k) for b < ndir, u from the blocks b < ndir;
//   exchange F[b] -= (pref/nk) sum_{k'} sum_{Q,a} [V^Q(k,k') dm[b](k')]_{ia} conj(V^Q(k,k'))_{ja};
//   Madelung F[b] -= mad_coef * S[b] dm[b] S[b], S[b][k] at S + b * s_block_stride + k * nao^2.
// The scalar kernel is nsp = ndir = ns, pref = mad_coef = 0.5 (ns = 1) or 1; the two-component
// kernel is the blocks (aa, bb, ab), ndir = 2, pref = mad_coef = 1.
// `sub` (the GW integrals hold the pair subset of the context's q range, used when no separate HF
// integrals are set): the exchange sums k' = k + q over that q range only, and the direct and
// Madelung terms belong to the context whose range holds q = 0, so the partial Fock matrices of
// ranks that split the q-points add up to the full one.
static void hf_core(Context& c, const cplx* V, const cplx* dm, int nsp, int ndir, double pref, double madelung,
                    double mad_coef, const cplx* S, int64_t s_block_stride, cplx* F, cudaStream_t st) {
  const gb200_dims& d = c.d;
  const int nk = d.nk, NQ = d.NQ;
  const int64_t nao = d.nao, nao2 = nao * nao, pe = c.pair_elems();
  GB_CUDA(cudaMemsetAsync(F, 0, (size_t)nsp * nk * nao2 * sizeof(cplx), st));
  const bool sub = V == c.V.get() && c.v_subset();
  int q0 = 0, q1 = nk;
  if (sub) {
    require(c.have_kq, GB200_ERR_STATE, "hf_fock: a pair subset of the integrals needs the k/q maps");
    q0 = std::max(0, c.q_begin);
    q1 = c.q_end < 0 ? nk : std::min(nk, c.q_end);
    require_q_pairs(c, q0, q1);
  }
  const bool own_q0 = !sub || (q0 == 0 && q1 > 0);
  // ---- direct (Hartree) term ----
  if (ndir > 0 && own_q0) {
    cplx* dmT = (cplx*)c.scratch.get(SL_HF_DMT, (size_t)ndir * nk * nao2 * sizeof(cplx));
    cplx* u = (cplx*)c.scratch.get(SL_HF_U, (size_t)NQ * sizeof(cplx));
    int64_t* tab = (int64_t*)c.scratch.get(SL_HF_TAB, (size_t)nk * ndir * sizeof(int64_t));
    {
      int64_t total = (int64_t)ndir * nk * nao2;
      unsigned g = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
      dm_transpose_kernel<<<std::max(1u, g), 256, 0, st>>>(dm, dmT, ndir, nk, (int)nao);
      GB_CHECK_LAUNCH();
      if (sub) diag_slot_table_kernel<<<(unsigned)((nk * ndir + 255) / 256), 256, 0, st>>>(tab, c.tab_v_diag.get(), nk, ndir);
      else diag_pair_table_kernel<<<(unsigned)((nk * ndir + 255) / 256), 256, 0, st>>>(tab, nk, ndir, pe);
      GB_CHECK_LAUNCH();
    }
    ZGemm g;  // u[Q] = (1/nk) sum_{(k,b),(a,a')} V(k,k)[Q][a][a'] dmT[(k,b)][a][a']
    g.M = NQ; g.N = 1; g.K = (int64_t)nk * ndir * nao2;
    g.A.ptr = V; g.A.row = lin(nao2); g.A.col = twotab(nao2, 1, tab);
    g.B.ptr = dmT; g.B.row = lin(1); g.B.col = lin(0);
    g.C.ptr = u; g.C.row = lin(1); g.C.col = lin(0);
    g.alpha = cmk(1.0 / nk, 0.0);
    zgemm_fp64(g, st);
    ZGemm h;  // F[b][k][(i,j)] += sum_Q u[Q] V(k,k)[Q][(i,j)]  for b < ndir
    h.M = 1; h.N = nao2; h.K = NQ;
    h.nb0 = nk; h.nb2 = ndir;
    h.A.ptr = u; h.A.row = lin(0); h.A.col = lin(1);
    h.B.ptr = V; h.B.row = lin(nao2); h.B.col = lin(1);
    if (sub) h.B.bat.tab0 = c.tab_v_diag.get();  // block (k,k) of the subset
    else h.B.bat.s0 = ((int64_t)nk + 1) * pe;     // pair (k,k) of the full [nk][nk] storage
    h.C.ptr = F; h.C.row = lin(0); h.C.col = lin(1);
    h.C.bat.s0 = nao2; h.C.bat.s2 = (int64_t)nk * nao2;
    h.beta = cmk(1.0, 0.0);
    zgemm_fp64(h, st);
  }
  // ---- exchange term over the q range of a pair subset: per q, all k at once ----
  if (sub) {
    cplx* Y = (cplx*)c.scratch.get(SL_HF_Y, (size_t)nk * nsp * pe * sizeof(cplx));
    for (int q = q0; q < q1; ++q) {
      const int64_t* tVp = c.tab_pair_plus.get() + (int64_t)q * nk;  // V(k, k+q)
      const int64_t* tDp = c.tab_g_plus.get() + (int64_t)q * nk;     // block k+q of dm
      ZGemm y;  // Y[k][b][(Q,i)][a] = sum_a' V(k,k+q)[(Q,i)][a'] dm[b][k+q][a'][a]
      y.M = (int64_t)NQ * nao; y.N = nao; y.K = nao;
      y.nb0 = nk; y.nb1 = nsp;
      y.A = dense(V, nao); y.A.bat.tab0 = tVp;
      y.B = dense(dm, nao); y.B.bat.tab0 = tDp; y.B.bat.s1 = (int64_t)nk * nao2;
      y.C.ptr = Y; y.C.row = lin(nao); y.C.col = lin(1);
      y.C.bat.s0 = (int64_t)nsp * pe; y.C.bat.s1 = pe;
      zgemm_fp64(y, st);
      ZGemm x;  // F[b][k][i][j] -= (pref/nk) sum_{Q,a} Y[k][b][Q][i][a] conj(V(k,k+q)[Q][j][a])
      x.M = nao; x.N = nao; x.K = (int64_t)NQ * nao;
      x.nb0 = nk; x.nb1 = nsp;
      x.A.ptr = Y; x.A.row = lin(nao); x.A.col = two(nao, 1, nao2);
      x.A.bat.s0 = (int64_t)nsp * pe; x.A.bat.s1 = pe;
      x.B.ptr = V; x.B.row = two(nao, 1, nao2); x.B.col = lin(nao); x.B.conj = true;
      x.B.bat.tab0 = tVp;
      x.C.ptr = F; x.C.row = lin(nao); x.C.col = lin(1);
      x.C.bat.s0 = nao2; x.C.bat.s1 = (int64_t)nk * nao2;
      x.alpha = cmk(-pref / nk, 0.0); x.beta = cmk(1.0, 0.0);
      zgemm_fp64(x, st);
    }
  }
  // ---- exchange term, blocked over k ----
  // Per k the exchange is an nao x nao result contracted over K = (k', Q, a), i.e. nk*NQ*nao
  // terms.  One batch of the second contraction per (k, b, k') keeps the GPU busy (a single
  // batch per k would leave most SMs idle); the per-k' partial results are then summed in k'
  // order by exchange_reduce_kernel, so the result is deterministic.
  if (!sub) {
    const int64_t per_k = (int64_t)nsp * nk * pe;
    const double budget = c.budget_or(8e9, 0.5);
    int kb = (int)std::max(1.0, std::floor(budget / ((double)per_k * sizeof(cplx))));
    kb = std::min(kb, nk);
    cplx* Y = (cplx*)c.scratch.get(SL_HF_Y, (size_t)kb * per_k * sizeof(cplx));
    cplx* P = (cplx*)c.scratch.get(SL_TMP, (size_t)kb * nsp * nk * nao2 * sizeof(cplx));
    for (int k0 = 0; k0 < nk; k0 += kb) {
      const int kbk = std::min(kb, nk - k0);
      ZGemm y;  // Y[kk][b][k'][(Q,i)][a] = sum_a' V(k,k')[(Q,i)][a'] dm[b][k'][a'][a]
      y.M = (int64_t)NQ * nao; y.N = nao; y.K = nao;
      y.nb0 = kbk; y.nb1 = nsp; y.nb2 = nk;
      y.A = dense(V + (int64_t)k0 * nk * pe, nao);
      y.A.bat.s0 = (int64_t)nk * pe; y.A.bat.s2 = pe;
      y.B = dense(dm, nao); y.B.bat.s1 = (int64_t)nk * nao2; y.B.bat.s2 = nao2;
      y.C.ptr = Y; y.C.row = lin(nao); y.C.col = lin(1);
      y.C.bat.s0 = per_k; y.C.bat.s1 = (int64_t)nk * pe; y.C.bat.s2 = pe;
      zgemm_fp64(y, st);
      ZGemm x;  // P[kk][b][k'][i][j] = sum_{Q,a} Y[kk][b][k'][Q][i][a] conj(V(k,k')[Q][j][a])
      x.M = nao; x.N = nao; x.K = (int64_t)NQ * nao;
      x.nb0 = kbk; x.nb1 = nsp; x.nb2 = nk;
      x.A.ptr = Y; x.A.row = lin(nao); x.A.col = two(nao, 1, nao2);
      x.A.bat.s0 = per_k; x.A.bat.s1 = (int64_t)nk * pe; x.A.bat.s2 = pe;
      x.B.ptr = V + (int64_t)k0 * nk * pe; x.B.row = two(nao, 1, nao2); x.B.col = lin(nao); x.B.conj = true;
      x.B.bat.s0 = (int64_t)nk * pe; x.B.bat.s2 = pe;
      x.C.ptr = P; x.C.row = lin(nao); x.C.col = lin(1);
      x.C.bat.s0 = (int64_t)nsp * nk * nao2; x.C.bat.s1 = (int64_t)nk * nao2; x.C.bat.s2 = nao2;
      zgemm_fp64(x, st);
      const int64_t nout = (int64_t)kbk * nsp * nao2;
      exchange_reduce_kernel<<<(unsigned)((nout + 255) / 256), 256, 0, st>>>(P, F, kbk, nsp, nk, k0, nao2, -pref / nk);
      GB_CHECK_LAUNCH();
    }
  }
  // ---- Madelung / Ewald term ----
  if (madelung != 0.0 && own_q0) {
    cplx* T = (cplx*)c.scratch.get(SL_TMP, (size_t)nsp * nk * nao2 * sizeof(cplx));
    ZGemm a;  // T = S dm
    a.M = nao; a.N = nao; a.K = nao; a.nb1 = nsp; a.nb2 = nk;
    a.A = dense(S, nao); a.A.bat.s1 = s_block_stride; a.A.bat.s2 = nao2;
    a.B = dense(dm, nao); a.B.bat.s1 = (int64_t)nk * nao2; a.B.bat.s2 = nao2;
    a.C.ptr = T; a.C.row = lin(nao); a.C.col = lin(1); a.C.bat.s1 = (int64_t)nk * nao2; a.C.bat.s2 = nao2;
    zgemm_fp64(a, st);
    ZGemm b;  // F -= coef * madelung * T S
    b.M = nao; b.N = nao; b.K = nao; b.nb1 = nsp; b.nb2 = nk;
    b.A = dense(T, nao); b.A.bat.s1 = (int64_t)nk * nao2; b.A.bat.s2 = nao2;
    b.B = dense(S, nao); b.B.bat.s1 = s_block_stride; b.B.bat.s2 = nao2;
    b.C.ptr = F; b.C.row = lin(nao); b.C.col = lin(1); b.C.bat.s1 = (int64_t)nk * nao2; b.C.bat.s2 = nao2;
    b.alpha = cmk(-mad_coef * madelung, 0.0); b.beta = cmk(1.0, 0.0);
    zgemm_fp64(b, st);
  }
}

void hf_fock(Context& c, const cplx* dm, const cplx* S, double madelung, cplx* F, cudaStream_t st) {
  const gb200_dims& d = c.d;
  require(c.have_Vhf || c.have_V, GB200_ERR_STATE, "hf_fock: integrals not set");
  const cplx* V = c.have_Vhf ? c.Vhf.get() : c.V.get();
  const int nk = d.nk;
  const int64_t nao = d.nao, nao2 = nao * nao;
  if (d.nso == d.nao) {
    const double pref = (d.ns == 2) ? 1.0 : 0.5;  // hf_cpu_kernels.cpp:98
    hf_core(c, V, dm, d.ns, d.ns, pref, madelung, pref, S, (int64_t)nk * nao2, F, st);
    return;
  }
  // two-component (X2C) input, hf_x2c_cpu_kernel::solve (hf_cpu_kernels.cpp:148-279): the
  // spin blocks aa, bb, ab of dm go through the scalar machinery with coefficient 1, the direct
  // term from aa + bb lands on aa and bb, the Madelung term uses S_aa, and F_ba = F_ab^H
  require(d.ns == 1 && d.nso == 2 * d.nao, GB200_ERR_INVALID, "hf_fock: two-component input needs ns = 1, nso = 2 nao");
  cplx* blk = (cplx*)c.scratch.get(SL_X2C_DM, (size_t)3 * nk * nao2 * sizeof(cplx));
  cplx* Saa = (cplx*)c.scratch.get(SL_X2C_S, (size_t)nk * nao2 * sizeof(cplx));
  cplx* Fb = (cplx*)c.scratch.get(SL_X2C_F, (size_t)3 * nk * nao2 * sizeof(cplx));
  const int64_t total = (int64_t)nk * nao2;
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
  x2c_split_kernel<<<g, 256, 0, st>>>(dm, S, blk, Saa, nk, (int)nao);
  GB_CHECK_LAUNCH();
  hf_core(c, V, blk, 3, 2, 1.0, madelung, 1.0, Saa, 0, Fb, st);
  x2c_assemble_kernel<<<g, 256, 0, st>>>(Fb, F, nk, (int)nao);
  GB_CHECK_LAUNCH();
}

}  // namespace gb200
