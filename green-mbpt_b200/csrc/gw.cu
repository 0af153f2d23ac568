// GW self-energy on one GPU: P0(tau,q) -> W(tau,q) -> Sigma(tau,k).
//
// Follows gw_cpu_kernel::solve (green-mbpt src/gw_cpu_kernel.cpp:31-134) with
// the MPI decomposition replaced by batched device contractions:
//  * the q loop stays (the reference's internode loop, :45-48);
//  * the k1 and tau loops become batch dimensions of one GEMM per step,
//    blocked over k to bound the intermediates;
//  * the three ZGEMMs per (q,k,tau) of P0_contraction (:200-215) and
//    selfenergy_contraction (:359-373) become three batched GEMMs each:
//      P0:    T1 = V G(tau,k+q);  Bt = Gbar(beta-tau,k) T1;  P0 -= pref Bt . conj(V)
//      Sigma: Y1 = V G(tau,k-q);  Y2 = Y1^T W(tau);           Sigma -= Y2 . conj(V)
//    which is the same sum, P0_QQ' = -pref sum Gbar_tp V^Q_pm G_mn conj(V^Q'_tn),
//    Sigma_ij = -sum V^Q_im G_mn W_QQ' conj(V^Q'_jn), in a batched order.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "context.cuh"
#include "split.cuh"

namespace gb200 {
namespace {

// P0(t) = herm(P0(t)/nk), P0(nts-1-t) = P0(t) for t < nts/2 (gw_cpu_kernel.cpp:217-225).
__global__ void symmetrize_p0_kernel(cplx* P0, int nts, int NQ, double inv_nk) {
  const int nth = nts / 2;
  const int64_t npairs = (int64_t)NQ * (NQ + 1) / 2;
  const int64_t total = (int64_t)nth * npairs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int t = (int)(e / npairs);
    int64_t p = e - (int64_t)t * npairs;
    int i = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > p) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= p) ++i;
    int j = (int)(p - (int64_t)i * (i + 1) / 2);
    cplx* M = P0 + (int64_t)t * NQ * NQ;
    cplx* Mm = P0 + (int64_t)(nts - 1 - t) * NQ * NQ;
    cplx a = cscale(M[(int64_t)i * NQ + j], inv_nk);
    cplx b = cscale(M[(int64_t)j * NQ + i], inv_nk);
    cplx h = cscale(cadd(a, cconj(b)), 0.5);
    M[(int64_t)i * NQ + j] = h;
    M[(int64_t)j * NQ + i] = cconj(h);
    Mm[(int64_t)i * NQ + j] = h;
    Mm[(int64_t)j * NQ + i] = cconj(h);
  }
}

// Two-component G [nts][nk][2n][2n] -> spin blocks Gab[t][s][k] = G(t,k)[a-block, b-block] and
// Gba[t][s][k] = G(t,k)[b-block, a-block] for s = 2a + b (gw_cpu_kernel.cpp:166-187: G(k+q) takes
// block (a,b), Gbar(k) block (b,a))
__global__ void x2c_pack_g_kernel(const cplx* G, cplx* Gab, cplx* Gba, int nts, int nk, int n) {
  const int64_t n2 = (int64_t)n * n, so = 2 * (int64_t)n;
  const int64_t total = (int64_t)nts * 4 * nk * n2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % n2, i = r / n, j = r % n;
    const int64_t k = (e / n2) % nk, s = (e / (n2 * nk)) % 4, t = e / (n2 * nk * 4);
    const int64_t a = s / 2, b = s % 2;
    const cplx* M = G + (t * nk + k) * so * so;
    Gab[e] = M[(a * n + i) * so + b * n + j];
    Gba[e] = M[(b * n + i) * so + a * n + j];
  }
}

// spin-block self-energy Sps[t][s][k] -> two-component Sigma [nts][nk][2n][2n], block (a,b)
__global__ void x2c_unpack_sigma_kernel(const cplx* Sps, cplx* Sigma, int nts, int nk, int n) {
  const int64_t n2 = (int64_t)n * n, so = 2 * (int64_t)n;
  const int64_t total = (int64_t)nts * 4 * nk * n2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % n2, i = r / n, j = r % n;
    const int64_t k = (e / n2) % nk, s = (e / (n2 * nk)) % 4, t = e / (n2 * nk * 4);
    const int64_t a = s / 2, b = s % 2;
    Sigma[(t * nk + k) * so * so + (a * n + i) * so + b * n + j] = Sps[e];
  }
}

// S2[k] = block-diag(S_aa(k), S_aa(k)) from two-component S [nk][2n][2n] (the q -> 0 correction
// of two-component input uses the AO overlap S_aa on every spin block, mbpt_q0_utils_t.cpp:142-171)
__global__ void q0_x2c_overlap_kernel(const cplx* S, cplx* S2, int nk, int n) {
  const int64_t so = 2 * (int64_t)n, total = (int64_t)nk * so * so;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / (so * so), r = e % (so * so), i = r / so, j = r % so;
    const bool diag = (i < n) == (j < n);
    S2[e] = diag ? S[k * so * so + (i % n) * so + (j % n)] : cmk(0.0, 0.0);
  }
}

// T[t] *= coef[t] for T [nts][per_t]
__global__ void q0_scale_kernel(cplx* T, const cplx* coef, int nts, int64_t per_t) {
  const int64_t total = (int64_t)nts * per_t;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    T[e] = cmul(coef[e / per_t], T[e]);
}

// two-component correction: block ba = (block ab)^H (mbpt_q0_utils_t.cpp:164-168)
__global__ void q0_x2c_offdiag_kernel(cplx* D, int64_t nmat, int n) {
  const int64_t so = 2 * (int64_t)n, n2 = (int64_t)n * n, total = nmat * n2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = e / n2, r = e % n2, i = r / n, j = r % n;
    cplx* M = D + m * so * so;
    M[(j + n) * so + i] = cconj(M[i * so + (j + n)]);
  }
}

__global__ void add_kernel(cplx* Y, const cplx* X, int64_t count) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x)
    Y[e] = cadd(Y[e], X[e]);
}

inline unsigned grid_for(int64_t n, int nt) {
  int64_t g = (n + nt - 1) / nt;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

// Dense row-major matrix view helper.
ZOperand dense(const cplx* p, int64_t ld) {
  ZOperand o;
  o.ptr = p;
  o.row = lin(ld);
  o.col = lin(1);
  return o;
}

}  // namespace

void build_tables(Context& c) {
  // G offsets address the spin-block layout the contractions read: [t][s][k][nao][nao] (for
  // two-component input the 4 spin blocks repacked by gw_sigma)
  const int nk = c.d.nk, ns = c.ns_eff();
  const int64_t pe = c.pair_elems();
  const int64_t ge = (int64_t)c.d.nao * c.d.nao;
  std::vector<int64_t> pp(nk * nk), pm(nk * nk), gp(nk * nk), gm(nk * nk), ppns((size_t)nk * nk * ns);
  for (int q = 0; q < nk; ++q)
    for (int k = 0; k < nk; ++k) {
      int kp = c.kplus[(size_t)k * nk + q];
      int km = c.kminus[(size_t)k * nk + q];
      // V(k, k+q) and V(k, k-q); a block this context does not hold gets offset 0 (the q-points
      // that would read it are refused by require_q_pairs)
      pp[(size_t)q * nk + k] = std::max<int64_t>(0, c.v_block(k, kp)) * pe;
      pm[(size_t)q * nk + k] = std::max<int64_t>(0, c.v_block(k, km)) * pe;
      gp[(size_t)q * nk + k] = (int64_t)kp * ge;              // G(., ., k+q)
      gm[(size_t)q * nk + k] = (int64_t)km * ge;              // G(., ., k-q)
      for (int s = 0; s < ns; ++s) ppns[((size_t)q * nk + k) * ns + s] = pp[(size_t)q * nk + k];
    }
  c.tab_pair_plus.upload(pp.data(), pp.size(), c.stream);
  c.tab_pair_minus.upload(pm.data(), pm.size(), c.stream);
  c.tab_g_plus.upload(gp.data(), gp.size(), c.stream);
  c.tab_g_minus.upload(gm.data(), gm.size(), c.stream);
  c.tab_pair_plus_ns.upload(ppns.data(), ppns.size(), c.stream);
  GB_CUDA(cudaStreamSynchronize(c.stream));
}

void require_q_pairs(const Context& c, int q0, int q1) {
  if (!c.v_subset()) return;
  const int nk = c.d.nk;
  for (int q = q0; q < q1; ++q)
    for (int k = 0; k < nk; ++k) {
      const int kp = c.kplus[(size_t)k * nk + q], km = c.kminus[(size_t)k * nk + q];
      require(c.v_block(k, kp) >= 0 && c.v_block(k, km) >= 0, GB200_ERR_STATE,
              "the GW integrals hold a pair subset without V(k, k+-q) for q-point " + std::to_string(q) +
                  " (k = " + std::to_string(k) + "): set the q range the subset was chosen for");
    }
}

void build_subset_tables(Context& c) {
  const int nk = c.d.nk;
  const int64_t pe = c.pair_elems();
  std::vector<int64_t> dg(nk);
  for (int k = 0; k < nk; ++k) dg[k] = std::max<int64_t>(0, c.v_block(k, k)) * pe;  // block (k, k)
  c.tab_v_diag.upload(dg.data(), dg.size(), c.stream);
  GB_CUDA(cudaStreamSynchronize(c.stream));
}

// Choose the k-block size so that the two largest intermediates fit the budget.
static int choose_kblock(const Context& c, int64_t elems_per_k) {
  // leave headroom; at most 24 GB for the GW intermediates unless the caller set a budget
  const double budget = c.budget_or(24e9, 0.6);
  double per_k = 2.0 * (double)elems_per_k * sizeof(cplx);
  int kb = (int)std::max(1.0, std::floor(budget / per_k));
  return std::min(kb, c.d.nk);
}

cplx extrapolate_q0(const cplx* eps_n, const std::vector<double>& q_abs, int fit_order, double q_max) {
  // first occurrence of every distinct |q| in (0, q_max] (filter_q_abs), quadratic least squares
  // by the normal equations solved with full pivoting (polyfit); rank-deficient systems take 0
  // for the undetermined coefficients
  std::vector<double> x, y;
  for (size_t i = 0; i < q_abs.size(); ++i) {
    const double qa = q_abs[i];
    if (!(qa > 0.0 && qa <= q_max)) continue;
    if (std::find(x.begin(), x.end(), qa) != x.end()) continue;
    x.push_back(qa);
    y.push_back(eps_n[i].x);
  }
  const int m = fit_order + 1;
  std::vector<double> A((size_t)m * m, 0.0), b(m, 0.0);
  for (size_t i = 0; i < x.size(); ++i) {
    std::vector<double> row(m);
    for (int j = 0; j < m; ++j) row[j] = std::pow(x[i], j);
    for (int r = 0; r < m; ++r) {
      b[r] += row[r] * y[i];
      for (int cc = 0; cc < m; ++cc) A[r * m + cc] += row[r] * row[cc];
    }
  }
  std::vector<int> colp(m);
  for (int j = 0; j < m; ++j) colp[j] = j;
  double amax = 0.0;
  for (double v : A) amax = std::max(amax, std::fabs(v));
  int rank = 0;
  for (int piv = 0; piv < m; ++piv) {
    int pr = piv, pc = piv;
    double best = -1.0;
    for (int r = piv; r < m; ++r)
      for (int cc = piv; cc < m; ++cc)
        if (std::fabs(A[r * m + cc]) > best) { best = std::fabs(A[r * m + cc]); pr = r; pc = cc; }
    if (best <= 1e-14 * amax || best == 0.0) break;
    for (int cc = 0; cc < m; ++cc) std::swap(A[piv * m + cc], A[pr * m + cc]);
    std::swap(b[piv], b[pr]);
    for (int r = 0; r < m; ++r) std::swap(A[r * m + piv], A[r * m + pc]);
    std::swap(colp[piv], colp[pc]);
    for (int r = piv + 1; r < m; ++r) {
      const double f = A[r * m + piv] / A[piv * m + piv];
      for (int cc = piv; cc < m; ++cc) A[r * m + cc] -= f * A[piv * m + cc];
      b[r] -= f * b[piv];
    }
    ++rank;
  }
  std::vector<double> z(m, 0.0);
  for (int r = rank - 1; r >= 0; --r) {
    double v = b[r];
    for (int cc = r + 1; cc < rank; ++cc) v -= A[r * m + cc] * z[cc];
    z[r] = v / A[r * m + r];
  }
  std::vector<double> coef(m, 0.0);
  for (int j = 0; j < m; ++j) coef[colp[j]] = z[j];
  return cmk(coef[0], 0.0);
}

// Sigma += -madelung eps_inv_q0(t) S G(t) S (GW_q0_correction, mbpt_q0_utils_t.cpp:88-178)
static void apply_q0(Context& c, const cplx* G, cplx* Sigma, cudaStream_t st) {
  const gb200_dims& d = c.d;
  require(c.have_H, GB200_ERR_STATE, "q0 correction: the overlap (gb200_dyson_set_hamiltonian) must be set");
  const int nk = d.nk, nts = d.nts, nw_b = d.nw_b;
  const int64_t nso = d.nso, m2 = nso * nso, nmat = (int64_t)d.ns * nk;
  std::vector<cplx> eps((size_t)nw_b * nk);
  GB_CUDA(cudaMemcpyAsync(eps.data(), c.eps_inv.get(), eps.size() * sizeof(cplx), cudaMemcpyDeviceToHost, st));
  GB_CUDA(cudaStreamSynchronize(st));
  std::vector<cplx> ew(nw_b), coef(nts);
  for (int n = 0; n < nw_b; ++n) ew[n] = extrapolate_q0(eps.data() + (size_t)n * nk, c.q_abs, 2, 1.0);
  for (int t = 0; t < nts; ++t) {
    cplx acc = cmk(0.0, 0.0);
    for (int n = 0; n < nw_b; ++n) acc = cadd(acc, cmul(c.Ttn_b_host[(size_t)t * nw_b + n], ew[n]));
    coef[t] = cscale(acc, -c.q0_madelung);
  }
  cplx* dcoef = (cplx*)c.scratch.get(SL_Q0_E, (size_t)nts * sizeof(cplx));
  GB_CUDA(cudaMemcpyAsync(dcoef, coef.data(), (size_t)nts * sizeof(cplx), cudaMemcpyHostToDevice, st));
  const cplx* Sm = c.S.get();
  if (c.x2c()) {
    cplx* S2 = (cplx*)c.scratch.get(SL_Q0_S, (size_t)nk * m2 * sizeof(cplx));
    q0_x2c_overlap_kernel<<<grid_for((int64_t)nk * m2, 256), 256, 0, st>>>(c.S.get(), S2, nk, (int)d.nao);
    GB_CHECK_LAUNCH();
    Sm = S2;
  }
  const int64_t per_t = nmat * m2;
  cplx* T = (cplx*)c.scratch.get(SL_Q0_T, (size_t)nts * per_t * sizeof(cplx));
  cplx* D = (cplx*)c.scratch.get(SL_Q0_D, (size_t)nts * per_t * sizeof(cplx));
  ZGemm a;  // T[t][sk] = S[sk] G[t][sk]
  a.M = nso; a.N = nso; a.K = nso; a.nb1 = nts; a.nb2 = nmat;
  a.A = dense(Sm, nso); a.A.bat.s2 = m2;
  a.B = dense(G, nso); a.B.bat.s1 = per_t; a.B.bat.s2 = m2;
  a.C.ptr = T; a.C.row = lin(nso); a.C.col = lin(1); a.C.bat.s1 = per_t; a.C.bat.s2 = m2;
  zgemm_fp64(a, st);
  q0_scale_kernel<<<grid_for((int64_t)nts * per_t, 256), 256, 0, st>>>(T, dcoef, nts, per_t);
  GB_CHECK_LAUNCH();
  ZGemm b;  // D[t][sk] = T[t][sk] S[sk]
  b.M = nso; b.N = nso; b.K = nso; b.nb1 = nts; b.nb2 = nmat;
  b.A = dense(T, nso); b.A.bat.s1 = per_t; b.A.bat.s2 = m2;
  b.B = dense(Sm, nso); b.B.bat.s2 = m2;
  b.C.ptr = D; b.C.row = lin(nso); b.C.col = lin(1); b.C.bat.s1 = per_t; b.C.bat.s2 = m2;
  zgemm_fp64(b, st);
  if (c.x2c()) {
    q0_x2c_offdiag_kernel<<<grid_for((int64_t)nts * nmat * d.nao * d.nao, 256), 256, 0, st>>>(D, (int64_t)nts * nmat,
                                                                                             (int)d.nao);
    GB_CHECK_LAUNCH();
  }
  add_kernel<<<grid_for((int64_t)nts * per_t, 256), 256, 0, st>>>(Sigma, D, (int64_t)nts * per_t);
  GB_CHECK_LAUNCH();
}

namespace {

// One GW self-energy evaluation of a context, in the steps that the single-system loop and the
// batched loop both drive: per q-point the P0 contractions of each k-block, the aux-basis solve,
// and the Sigma contractions of each k-block (gw_cpu_kernel.cpp:31-72,74-134).
struct GwRun {
  Context& c;
  cudaStream_t st;
  const gb200_dims& d;
  bool x2c;
  int nk, ns, nts, nth, NQ, nw_b;
  int64_t nao, nao2, pe, ge, g_s, g_t;
  double pref;
  cplx* Sigma_out;
  const cplx* G_in;
  const cplx* G;
  const cplx* Gbar;  // the operand of Gbar(beta - tau, k): block (b,a) for two-component input
  cplx* Sigma;
  int kb = 1;
  int64_t per_k_sigma = 0;
  cplx *P0 = nullptr, *Pw = nullptr, *Pinv = nullptr, *aug = nullptr, *X1 = nullptr, *X2 = nullptr;
  int q0 = 0, q1 = 0;
  // exponent sink (split precision on the tensor cores): (e) records the column exponents of Y2
  // for (f) as it stores Y2, so that slicing Y2 needs no separate exponent pass.  Measured on the
  // c2 shapes it costs (e) about 0.4 of the pass it saves; in the epilogue-bound (b) it would cost
  // more than the pass for Bt, so (b) -> (c) keeps the pass.
  bool sink_s = false;
  int32_t* sink = nullptr;
  int64_t sink_ld_s = 0;

  GwRun(Context& c_, const cplx* G_, cplx* Sigma_, cudaStream_t st_) : c(c_), st(st_), d(c_.d) {
    require(d.nts % 2 == 0, GB200_ERR_WRONG_GRID, "Number of tau points should be even!!!");
    require(c.have_kq && c.have_grid && c.have_V, GB200_ERR_STATE, "gw_sigma: k/q maps, grid and integrals must be set");
    // two-component input: the contractions run over the 4 spin blocks of G (pseudo spins,
    // gw_cpu_kernel.cpp:166-168,326-327) on a repacked copy, prefactor 1
    x2c = c.x2c();
    nk = d.nk; ns = c.ns_eff(); nts = d.nts; nth = nts / 2; NQ = d.NQ; nw_b = d.nw_b;
    nao = d.nao; nao2 = nao * nao;
    pe = c.pair_elems();
    ge = nao2;                      // one G matrix
    g_s = (int64_t)nk * ge;         // stride of spin in G
    g_t = (int64_t)ns * g_s;        // stride of tau in G
    pref = (d.ns == 2 || x2c) ? 1.0 : 2.0;  // gw_cpu_kernel.cpp:167
    Sigma_out = Sigma_;
    G_in = G_;
    G = G_;
    Gbar = G_;
    Sigma = Sigma_;
    if (x2c) {
      const int64_t n = (int64_t)nts * 4 * nk * nao2;
      cplx* Gab = (cplx*)c.scratch.get(SL_X2C_GAB, (size_t)n * sizeof(cplx));
      cplx* Gba = (cplx*)c.scratch.get(SL_X2C_GBA, (size_t)n * sizeof(cplx));
      x2c_pack_g_kernel<<<grid_for(n, 256), 256, 0, st>>>(G_, Gab, Gba, nts, nk, (int)nao);
      GB_CHECK_LAUNCH();
      G = Gab;
      Gbar = Gba;
      Sigma = (cplx*)c.scratch.get(SL_X2C_SIG, (size_t)n * sizeof(cplx));
    }
    GB_CUDA(cudaMemsetAsync(Sigma, 0, (size_t)nts * ns * nk * nao2 * sizeof(cplx), st));
    per_k_sigma = (int64_t)nts * ns * pe;
    kb = choose_kblock(c, per_k_sigma);
    P0 = (cplx*)c.scratch.get(SL_P0, (size_t)nts * NQ * NQ * sizeof(cplx));
    Pw = (cplx*)c.scratch.get(SL_PW, (size_t)nw_b * NQ * NQ * sizeof(cplx));
    Pinv = (cplx*)c.scratch.get(SL_PINV, (size_t)nw_b * NQ * NQ * sizeof(cplx));
    aug = (cplx*)c.scratch.get(SL_AUG, (size_t)nw_b * NQ * 2 * NQ * sizeof(cplx));
    X1 = (cplx*)c.scratch.get(SL_Y1, (size_t)kb * per_k_sigma * sizeof(cplx));
    X2 = (cplx*)c.scratch.get(SL_Y2, (size_t)kb * per_k_sigma * sizeof(cplx));
    if (c.prec_mode == GB200_PREC_SPLIT && c.split_core == 0 && nao % 8 == 0) {
      auto slices_of = [&](int stage) { return c.contraction_slices[stage] > 0 ? c.contraction_slices[stage] : c.slices; };
      sink_s = NQ <= split_max_chunk(slices_of(4));
      sink_ld_s = (int64_t)nts * ns * nao;
      if (sink_s) sink = (int32_t*)c.scratch.get(SL_SINK, (size_t)kb * sink_ld_s * sizeof(int32_t));
    }
    if (c.q0_on) {
      require(c.q_begin <= 0 && (c.q_end < 0 || c.q_end >= nk), GB200_ERR_INVALID,
              "q0 correction: needs all q-points in one context (it extrapolates over q)");
      c.eps_inv.alloc((size_t)nw_b * nk);
    }
    // this context's share of the q loop (gw_cpu_kernel.cpp:45 distributes q over nodes the same
    // way); the partial Sigma is already divided by nk, so shards sum to the full self-energy
    q0 = std::max(0, c.q_begin);
    q1 = c.q_end < 0 ? nk : std::min(nk, c.q_end);
    require_q_pairs(c, q0, q1);
  }

  int nkblocks() const { return (nk + kb - 1) / kb; }

  // ---------------- polarization P0(tau, q), tau in the first half ---------
  void p0_begin(int) { GB_CUDA(cudaMemsetAsync(P0, 0, (size_t)nts * NQ * NQ * sizeof(cplx), st)); }

  void p0_gemms(int q, int k0, ZGemm (&out)[3]) {
    const int kbk = std::min(kb, nk - k0);
    const int64_t* tVp = c.tab_pair_plus.get() + (int64_t)q * nk + k0;
    const int64_t* tGp = c.tab_g_plus.get() + (int64_t)q * nk + k0;
    const int64_t blkT1 = (int64_t)nth * ns * pe;  // per kk in T1
      // (a) T1[kk][t][s][(Q,p)][n] = sum_m V(k,k+q)[(Q,p)][m] G(t,s,k+q)[m][n], computed as its
    //     transpose T1^T = G^T V^T so that the large operand V is the right (column) operand:
    //     rows ((t,s),n) (M = nth*ns*nao), columns (Q,p) (N = NQ*nao), K = m
    ZGemm a;
    a.M = (int64_t)nth * ns * nao; a.N = (int64_t)NQ * nao; a.K = nao;
    a.nb0 = kbk;
    a.A.ptr = G; a.A.row = two(nao, 1, g_s); a.A.col = lin(nao); a.A.bat.tab0 = tGp;
    a.B.ptr = c.V.get(); a.B.row = lin(1); a.B.col = lin(nao); a.B.bat.tab0 = tVp;
    a.C.ptr = X1; a.C.row = two(nao, 1, pe); a.C.col = lin(nao);
    a.C.bat.s0 = blkT1;
    // (b) Bt[t][kk][s][Q][r][n] = sum_p Gbar(nts-1-t, s, k)[r][p] T1[kk][t][s][Q][p][n]
    ZGemm b;
    b.M = nao; b.N = (int64_t)NQ * nao; b.K = nao;
    b.nb0 = kbk; b.nb1 = nth; b.nb2 = ns;
    b.A = dense(Gbar + (int64_t)(nts - 1) * g_t + (int64_t)k0 * ge, nao);
    b.A.bat.s0 = ge; b.A.bat.s1 = -g_t; b.A.bat.s2 = g_s;
    b.B.ptr = X1; b.B.row = lin(nao); b.B.col = two(nao, 1, nao2);
    b.B.bat.s0 = blkT1; b.B.bat.s1 = (int64_t)ns * pe; b.B.bat.s2 = pe;
    b.C.ptr = X2; b.C.row = lin(nao); b.C.col = two(nao, 1, nao2);
    b.C.bat.s0 = (int64_t)ns * pe; b.C.bat.s1 = (int64_t)kbk * ns * pe; b.C.bat.s2 = pe;
    // (c) P0[t][Q][Q'] -= pref sum_{(kk,s),(r,n)} Bt[t][(kk,s)][Q][(r,n)] conj(V(k,k+q)[Q'][(r,n)]),
    //     computed as P0^T = conj(V) Bt^T: the tau-independent V is the left operand (sliced
    //     once per call), Bt the right one; rows Q', columns Q, K = ((kk,s),(r,n))
    ZGemm cc;
    cc.M = NQ; cc.N = NQ; cc.K = (int64_t)kbk * ns * nao2;
    cc.nb0 = 1; cc.nb1 = 1; cc.nb2 = nth;
    cc.A.ptr = c.V.get(); cc.A.row = lin(nao2); cc.A.conj = true;
    cc.A.col = twotab(nao2, 1, c.tab_pair_plus_ns.get() + ((int64_t)q * nk + k0) * ns);
    cc.B.ptr = X2; cc.B.col = lin(nao2); cc.B.row = two(nao2, 1, (int64_t)NQ * nao2);
    cc.B.bat.s2 = (int64_t)kbk * ns * pe;
    cc.C.ptr = P0; cc.C.row = lin(1); cc.C.col = lin(NQ); cc.C.bat.s2 = (int64_t)NQ * NQ;
    cc.alpha = cmk(-pref, 0.0); cc.beta = cmk(1.0, 0.0);
    out[0] = a;
    out[1] = b;
    out[2] = cc;
  }

  // ---------------- screened interaction (gw_cpu_kernel.cpp:227-279) -------
  void w_solve(int q) {
    {  // P0 = herm(P0 / nk), P0(beta - tau) = P0(tau) (gw_cpu_kernel.cpp:217-225)
      int64_t total = (int64_t)nth * NQ * (NQ + 1) / 2;
      symmetrize_p0_kernel<<<grid_for(total, 256), 256, 0, st>>>(P0, nts, NQ, 1.0 / nk);
      GB_CHECK_LAUNCH();
    }
    {
      ZGemm f;  // Pw[n] = sum_t Tnt_b[n][t] P0[t]
      f.M = nw_b; f.N = (int64_t)NQ * NQ; f.K = nts;
      f.A = dense(c.Tnt_b.get(), nts);
      f.B = dense(P0, (int64_t)NQ * NQ);
      f.C.ptr = Pw; f.C.row = lin((int64_t)NQ * NQ); f.C.col = lin(1);
      zgemm_fp64(f, st);
      // temp = LDLT(I - Pw)^-1 on the lower triangle, then hermitize
      invert_large_batched(Pw, Pinv, aug, nw_b, NQ, true, true, st);
      hermitize_batched(Pinv, nw_b, NQ, 1.0, st);
      ZGemm m;  // Pw[n] <- temp[n] Pw[n] (written to aug as scratch, then used)
      m.M = NQ; m.N = NQ; m.K = NQ; m.nb2 = nw_b;
      m.A = dense(Pinv, NQ); m.A.bat.s2 = (int64_t)NQ * NQ;
      m.B = dense(Pw, NQ); m.B.bat.s2 = (int64_t)NQ * NQ;
      m.C.ptr = aug; m.C.row = lin(NQ); m.C.col = lin(1); m.C.bat.s2 = (int64_t)NQ * NQ;
      zgemm_fp64(m, st);
      if (c.q0_on) {
        // head of P(i Omega_n, q) on the plane-wave G = 0 component: eps_inv[n][q] =
        // conj(A_q) P(i Omega_n) A_q (aux_to_PW_00, mbpt_q0_utils_t.cpp:11-20)
        cplx* y = (cplx*)c.scratch.get(SL_Q0_Y, (size_t)nw_b * NQ * sizeof(cplx));
        const cplx* Aq = c.AqQ.get() + (int64_t)q * NQ;
        ZGemm hy;  // y[n][Q] = sum_Q' P[n][Q][Q'] A_q[Q']
        hy.M = NQ; hy.N = 1; hy.K = NQ; hy.nb2 = nw_b;
        hy.A = dense(aug, NQ); hy.A.bat.s2 = (int64_t)NQ * NQ;
        hy.B.ptr = Aq; hy.B.row = lin(1); hy.B.col = lin(0);
        hy.C.ptr = y; hy.C.row = lin(1); hy.C.col = lin(0); hy.C.bat.s2 = NQ;
        zgemm_fp64(hy, st);
        ZGemm he;  // eps_inv[n][q] = sum_Q conj(A_q[Q]) y[n][Q]
        he.M = 1; he.N = 1; he.K = NQ; he.nb2 = nw_b;
        he.A.ptr = Aq; he.A.row = lin(0); he.A.col = lin(1); he.A.conj = true;
        he.B.ptr = y; he.B.row = lin(1); he.B.col = lin(0); he.B.bat.s2 = NQ;
        he.C.ptr = c.eps_inv.get() + q; he.C.row = lin(0); he.C.col = lin(0); he.C.bat.s2 = nk;
        zgemm_fp64(he, st);
      }
      ZGemm bt;  // W(tau) = sum_n Ttn_b[t][n] P(i Omega_n) -> stored in P0
      bt.M = nts; bt.N = (int64_t)NQ * NQ; bt.K = nw_b;
      bt.A = dense(c.Ttn_b.get(), nw_b);
      bt.B = dense(aug, (int64_t)NQ * NQ);
      bt.C.ptr = P0; bt.C.row = lin((int64_t)NQ * NQ); bt.C.col = lin(1);
      zgemm_fp64(bt, st);
    }
  }

  // ---------------- self-energy contribution of this q ---------------------
  void sigma_gemms(int q, int k0, ZGemm (&out)[3]) {
    const int kbk = std::min(kb, nk - k0);
    const int64_t* tVm = c.tab_pair_minus.get() + (int64_t)q * nk + k0;
    const int64_t* tGm = c.tab_g_minus.get() + (int64_t)q * nk + k0;
    const int64_t blk = (int64_t)nts * ns * pe;  // per kk in Y1 / Y2
      // (d) Y1[kk][t][s][(Q,i)][n] = sum_m V(k,k-q)[(Q,i)][m] G(t,s,k-q)[m][n], as its transpose
    //     (V the right operand): rows ((t,s),n), columns (Q,i), K = m
    ZGemm dd;
    dd.M = (int64_t)nts * ns * nao; dd.N = (int64_t)NQ * nao; dd.K = nao;
    dd.nb0 = kbk;
    dd.A.ptr = G; dd.A.row = two(nao, 1, g_s); dd.A.col = lin(nao); dd.A.bat.tab0 = tGm;
    dd.B.ptr = c.V.get(); dd.B.row = lin(1); dd.B.col = lin(nao); dd.B.bat.tab0 = tVm;
    dd.C.ptr = X1; dd.C.row = two(nao, 1, pe); dd.C.col = lin(nao);
    dd.C.bat.s0 = blk;
    // (e) Y2[kk][t][s][(i,n)][Q'] = sum_Q Y1[kk][t][s][Q][(i,n)] W(t)[Q][Q'], as Y2^T = W^T Y1:
    //     the small W(t) is the left operand, Y1 the right one; rows Q', columns (kk,(i,n)), K = Q
    ZGemm e;
    e.M = NQ; e.N = (int64_t)kbk * nao2; e.K = NQ;
    e.nb0 = 1; e.nb1 = nts; e.nb2 = ns;
    e.A.ptr = P0; e.A.row = lin(1); e.A.col = lin(NQ); e.A.bat.s1 = (int64_t)NQ * NQ;
    e.B.ptr = X1; e.B.row = lin(nao2); e.B.col = two(nao2, 1, blk);
    e.B.bat.s1 = (int64_t)ns * pe; e.B.bat.s2 = pe;
    e.C.ptr = X2; e.C.row = lin(1); e.C.col = two(nao2, NQ, blk);
    e.C.bat.s1 = (int64_t)ns * pe; e.C.bat.s2 = pe;
    // (f) Sigma[t][s][k][i][j] -= sum_{(n,Q')} Y2[kk][t][s][i][(n,Q')] conj(V(k,k-q)[Q'][j][n]), as
    //     Sigma^T = conj(V) Y2^T: rows j (M = nao), columns ((t,s),i) (N = nts*ns*nao),
    //     K = (n,Q'); the large Y2 is the right operand
    ZGemm f;
    f.M = nao; f.N = (int64_t)nts * ns * nao; f.K = nao * NQ;
    f.nb0 = kbk;
    f.A.ptr = c.V.get(); f.A.row = lin(nao); f.A.col = two(NQ, nao2, 1); f.A.conj = true;
    f.A.bat.tab0 = tVm;
    f.B.ptr = X2; f.B.row = lin(1); f.B.col = two(nao, nao * NQ, pe);
    f.B.bat.s0 = blk;
    f.C.ptr = Sigma + (int64_t)k0 * ge; f.C.row = lin(1); f.C.col = two(nao, nao, g_s);
    f.C.bat.s0 = ge;
    f.alpha = cmk(-1.0, 0.0); f.beta = cmk(1.0, 0.0);
    if (sink_s) {
      // column ((t,s),i) of (f)'s B in batch kk: Y2[kk][t][s][i][*], i.e. (e)'s columns
      // (kk,(i,n)) in its batch (t, s): entry kk ld + (t ns + s) nao + i
      e.sink.expo = sink; e.sink.c1 = (int64_t)ns * nao; e.sink.c2 = nao;
      e.sink.d1 = nao; e.sink.m1 = nao; e.sink.s1 = 1; e.sink.d2 = nao2; e.sink.s2 = sink_ld_s;
      e.sink.count = (int64_t)kbk * sink_ld_s;
      f.B_expo = sink; f.B_expo_ld = sink_ld_s;
    }
    out[0] = dd;
    out[1] = e;
    out[2] = f;
  }

  void finish() {
    scale_inplace(Sigma, (int64_t)nts * ns * nk * nao2, 1.0 / nk, st);  // gw_cpu_kernel.cpp:55
    if (x2c) {
      const int64_t n = (int64_t)nts * 4 * nk * nao2;
      x2c_unpack_sigma_kernel<<<grid_for(n, 256), 256, 0, st>>>(Sigma, Sigma_out, nts, nk, (int)nao);
      GB_CHECK_LAUNCH();
    }
    if (c.q0_on) apply_q0(c, G_in, Sigma_out, st);
  }
};

// slices of contraction `stage` of a context in split precision (0: FP64)
int stage_slices(const Context& c, int stage) {
  if (c.prec_mode != GB200_PREC_SPLIT) return 0;
  return c.contraction_slices[stage] > 0 ? c.contraction_slices[stage] : c.slices;
}

void check_split_error(Context& c, cudaStream_t st) {
  if (c.prec_mode != GB200_PREC_SPLIT) return;
  int e = split_check_error(c, st);
  require(e == 0, GB200_ERR_CUDA, "split contraction: tensor-core pipeline wait timed out (code " + std::to_string(e) + ")");
}

}  // namespace

void gw_sigma(Context& c, const cplx* G, cplx* Sigma, cudaStream_t st) {
  for (int i = 0; i < 5; ++i)
    if (!c.ev[i]) GB_CUDA(cudaEventCreate(&c.ev[i]));
  GB_CUDA(cudaEventRecord(c.ev[0], st));
  GwRun r(c, G, Sigma, st);
  // the P0 and Sigma contractions run in the selected precision; the
  // transforms and the aux-basis solve always run in FP64
  SplitEngine* se = c.prec_mode == GB200_PREC_SPLIT ? split_engine(c) : nullptr;
  auto contract = [&](const ZGemm& g, int stage) {
    if (se) split_gemm(c, *se, g, st, c.contraction_slices[stage]);
    else zgemm_fp64(g, st);
  };
  // stage timings: events recorded on the stream and read after the loop, so the host never
  // waits inside it
  const size_t nev = (size_t)std::max(0, r.q1 - r.q0) * 4;
  while (c.qev.size() < nev) {
    cudaEvent_t e;
    GB_CUDA(cudaEventCreate(&e));
    c.qev.push_back(e);
  }
  ZGemm g3[3];
  for (int q = r.q0; q < r.q1; ++q) {
    cudaEvent_t* qe = c.qev.data() + (size_t)(q - r.q0) * 4;
    GB_CUDA(cudaEventRecord(qe[0], st));
    r.p0_begin(q);
    for (int k0 = 0; k0 < r.nk; k0 += r.kb) {
      r.p0_gemms(q, k0, g3);
      for (int i = 0; i < 3; ++i) contract(g3[i], i);
    }
    GB_CUDA(cudaEventRecord(qe[1], st));
    r.w_solve(q);
    GB_CUDA(cudaEventRecord(qe[2], st));
    for (int k0 = 0; k0 < r.nk; k0 += r.kb) {
      r.sigma_gemms(q, k0, g3);
      for (int i = 0; i < 3; ++i) contract(g3[i], 3 + i);
    }
    GB_CUDA(cudaEventRecord(qe[3], st));
  }
  r.finish();
  check_split_error(c, st);
  GB_CUDA(cudaEventRecord(c.ev[4], st));
  GB_CUDA(cudaEventSynchronize(c.ev[4]));
  float tot = 0, t_p0 = 0, t_w = 0, t_sig = 0;
  GB_CUDA(cudaEventElapsedTime(&tot, c.ev[0], c.ev[4]));
  for (int q = r.q0; q < r.q1; ++q) {
    const cudaEvent_t* qe = c.qev.data() + (size_t)(q - r.q0) * 4;
    float a_ms = 0, b_ms = 0, c_ms = 0;
    GB_CUDA(cudaEventElapsedTime(&a_ms, qe[0], qe[1]));
    GB_CUDA(cudaEventElapsedTime(&b_ms, qe[1], qe[2]));
    GB_CUDA(cudaEventElapsedTime(&c_ms, qe[2], qe[3]));
    t_p0 += a_ms; t_w += b_ms; t_sig += c_ms;
  }
  c.timings[0] = t_p0; c.timings[1] = t_w; c.timings[2] = t_sig; c.timings[3] = tot;
}

void gw_sigma_batch(const std::vector<Context*>& cs, const std::vector<const cplx*>& G, const std::vector<cplx*>& Sigma,
                    cudaStream_t st) {
  require(!cs.empty() && cs.size() == G.size() && cs.size() == Sigma.size(), GB200_ERR_INVALID,
          "gw_sigma_batch: one G and one Sigma per context");
  for (size_t i = 0; i < cs.size(); ++i)
    for (size_t j = 0; j < i; ++j) require(cs[i] != cs[j], GB200_ERR_INVALID, "gw_sigma_batch: a context appears twice");
  std::vector<std::unique_ptr<GwRun>> runs;
  for (size_t i = 0; i < cs.size(); ++i) runs.emplace_back(new GwRun(*cs[i], G[i], Sigma[i], st));
  // one stage of every system that takes part: a grouped tensor-core launch when all of them run
  // that stage in split precision with the same slice count, else one contraction each
  auto contract_all = [&](std::vector<Context*>& ctx, std::vector<ZGemm>& gs, int stage) {
    if (gs.empty()) return;
    const int S = stage_slices(*ctx[0], stage);
    bool grouped = S > 0;
    for (Context* x : ctx) grouped = grouped && stage_slices(*x, stage) == S;
    if (grouped) {
      split_gemm_group(ctx, gs, st, S);
      return;
    }
    for (size_t i = 0; i < ctx.size(); ++i) {
      if (stage_slices(*ctx[i], stage) > 0) split_gemm(*ctx[i], *split_engine(*ctx[i]), gs[i], st, stage_slices(*ctx[i], stage));
      else zgemm_fp64(gs[i], st);
    }
  };
  int rounds = 0;
  for (auto& r : runs) rounds = std::max(rounds, r->q1 - r->q0);
  // round i: the i-th q-point of every system that has one, its k-blocks in step
  for (int i = 0; i < rounds; ++i) {
    std::vector<GwRun*> act;
    for (auto& r : runs)
      if (r->q0 + i < r->q1) act.push_back(r.get());
    int nblk = 0;
    for (GwRun* r : act) {
      r->p0_begin(r->q0 + i);
      nblk = std::max(nblk, r->nkblocks());
    }
    for (int half = 0; half < 2; ++half) {
      if (half == 1)
        for (GwRun* r : act) r->w_solve(r->q0 + i);
      for (int j = 0; j < nblk; ++j) {
        std::vector<Context*> ctx;
        std::vector<ZGemm> gs[3];
        for (GwRun* r : act) {
          if (j >= r->nkblocks()) continue;
          ZGemm g3[3];
          if (half == 0) r->p0_gemms(r->q0 + i, j * r->kb, g3);
          else r->sigma_gemms(r->q0 + i, j * r->kb, g3);
          ctx.push_back(&r->c);
          for (int m = 0; m < 3; ++m) gs[m].push_back(g3[m]);
        }
        for (int m = 0; m < 3; ++m) contract_all(ctx, gs[m], 3 * half + m);
      }
    }
  }
  for (auto& r : runs) r->finish();
  for (Context* x : cs) check_split_error(*x, st);
}

}  // namespace gb200
