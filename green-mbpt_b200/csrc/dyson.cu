// Dyson step, electron count / chemical potential and energies on one GPU.
//
// compute_G    : dyson.cpp:238-288 (hermitize, tau -> i w, invert, i w -> tau)
// find_mu      : dyson.cpp:101-174 (bracket by 0.5, then bisection)
// n_el(mu)     : dyson.cpp:72-99.  The reference diagonalizes S^-1 X once and
//                sums 1/(i w + mu - lambda); here the same trace is taken as
//                Tr[(z S - X)^-1 S] = sum_i 1/(z - lambda_i) with one batched
//                inverse per evaluation.
// energies     : common_utils.cpp:5-55
#include <algorithm>
#include <cmath>

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

// X[n][s][k] = H + Sigma1 + Sigma_w[n]   (mu-independent part)
__global__ void build_x_kernel(const cplx* H, const cplx* S1, const cplx* Sw, cplx* X, int64_t nmat_sk, int64_t m2, int nw) {
  const int64_t per_w = nmat_sk * m2;
  const int64_t total = (int64_t)nw * per_w;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e % per_w;
    X[e] = cadd(cadd(H[r], S1[r]), Sw[e]);
  }
}

// A[n][s][k] = (i w_n + mu) S - X[n][s][k]
__global__ void build_a_kernel(const cplx* S, const cplx* X, const double* wn, double mu, cplx* A, int64_t nmat_sk,
                               int64_t m2, int nw) {
  const int64_t per_w = nmat_sk * m2;
  const int64_t total = (int64_t)nw * per_w;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t n = e / per_w;
    int64_t r = e - n * per_w;
    cplx z = cmk(mu, wn[n]);
    A[e] = csub(cmul(z, S[r]), X[e]);
  }
}

// out[n] = sum_{s,k} w * Tr(A[n][s][k] B[s][k] or B[n][s][k])  (one block per n)
__global__ void trace_product_kernel(const cplx* A, const cplx* B, bool b_per_w, cplx* out, int64_t nmat_sk, int m,
                                     double weight) {
  const int64_t n = blockIdx.x;
  const int64_t m2 = (int64_t)m * m;
  const cplx* An = A + n * nmat_sk * m2;
  const cplx* Bn = b_per_w ? B + n * nmat_sk * m2 : B;
  double re = 0.0, im = 0.0;
  for (int64_t e = threadIdx.x; e < nmat_sk * m2; e += blockDim.x) {
    int64_t mat = e / m2;
    int r = (int)(e % m2);
    int i = r / m, j = r % m;
    cplx p = cmul(An[mat * m2 + (int64_t)i * m + j], Bn[mat * m2 + (int64_t)j * m + i]);
    re += p.x;
    im += p.y;
  }
  __shared__ double sr[256], si[256];
  sr[threadIdx.x] = re;
  si[threadIdx.x] = im;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sr[threadIdx.x] += sr[threadIdx.x + s];
      si[threadIdx.x] += si[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = cmk(sr[0] * weight, si[0] * weight);
}

// per-(s,k) traces for E_HF, E_1b: out[mat] = (Tr(dm (S1 + 2H)), Tr(dm H)), dm = pref * G(beta)
__global__ void hf_energy_kernel(const cplx* Gb, const cplx* S1, const cplx* H, double pref, int64_t nmat, int m,
                                 double* out2) {
  __shared__ double sa[256], sb[256];
  double a = 0.0, b = 0.0;
  const int64_t m2 = (int64_t)m * m;
  for (int64_t e = threadIdx.x; e < nmat * m2; e += blockDim.x) {
    int64_t mat = e / m2;
    int r = (int)(e % m2);
    int i = r / m, j = r % m;
    cplx dm = cscale(Gb[mat * m2 + (int64_t)i * m + j], pref);
    cplx h = H[mat * m2 + (int64_t)j * m + i];
    cplx s1 = S1[mat * m2 + (int64_t)j * m + i];
    a += cmul(dm, cadd(s1, cscale(h, 2.0))).x;
    b += cmul(dm, h).x;
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sb[threadIdx.x] += sb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out2[0] = sa[0];
    out2[1] = sb[0];
  }
}

double* device_wn(Context& c, cudaStream_t st) {
  double* wn = (double*)c.scratch.get(SL_RED, (size_t)(c.d.nw + 8) * sizeof(double) + (size_t)(c.d.nw + 8) * sizeof(cplx));
  GB_CUDA(cudaMemcpyAsync(wn, c.wsample_f.data(), c.d.nw * sizeof(double), cudaMemcpyHostToDevice, st));
  return wn;
}

cplx* device_red(Context& c) {
  char* base = (char*)c.scratch.get(SL_RED, (size_t)(c.d.nw + 8) * sizeof(double) + (size_t)(c.d.nw + 8) * sizeof(cplx));
  return (cplx*)(base + (size_t)(c.d.nw + 8) * sizeof(double));
}

// tau -> i w for a [nts][ns*nk*m2] array
void tau_to_omega(Context& c, const cplx* Ft, cplx* Fw, cudaStream_t st) {
  ZGemm g;
  g.M = c.d.nw; g.N = c.mat_elems(); g.K = c.d.nts;
  g.A = dense(c.Tnt_f.get(), c.d.nts);
  g.B = dense(Ft, c.mat_elems());
  g.C.ptr = Fw; g.C.row = lin(c.mat_elems()); g.C.col = lin(1);
  zgemm_fp64(g, st);
}

}  // namespace

void dyson_compute_G(Context& c, cplx* Sigma1, cplx* Sigma_tau, double mu, cplx* G, cudaStream_t st) {
  require(c.have_grid && c.have_H, GB200_ERR_STATE, "compute_G: grid and Hamiltonian must be set");
  const gb200_dims& d = c.d;
  const int64_t nsk = (int64_t)d.ns * d.nk, m2 = (int64_t)d.nso * d.nso;
  hermitize_batched(Sigma1, nsk, d.nso, 1.0, st);                       // dyson.cpp:196
  hermitize_batched(Sigma_tau, (int64_t)d.nts * nsk, d.nso, 1.0, st);   // dyson.cpp:198
  cplx* Sw = (cplx*)c.scratch.get(SL_DY_SW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* X = (cplx*)c.scratch.get(SL_DY_X, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* Gw = (cplx*)c.scratch.get(SL_DY_GW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  tau_to_omega(c, Sigma_tau, Sw, st);
  double* wn = device_wn(c, st);
  const int64_t total = (int64_t)d.nw * nsk * m2;
  build_x_kernel<<<grid_for(total, 256), 256, 0, st>>>(c.H.get(), Sigma1, Sw, X, nsk, m2, d.nw);
  GB_CHECK_LAUNCH();
  build_a_kernel<<<grid_for(total, 256), 256, 0, st>>>(c.S.get(), X, wn, mu, Sw, nsk, m2, d.nw);
  GB_CHECK_LAUNCH();
  invert_small_batched(Sw, Gw, (int64_t)d.nw * nsk, d.nso, st);
  ZGemm g;  // G(tau) = Ttn_f G(i w)
  g.M = d.nts; g.N = c.mat_elems(); g.K = d.nw;
  g.A = dense(c.Ttn_f.get(), d.nw);
  g.B = dense(Gw, c.mat_elems());
  g.C.ptr = G; g.C.row = lin(c.mat_elems()); g.C.col = lin(1);
  zgemm_fp64(g, st);
}

void dyson_prepare_X(Context& c, cplx* Sigma1, cplx* Sigma_tau, bool hermitize, cudaStream_t st) {
  require(c.have_grid && c.have_H, GB200_ERR_STATE, "find_mu: grid and Hamiltonian must be set");
  const gb200_dims& d = c.d;
  const int64_t nsk = (int64_t)d.ns * d.nk, m2 = (int64_t)d.nso * d.nso;
  if (hermitize) {
    hermitize_batched(Sigma1, nsk, d.nso, 1.0, st);
    hermitize_batched(Sigma_tau, (int64_t)d.nts * nsk, d.nso, 1.0, st);
  }
  cplx* Sw = (cplx*)c.scratch.get(SL_DY_SW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* X = (cplx*)c.scratch.get(SL_DY_X, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  tau_to_omega(c, Sigma_tau, Sw, st);
  const int64_t total = (int64_t)d.nw * nsk * m2;
  build_x_kernel<<<grid_for(total, 256), 256, 0, st>>>(c.H.get(), Sigma1, Sw, X, nsk, m2, d.nw);
  GB_CHECK_LAUNCH();
}

double dyson_electrons_prepared(Context& c, double mu, cudaStream_t st) {
  const gb200_dims& d = c.d;
  const int64_t nsk = (int64_t)d.ns * d.nk, m2 = (int64_t)d.nso * d.nso;
  cplx* A = (cplx*)c.scratch.get(SL_DY_SW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* X = (cplx*)c.scratch.get(SL_DY_X, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* Gw = (cplx*)c.scratch.get(SL_DY_GW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  double* wn = device_wn(c, st);
  cplx* red = device_red(c);
  const int64_t total = (int64_t)d.nw * nsk * m2;
  build_a_kernel<<<grid_for(total, 256), 256, 0, st>>>(c.S.get(), X, wn, mu, A, nsk, m2, d.nw);
  GB_CHECK_LAUNCH();
  invert_small_batched(A, Gw, (int64_t)d.nw * nsk, d.nso, st);
  // trace_w[n] = nkpw * sum_{s,k} weight_k Tr[G(i w_n) S]   (weight 1, nkpw = 1/nk)
  trace_product_kernel<<<d.nw, 256, 0, st>>>(Gw, c.S.get(), false, red, nsk, d.nso, 1.0 / d.nk);
  GB_CHECK_LAUNCH();
  std::vector<cplx> tw(d.nw);
  GB_CUDA(cudaMemcpyAsync(tw.data(), red, d.nw * sizeof(cplx), cudaMemcpyDeviceToHost, st));
  GB_CUDA(cudaStreamSynchronize(st));
  double re = 0.0;
  for (int n = 0; n < d.nw; ++n) re += cmul(c.Ttn_beta[n], tw[n]).x;
  const double prefactor = (d.ns == 2 || c.x2c()) ? 1.0 : 2.0;  // dyson.cpp:95
  return prefactor * -re;
}

double dyson_find_mu(Context& c, double mu0, double nel_target, double tol, double* nel_out, cudaStream_t st) {
  // dyson.cpp:101-174, same bracket/bisection sequence and stall check
  double mu = mu0, nel, nel1, nel2, nel_old, mu1, mu2;
  const double delta = 0.5;
  nel = dyson_electrons_prepared(c, mu, st);
  if (std::abs((nel - nel_target) / nel_target) > tol) {
    if (nel > nel_target) {
      mu1 = mu - delta;
      int guard = 0;
      do {
        nel1 = dyson_electrons_prepared(c, mu1, st);
        mu1 -= delta;
        require(++guard < 100000, GB200_ERR_MU_SEARCH, "Chemical potential search failed.");
      } while (nel1 > nel_target);
      mu2 = mu;
      nel2 = nel;
    } else {
      mu2 = mu + delta;
      int guard = 0;
      do {
        nel2 = dyson_electrons_prepared(c, mu2, st);
        mu2 += delta;
        require(++guard < 100000, GB200_ERR_MU_SEARCH, "Chemical potential search failed.");
      } while (nel2 < nel_target);
      mu1 = mu;
      nel1 = nel;
    }
    (void)nel1;
    (void)nel2;
    while (std::abs((nel - nel_target) / nel_target) > tol && std::abs(mu2 - mu1) > 0.01 * tol) {
      mu = (mu1 + mu2) * 0.5;
      nel_old = dyson_electrons_prepared(c, mu, st);
      if (std::abs((nel_old - nel_target) / nel_target) > tol && std::abs(nel - nel_old) < 0.001 * tol) {
        throw Error(GB200_ERR_MU_SEARCH, "Chemical potential search failed.");
      }
      nel = nel_old;
      if (nel > nel_target) mu2 = mu;
      else mu1 = mu;
    }
  }
  if (nel_out) *nel_out = nel;
  return mu;
}

void energy(Context& c, const cplx* G, const cplx* Sigma1, const cplx* Sigma_tau, double* e3, cudaStream_t st) {
  require(c.have_grid && c.have_H, GB200_ERR_STATE, "energy: grid and Hamiltonian must be set");
  const gb200_dims& d = c.d;
  const int64_t nsk = (int64_t)d.ns * d.nk, m2 = (int64_t)d.nso * d.nso;
  cplx* Gw = (cplx*)c.scratch.get(SL_DY_GW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  cplx* Sw = (cplx*)c.scratch.get(SL_DY_SW, (size_t)d.nw * nsk * m2 * sizeof(cplx));
  tau_to_omega(c, G, Gw, st);
  tau_to_omega(c, Sigma_tau, Sw, st);
  cplx* red = device_red(c);
  trace_product_kernel<<<d.nw, 256, 0, st>>>(Gw, Sw, true, red, nsk, d.nso, 1.0);
  GB_CHECK_LAUNCH();
  double* h2 = (double*)(red + d.nw);
  const double dm_pref = (d.ns == 2 || c.x2c()) ? -1.0 : -2.0;  // common_utils.cpp:18
  hf_energy_kernel<<<1, 256, 0, st>>>(G + (int64_t)(d.nts - 1) * nsk * m2, Sigma1, c.H.get(), dm_pref, nsk, d.nso, h2);
  GB_CHECK_LAUNCH();
  std::vector<cplx> gs(d.nw);
  double hh[2];
  GB_CUDA(cudaMemcpyAsync(gs.data(), red, d.nw * sizeof(cplx), cudaMemcpyDeviceToHost, st));
  GB_CUDA(cudaMemcpyAsync(hh, h2, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  GB_CUDA(cudaStreamSynchronize(st));
  double re = 0.0;
  for (int n = 0; n < d.nw; ++n) re += cmul(c.Ttn_beta[n], gs[n]).x;
  const double e_pref = (d.ns == 1 && !c.x2c()) ? 1.0 : 0.5;  // common_utils.cpp:37
  const double nkpw = 1.0 / d.nk;
  e3[0] = hh[1] * nkpw;               // E_1b
  e3[1] = 0.5 * hh[0] * nkpw;         // E_HF
  e3[2] = -re * e_pref * nkpw;        // E_corr (Galitskii-Migdal)
}

}  // namespace gb200
