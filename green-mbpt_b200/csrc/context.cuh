// The context behind the C ABI: dimensions, resident device inputs, the
// scratch arena and the per-q offset tables of the k +- q maps.
#pragma once

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace gb200 {

// Owning device allocation.
template <typename T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  ~DevArray() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) return;
    GB_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T* host, size_t count, cudaStream_t st) {
    alloc(count);
    GB_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  T* get() const { return p; }
};

// Named scratch buffers that only grow.
struct Scratch {
  std::vector<std::unique_ptr<DevArray<char>>> bufs;
  void* get(int slot, size_t bytes) {
    if ((int)bufs.size() <= slot) bufs.resize(slot + 1);
    if (!bufs[slot]) bufs[slot].reset(new DevArray<char>());
    bufs[slot]->alloc(bytes);
    return bufs[slot]->p;
  }
  void release() { bufs.clear(); }
};

enum ScratchSlot {
  SL_T1 = 0, SL_BT, SL_P0, SL_PW, SL_AUG, SL_TMP, SL_Y1, SL_Y2,
  SL_HF_Y, SL_HF_U, SL_HF_DMT, SL_DY_SW, SL_DY_GW, SL_DY_X, SL_RED, SL_IO_G, SL_IO_S,
  SL_IO_S1, SL_IO_H, SL_DM, SL_PINV, SL_SPLIT0, SL_HF_TAB, SL_X2C_DM, SL_X2C_S, SL_X2C_F, SL_X2C_GAB, SL_X2C_GBA,
  SL_X2C_SIG, SL_Q0_Y, SL_Q0_T, SL_Q0_D, SL_Q0_E, SL_Q0_S, SL_ADJ_TH, SL_ADJ_PTW, SL_ADJ_W, SL_ADJ_WB,
  SL_ADJ_PTWB, SL_ADJ_PWB, SL_ADJ_THB, SL_ADJ_XB, SL_ADJ_AB, SL_ADJ_P0B, SL_ADJ_P0HB, SL_ADJ_X3, SL_ADJ_TAB, SL_ADJ_TQ, SL_ADJ_VBF, SL_ADJ_VBH,
  SL_SINK, SL_COUNT
};

struct SplitEngine;

// One timed launch of the tensor-core contraction kernel (CUDA events on its stream)
// with the FP64-equivalent complex flops of the contraction it performed.
struct KernelRecord {
  cudaEvent_t start = nullptr, stop = nullptr;
  double alg_flops = 0.0;
};

struct Context {
  gb200_dims d{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  int prec_mode = GB200_PREC_FP64;
  int slices = 4;
  // slices of the P0 contractions (a)-(c) and the Sigma contractions (d)-(f); 0 takes `slices`
  int contraction_slices[6] = {0, 0, 0, 0, 0, 0};
  // bytes the blocked intermediates of one call may take (GW: the two k-block buffers; HF: the
  // exchange intermediates); 0 takes a default share of the free device memory
  double mem_budget = 0.0;
  double budget_or(double cap, double free_share) const {
    if (mem_budget > 0.0) return mem_budget;
    size_t free_b = 0, total_b = 0;
    GB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    return std::min(cap, free_share * (double)free_b);
  }
  int split_core = 0;             // 0: tcgen05 tensor cores, 1: CUDA-core validation core
  int tile_bn = 0;                // column tile of the split contractions (0: the widest that fits)
  SplitEngine* split = nullptr;

  bool have_kq = false, have_grid = false, have_V = false, have_Vhf = false, have_H = false;
  std::vector<int32_t> kplus, kminus;  // [nk * nk]

  // transforms
  DevArray<cplx> Tnt_f, Ttn_f, Tnt_b, Ttn_b;
  std::vector<double> wsample_f;
  std::vector<cplx> Ttn_beta;  // host copy of the tau = beta row of Ttn_f
  std::vector<cplx> Ttn_b_host;  // host copy of Ttn_b [nts][nw_b]
  // q -> 0 correction ("extrapolate" treatment, mbpt_q0_utils_t): AqQ [nk][NQ] on the device,
  // |q| on the host, the Madelung constant; eps_inv [nw_b][nk] collects the heads of P(i Omega, q)
  bool q0_on = false;
  DevArray<cplx> AqQ, eps_inv;
  std::vector<double> q_abs;
  double q0_madelung = 0.0;

  // integrals, all ordered pairs [nk][nk][NQ][nao][nao]; the GW set may instead hold a subset
  // (q-sharded storage): then v_slot[k1 * nk + k2] is the block of (k1, k2) in V, -1 where this
  // context does not hold it
  DevArray<cplx> V, Vhf;
  std::vector<int64_t> v_slot;
  // Dyson inputs [ns][nk][nso][nso]
  DevArray<cplx> H, S;

  // per-q offset tables (device): [nq][nk] or [nq][nk*ns]
  DevArray<int64_t> tab_pair_plus, tab_pair_minus, tab_g_plus, tab_g_minus, tab_pair_plus_ns;
  DevArray<int64_t> tab_v_diag;  // pair subset: offset of block (k, k) in V per k (0 where not held)

  Scratch scratch;
  float timings[4] = {0, 0, 0, 0};
  // q-points handled by this context: [q_begin, q_end) (a shard of the q loop; default all)
  int q_begin = 0, q_end = -1;
  // stored pairs delivered so far by the chunked device upload
  int64_t pairs_set_gw = 0, pairs_set_hf = 0;
  // statistics of the tensor-core contraction kernel (off unless requested)
  bool stats_on = false;
  std::vector<KernelRecord> records;
  size_t records_used = 0;
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  // stage boundaries of the GW q loop (4 per q-point), read once after the loop
  std::vector<cudaEvent_t> qev;

  bool v_subset() const { return !v_slot.empty(); }
  // block index of the ordered pair (k1, k2) in V, -1 if it is not held
  int64_t v_block(int k1, int k2) const {
    const int64_t i = (int64_t)k1 * d.nk + k2;
    return v_slot.empty() ? i : v_slot[(size_t)i];
  }
  int64_t nao() const { return d.nao; }
  int64_t pair_elems() const { return (int64_t)d.NQ * d.nao * d.nao; }
  // two-component (X2C) input: nso = 2 nao, the GW contractions run over the 4 spin blocks
  bool x2c() const { return d.nso == 2 * d.nao; }
  int ns_eff() const { return x2c() ? 4 : d.ns; }
  int64_t g_elems() const { return (int64_t)d.nts * d.ns * d.nk * d.nso * d.nso; }
  int64_t mat_elems() const { return (int64_t)d.ns * d.nk * d.nso * d.nso; }
};

// stages implemented in the .cu files
void build_tables(Context& c);
void build_subset_tables(Context& c);
// GB200_ERR_STATE unless V holds every pair the q-points [q0, q1) read: (k, k+q) and (k, k-q)
void require_q_pairs(const Context& c, int q0, int q1);
void gw_sigma(Context& c, const cplx* G, cplx* Sigma, cudaStream_t st);
// the self-energies of several contexts together: their q-points in step (round i takes the i-th
// q-point of every context that has one, k-blocks in step), each contraction stage of the round
// in one grouped tensor-core launch when every context runs it in split precision
void gw_sigma_batch(const std::vector<Context*>& cs, const std::vector<const cplx*>& G, const std::vector<cplx*>& Sigma,
                    cudaStream_t st);
// Gb = d/dG of Re sum conj(Sb) Sigma(G, V) (FP64; no two-component input, no q -> 0 correction);
// with Vb non-null also d/dV on the full pair set [nk][nk][NQ][nao][nao] (zeroed here)
void gw_sigma_vjp(Context& c, const cplx* G, const cplx* Sb, cplx* Gb, cplx* Vb, cudaStream_t st);
// gradient of the half-stored integrals [nk(nk+1)/2][NQ][nao][nao] from the one of the full pair set
void fold_pair_gradient(Context& c, const cplx* full, cplx* half, cudaStream_t st);
// q -> 0 limit of the collected heads eps_inv[nw_b][nq] (mbpt_q0_utils_t.cpp:30-86), on the host
cplx extrapolate_q0(const cplx* eps_n, const std::vector<double>& q_abs, int fit_order, double q_max);
void hf_fock(Context& c, const cplx* dm, const cplx* S, double madelung, cplx* F, cudaStream_t st);
void dyson_compute_G(Context& c, cplx* Sigma1, cplx* Sigma_tau, double mu, cplx* G, cudaStream_t st);
void dyson_prepare_X(Context& c, cplx* Sigma1, cplx* Sigma_tau, bool hermitize, cudaStream_t st);
double dyson_electrons_prepared(Context& c, double mu, cudaStream_t st);
double dyson_find_mu(Context& c, double mu0, double nel_target, double tol, double* nel_out, cudaStream_t st);
void energy(Context& c, const cplx* G, const cplx* Sigma1, const cplx* Sigma_tau, double* e3, cudaStream_t st);

// linear algebra helpers (linalg.cu)
void hermitize_batched(cplx* X, int64_t nmat, int n, double scale, cudaStream_t st);
void invert_small_batched(const cplx* A, cplx* Ainv, int64_t nmat, int n, cudaStream_t st);
void invert_large_batched(const cplx* A, cplx* Ainv, cplx* aug, int64_t nmat, int n, bool herm_from_lower,
                          bool identity_minus, cudaStream_t st);
void scale_inplace(cplx* X, int64_t count, double s, cudaStream_t st);

}  // namespace gb200
