// C ABI entry points (include/gb200.h).  Every call catches gb200::Error and
// other exceptions and turns them into status codes plus a message kept in
// the context (gb200_last_error); nothing throws across the C boundary.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "context.cuh"
#include "split.cuh"

using namespace gb200;

namespace gb200 {
std::atomic<long long> g_launch_count{0};
}

namespace {

thread_local std::string g_create_error;

template <typename F>
int guarded(gb200_context* ctx, F&& f) {
  Context* c = reinterpret_cast<Context*>(ctx);
  try {
    if (!c) throw Error(GB200_ERR_INVALID, "null context");
    GB_CUDA(cudaSetDevice(c->device));
    f(*c);
    c->last_error.clear();
    return GB200_OK;
  } catch (const Error& e) {
    if (c) c->last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    if (c) c->last_error = "host allocation failed";
    return GB200_ERR_OOM;
  } catch (const std::exception& e) {
    if (c) c->last_error = e.what();
    return GB200_ERR_INVALID;
  }
}

// Scatter a chunk of stored pairs (k1 >= k2, index k1(k1+1)/2 + k2) into the
// full [nk][nk] storage: (k1,k2) directly and, for k1 > k2, (k2,k1) as the
// per-Q conjugate transpose (df_integral_t.h:68,169-176).
__global__ void scatter_pairs_kernel(const cplx* half_chunk, int64_t p0, int64_t cnt, cplx* full, int nk, int NQ,
                                     int nao) {
  const int64_t m2 = (int64_t)nao * nao;
  const int64_t pe = (int64_t)NQ * m2;
  const int64_t total = cnt * pe;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t lp = e / pe;
    int64_t r = e - lp * pe;
    int64_t idx = p0 + lp;
    int64_t k1 = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (k1 * (k1 + 1) / 2 > idx) --k1;
    while ((k1 + 1) * (k1 + 2) / 2 <= idx) ++k1;
    int64_t k2 = idx - k1 * (k1 + 1) / 2;
    int64_t Q = r / m2;
    int ij = (int)(r - Q * m2);
    int i = ij / nao, j = ij % nao;
    cplx v = half_chunk[e];
    full[(k1 * nk + k2) * pe + r] = v;
    if (k1 != k2) full[(k2 * nk + k1) * pe + Q * m2 + (int64_t)j * nao + i] = cconj(v);
  }
}

// The same for an explicit list of stored pairs: pair l of the chunk goes to block slot[2l] as it
// is and, unless it is a diagonal pair (slot[2l+1] < 0), to block slot[2l+1] as the per-Q
// conjugate transpose.
__global__ void scatter_pair_slots_kernel(const cplx* chunk, int64_t cnt, const int64_t* slot, cplx* V, int NQ,
                                          int nao) {
  const int64_t m2 = (int64_t)nao * nao;
  const int64_t pe = (int64_t)NQ * m2;
  const int64_t total = cnt * pe;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t lp = e / pe;
    const int64_t r = e - lp * pe;
    const int64_t Q = r / m2;
    const int ij = (int)(r - Q * m2);
    const int i = ij / nao, j = ij % nao;
    const cplx v = chunk[e];
    V[slot[2 * lp] * pe + r] = v;
    if (slot[2 * lp + 1] >= 0) V[slot[2 * lp + 1] * pe + Q * m2 + (int64_t)j * nao + i] = cconj(v);
  }
}

void upload_integrals(Context& c, DevArray<cplx>& dst, const double* V_half, int64_t npairs, bool on_device,
                      cudaStream_t st) {
  const int nk = c.d.nk;
  const int64_t pe = c.pair_elems();
  require(npairs == (int64_t)nk * (nk + 1) / 2, GB200_ERR_INVALID, "set_integrals: npairs must be nk(nk+1)/2");
  dst.alloc((size_t)nk * nk * pe);
  const cplx* src = reinterpret_cast<const cplx*>(V_half);
  if (on_device) {
    // the half storage is already on the GPU: scatter it in place, chunk by chunk
    const int64_t chunk_pairs = std::max<int64_t>(1, std::min<int64_t>(npairs, (int64_t)(4e9 / (pe * sizeof(cplx)))));
    for (int64_t p0 = 0; p0 < npairs; p0 += chunk_pairs) {
      int64_t cnt = std::min(chunk_pairs, npairs - p0);
      scatter_pairs_kernel<<<148 * 16, 256, 0, st>>>(src + p0 * pe, p0, cnt, dst.p, nk, c.d.NQ, c.d.nao);
      GB_CHECK_LAUNCH();
    }
    GB_CUDA(cudaStreamSynchronize(st));
    return;
  }
  // stream the host half storage through a bounded staging buffer
  const int64_t chunk_pairs = std::max<int64_t>(1, std::min<int64_t>(npairs, (int64_t)(1e9 / (pe * sizeof(cplx)))));
  DevArray<cplx> stage;
  stage.alloc((size_t)chunk_pairs * pe);
  for (int64_t p0 = 0; p0 < npairs; p0 += chunk_pairs) {
    int64_t cnt = std::min(chunk_pairs, npairs - p0);
    GB_CUDA(cudaMemcpyAsync(stage.p, src + p0 * pe, (size_t)cnt * pe * sizeof(cplx), cudaMemcpyHostToDevice, st));
    scatter_pairs_kernel<<<148 * 16, 256, 0, st>>>(stage.p, p0, cnt, dst.p, nk, c.d.NQ, c.d.nao);
    GB_CHECK_LAUNCH();
    GB_CUDA(cudaStreamSynchronize(st));
  }
}

struct HostIO {
  // pinned-free staging: plain cudaMemcpy from pageable host memory
  static void h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    GB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  }
  static void d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    GB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
  }
};

}  // namespace

namespace gb200 {
// message returned by gb200_last_error(NULL) for calls that have no context
void set_thread_error(const std::string& msg) { g_create_error = msg; }
}  // namespace gb200

extern "C" {

const char* gb200_version(void) { return "gb200 0.1.0 (integral format 1.0.0)"; }

// CheckVersion (common_defs.h:191-212): accept v >= 1.0.0 on major.minor.patch.
int gb200_check_integral_version(const char* v) {
  if (!v) return GB200_ERR_INVALID;
  int a = 0, b = 0, p = 0;
  char suffix[32] = "";
  int parsed = std::sscanf(v, "%d.%d.%d%31s", &a, &b, &p, suffix);
  if (parsed < 3) return GB200_ERR_INVALID;
  const int ref[3] = {1, 0, 0};
  bool ok;
  if (a != ref[0]) ok = a > ref[0];
  else if (b != ref[1]) ok = b > ref[1];
  else if (p != ref[2]) ok = p > ref[2];
  else ok = true;
  return ok ? GB200_OK : GB200_ERR_OUTDATED_INPUT;
}

int gb200_create(const gb200_dims* dims, int device, gb200_context** out) {
  if (!dims || !out) return GB200_ERR_INVALID;
  *out = nullptr;
  const gb200_dims& d = *dims;
  if (d.nk <= 0 || d.nao <= 0 || d.NQ <= 0 || d.nts <= 0 || d.nw <= 0 || d.nw_b <= 0 || !(d.beta > 0)) {
    g_create_error = "gb200_create: non-positive dimension";
    return GB200_ERR_INVALID;
  }
  if (d.ns != 1 && d.ns != 2) { g_create_error = "gb200_create: ns must be 1 or 2"; return GB200_ERR_INVALID; }
  if (d.nso != d.nao && !(d.nso == 2 * d.nao && d.ns == 1)) {
    g_create_error = "gb200_create: nso must equal nao, or 2 nao with ns = 1 (two-component input)";
    return GB200_ERR_INVALID;
  }
  if (d.nso > 64) { g_create_error = "gb200_create: nso > 64 is not supported"; return GB200_ERR_INVALID; }
  if (d.nts % 2 != 0) { g_create_error = "Number of tau points should be even!!!"; return GB200_ERR_WRONG_GRID; }
  Context* c = nullptr;
  try {
    int ndev = 0;
    GB_CUDA(cudaGetDeviceCount(&ndev));
    require(device >= 0 && device < ndev, GB200_ERR_INVALID, "gb200_create: bad device index");
    GB_CUDA(cudaSetDevice(device));
    c = new Context();
    c->d = d;
    c->device = device;
    GB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  } catch (const Error& e) {
    g_create_error = e.what();
    delete c;
    return e.code;
  }
  *out = reinterpret_cast<gb200_context*>(c);
  return GB200_OK;
}

void gb200_destroy(gb200_context* ctx) {
  Context* c = reinterpret_cast<Context*>(ctx);
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  split_release(*c);
  for (auto& r : c->records) {
    if (r.start) cudaEventDestroy(r.start);
    if (r.stop) cudaEventDestroy(r.stop);
  }
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->qev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* gb200_last_error(const gb200_context* ctx) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  return c ? c->last_error.c_str() : g_create_error.c_str();
}

int gb200_set_kq_maps(gb200_context* ctx, const int32_t* kplus, const int32_t* kminus) {
  return guarded(ctx, [&](Context& c) {
    require(kplus && kminus, GB200_ERR_INVALID, "set_kq_maps: null pointer");
    const int nk = c.d.nk;
    c.kplus.assign(kplus, kplus + (size_t)nk * nk);
    c.kminus.assign(kminus, kminus + (size_t)nk * nk);
    for (size_t i = 0; i < c.kplus.size(); ++i)
      require(c.kplus[i] >= 0 && c.kplus[i] < nk && c.kminus[i] >= 0 && c.kminus[i] < nk, GB200_ERR_INVALID,
              "set_kq_maps: k index out of range");
    build_tables(c);
    c.have_kq = true;
  });
}

int gb200_set_grid(gb200_context* ctx, const double* Tnt_f, const double* Ttn_f, const double* Tnt_b,
                   const double* Ttn_b, const double* wsample_f) {
  return guarded(ctx, [&](Context& c) {
    require(Tnt_f && Ttn_f && Tnt_b && Ttn_b && wsample_f, GB200_ERR_INVALID, "set_grid: null pointer");
    const gb200_dims& d = c.d;
    c.Tnt_f.upload(reinterpret_cast<const cplx*>(Tnt_f), (size_t)d.nw * d.nts, c.stream);
    c.Ttn_f.upload(reinterpret_cast<const cplx*>(Ttn_f), (size_t)d.nts * d.nw, c.stream);
    c.Tnt_b.upload(reinterpret_cast<const cplx*>(Tnt_b), (size_t)d.nw_b * d.nts, c.stream);
    c.Ttn_b.upload(reinterpret_cast<const cplx*>(Ttn_b), (size_t)d.nts * d.nw_b, c.stream);
    c.wsample_f.assign(wsample_f, wsample_f + d.nw);
    const cplx* tb = reinterpret_cast<const cplx*>(Ttn_f) + (size_t)(d.nts - 1) * d.nw;
    c.Ttn_beta.assign(tb, tb + d.nw);
    const cplx* tbb = reinterpret_cast<const cplx*>(Ttn_b);
    c.Ttn_b_host.assign(tbb, tbb + (size_t)d.nts * d.nw_b);
    GB_CUDA(cudaStreamSynchronize(c.stream));
    c.have_grid = true;
  });
}

int gb200_set_integrals(gb200_context* ctx, int which, const double* V_half, int64_t npairs) {
  return guarded(ctx, [&](Context& c) {
    require(V_half != nullptr, GB200_ERR_INVALID, "set_integrals: null pointer");
    if (which == GB200_INTEGRALS_GW) {
      c.v_slot.clear();
      upload_integrals(c, c.V, V_half, npairs, false, c.stream);
      if (c.have_kq) build_tables(c);
      c.have_V = true;
    } else if (which == GB200_INTEGRALS_HF) {
      upload_integrals(c, c.Vhf, V_half, npairs, false, c.stream);
      c.have_Vhf = true;
    } else {
      throw Error(GB200_ERR_INVALID, "set_integrals: unknown integral set");
    }
  });
}

int gb200_set_precision(gb200_context* ctx, int mode, int slices) {
  return guarded(ctx, [&](Context& c) {
    require(mode == GB200_PREC_FP64 || mode == GB200_PREC_SPLIT, GB200_ERR_INVALID, "set_precision: unknown mode");
    if (mode == GB200_PREC_SPLIT)
      require(slices >= 2 && slices <= 8, GB200_ERR_INVALID, "set_precision: slices must be in [2, 8]");
    c.prec_mode = mode;
    c.slices = slices;
  });
}

int gb200_set_memory_budget(gb200_context* ctx, double bytes) {
  return guarded(ctx, [&](Context& c) {
    require(bytes >= 0.0, GB200_ERR_INVALID, "set_memory_budget: negative budget");
    c.mem_budget = bytes;
  });
}

int gb200_set_contraction_slices(gb200_context* ctx, const int* slices6) {
  return guarded(ctx, [&](Context& c) {
    for (int i = 0; i < 6; ++i) {
      const int s = slices6 ? slices6[i] : 0;
      require(s == 0 || (s >= 2 && s <= 8), GB200_ERR_INVALID, "set_contraction_slices: slices must be 0 or in [2, 8]");
      c.contraction_slices[i] = s;
    }
  });
}

int gb200_set_split_engine(gb200_context* ctx, int engine) {
  return guarded(ctx, [&](Context& c) {
    require(engine == 0 || engine == 1, GB200_ERR_INVALID, "set_split_engine: engine must be 0 or 1");
    c.split_core = engine;
  });
}

int gb200_gw_sigma(gb200_context* ctx, const double* G, double* Sigma) {
  return guarded(ctx, [&](Context& c) {
    require(G && Sigma, GB200_ERR_INVALID, "gw_sigma: null pointer");
    const size_t bytes = c.g_elems() * sizeof(cplx);
    cplx* dG = (cplx*)c.scratch.get(SL_IO_G, bytes);
    cplx* dS = (cplx*)c.scratch.get(SL_IO_S, bytes);
    HostIO::h2d(dG, G, bytes, c.stream);
    gw_sigma(c, dG, dS, c.stream);
    HostIO::d2h(Sigma, dS, bytes, c.stream);
    GB_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int gb200_gw_sigma_device(gb200_context* ctx, const double* G_dev, double* Sigma_dev, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(G_dev && Sigma_dev, GB200_ERR_INVALID, "gw_sigma_device: null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    gw_sigma(c, reinterpret_cast<const cplx*>(G_dev), reinterpret_cast<cplx*>(Sigma_dev), st);
  });
}

int gb200_gw_sigma_batch_device(gb200_context* const* ctxs, int n, const double* const* G_dev,
                                double* const* Sigma_dev, void* stream) {
  if (!ctxs || n <= 0 || !ctxs[0]) {
    set_thread_error("gw_sigma_batch_device: no contexts");
    return GB200_ERR_INVALID;
  }
  return guarded(ctxs[0], [&](Context& c0) {
    require(G_dev && Sigma_dev, GB200_ERR_INVALID, "gw_sigma_batch_device: null pointer");
    std::vector<Context*> cs;
    std::vector<const cplx*> G;
    std::vector<cplx*> Sg;
    for (int i = 0; i < n; ++i) {
      require(ctxs[i] && G_dev[i] && Sigma_dev[i], GB200_ERR_INVALID, "gw_sigma_batch_device: null pointer");
      Context* c = reinterpret_cast<Context*>(ctxs[i]);
      require(c->device == c0.device, GB200_ERR_INVALID, "gw_sigma_batch_device: contexts on different devices");
      cs.push_back(c);
      G.push_back(reinterpret_cast<const cplx*>(G_dev[i]));
      Sg.push_back(reinterpret_cast<cplx*>(Sigma_dev[i]));
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : c0.stream;
    gw_sigma_batch(cs, G, Sg, st);
  });
}

int gb200_set_tile_width(gb200_context* ctx, int bn) {
  return guarded(ctx, [&](Context& c) {
    require(bn >= 0 && bn <= 256, GB200_ERR_INVALID, "set_tile_width: 0 (widest) or a width up to 256");
    c.tile_bn = bn;
  });
}

int gb200_gw_sigma_vjp(gb200_context* ctx, const double* G, const double* Sb, double* Gb, double* Vb) {
  return guarded(ctx, [&](Context& c) {
    require(G && Sb && Gb, GB200_ERR_INVALID, "gw_sigma_vjp: null pointer");
    const size_t bytes = c.g_elems() * sizeof(cplx);
    cplx* dG = (cplx*)c.scratch.get(SL_IO_G, bytes);
    cplx* dSb = (cplx*)c.scratch.get(SL_IO_S, bytes);
    cplx* dGb = (cplx*)c.scratch.get(SL_IO_S1, bytes);
    HostIO::h2d(dG, G, bytes, c.stream);
    HostIO::h2d(dSb, Sb, bytes, c.stream);
    const int64_t nk = c.d.nk, pe = c.pair_elems();
    cplx* dVf = Vb ? (cplx*)c.scratch.get(SL_ADJ_VBF, (size_t)nk * nk * pe * sizeof(cplx)) : nullptr;
    gw_sigma_vjp(c, dG, dSb, dGb, dVf, c.stream);
    HostIO::d2h(Gb, dGb, bytes, c.stream);
    if (Vb) {
      const size_t hb = (size_t)(nk * (nk + 1) / 2) * pe * sizeof(cplx);
      cplx* dVh = (cplx*)c.scratch.get(SL_ADJ_VBH, hb);
      fold_pair_gradient(c, dVf, dVh, c.stream);
      HostIO::d2h(Vb, dVh, hb, c.stream);
    }
    GB_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int gb200_gw_sigma_vjp_device(gb200_context* ctx, const double* G_dev, const double* Sb_dev, double* Gb_dev,
                              double* Vb_dev, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(G_dev && Sb_dev && Gb_dev, GB200_ERR_INVALID, "gw_sigma_vjp_device: null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    const int64_t nk = c.d.nk, pe = c.pair_elems();
    cplx* dVf = Vb_dev ? (cplx*)c.scratch.get(SL_ADJ_VBF, (size_t)nk * nk * pe * sizeof(cplx)) : nullptr;
    gw_sigma_vjp(c, reinterpret_cast<const cplx*>(G_dev), reinterpret_cast<const cplx*>(Sb_dev),
                 reinterpret_cast<cplx*>(Gb_dev), dVf, st);
    if (Vb_dev) fold_pair_gradient(c, dVf, reinterpret_cast<cplx*>(Vb_dev), st);
  });
}

int gb200_hf_fock(gb200_context* ctx, const double* dm, const double* S, double madelung, double* F) {
  return guarded(ctx, [&](Context& c) {
    require(dm && S && F, GB200_ERR_INVALID, "hf_fock: null pointer");
    const size_t bytes = c.mat_elems() * sizeof(cplx);
    cplx* ddm = (cplx*)c.scratch.get(SL_DM, bytes);
    cplx* dS = (cplx*)c.scratch.get(SL_IO_H, bytes);
    cplx* dF = (cplx*)c.scratch.get(SL_IO_S1, bytes);
    HostIO::h2d(ddm, dm, bytes, c.stream);
    HostIO::h2d(dS, S, bytes, c.stream);
    hf_fock(c, ddm, dS, madelung, dF, c.stream);
    HostIO::d2h(F, dF, bytes, c.stream);
    GB_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int gb200_hf_fock_device(gb200_context* ctx, const double* dm_dev, const double* S_dev, double madelung,
                         double* F_dev, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(dm_dev && S_dev && F_dev, GB200_ERR_INVALID, "hf_fock_device: null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    hf_fock(c, reinterpret_cast<const cplx*>(dm_dev), reinterpret_cast<const cplx*>(S_dev), madelung,
            reinterpret_cast<cplx*>(F_dev), st);
  });
}

int gb200_dyson_set_hamiltonian(gb200_context* ctx, const double* H, const double* S) {
  return guarded(ctx, [&](Context& c) {
    require(H && S, GB200_ERR_INVALID, "dyson_set_hamiltonian: null pointer");
    c.H.upload(reinterpret_cast<const cplx*>(H), c.mat_elems(), c.stream);
    c.S.upload(reinterpret_cast<const cplx*>(S), c.mat_elems(), c.stream);
    // dyson.cpp:44-45: S_k and H_k are hermitized on input
    hermitize_batched(c.H.get(), (int64_t)c.d.ns * c.d.nk, c.d.nso, 1.0, c.stream);
    hermitize_batched(c.S.get(), (int64_t)c.d.ns * c.d.nk, c.d.nso, 1.0, c.stream);
    GB_CUDA(cudaStreamSynchronize(c.stream));
    c.have_H = true;
  });
}

static void upload_sigmas(Context& c, const double* Sigma1, const double* Sigma_tau, cplx** d1, cplx** dt) {
  const size_t b1 = c.mat_elems() * sizeof(cplx), bt = c.g_elems() * sizeof(cplx);
  *d1 = (cplx*)c.scratch.get(SL_IO_S1, b1);
  *dt = (cplx*)c.scratch.get(SL_IO_S, bt);
  HostIO::h2d(*d1, Sigma1, b1, c.stream);
  HostIO::h2d(*dt, Sigma_tau, bt, c.stream);
}

int gb200_dyson_find_mu(gb200_context* ctx, const double* Sigma1, const double* Sigma_tau, double mu0,
                        double nel_target, double tol, double* mu_out, double* nel_out) {
  return guarded(ctx, [&](Context& c) {
    require(Sigma1 && Sigma_tau && mu_out, GB200_ERR_INVALID, "find_mu: null pointer");
    require(nel_target > 0 && tol > 0, GB200_ERR_INVALID, "find_mu: nel and tol must be positive");
    cplx *d1, *dt;
    upload_sigmas(c, Sigma1, Sigma_tau, &d1, &dt);
    // selfenergy_eigenspectra (dyson.cpp:48-70) reads the self-energies as given
    dyson_prepare_X(c, d1, dt, false, c.stream);
    *mu_out = dyson_find_mu(c, mu0, nel_target, tol, nel_out, c.stream);
  });
}

int gb200_dyson_electrons(gb200_context* ctx, const double* Sigma1, const double* Sigma_tau, double mu,
                          double* nel_out) {
  return guarded(ctx, [&](Context& c) {
    require(Sigma1 && Sigma_tau && nel_out, GB200_ERR_INVALID, "dyson_electrons: null pointer");
    cplx *d1, *dt;
    upload_sigmas(c, Sigma1, Sigma_tau, &d1, &dt);
    dyson_prepare_X(c, d1, dt, false, c.stream);
    *nel_out = dyson_electrons_prepared(c, mu, c.stream);
  });
}

int gb200_dyson_compute_G(gb200_context* ctx, double* Sigma1, double* Sigma_tau, double mu, double* G) {
  return guarded(ctx, [&](Context& c) {
    require(Sigma1 && Sigma_tau && G, GB200_ERR_INVALID, "compute_G: null pointer");
    cplx *d1, *dt;
    upload_sigmas(c, Sigma1, Sigma_tau, &d1, &dt);
    cplx* dG = (cplx*)c.scratch.get(SL_IO_G, c.g_elems() * sizeof(cplx));
    dyson_compute_G(c, d1, dt, mu, dG, c.stream);
    HostIO::d2h(Sigma1, d1, c.mat_elems() * sizeof(cplx), c.stream);
    HostIO::d2h(Sigma_tau, dt, c.g_elems() * sizeof(cplx), c.stream);
    HostIO::d2h(G, dG, c.g_elems() * sizeof(cplx), c.stream);
    GB_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int gb200_energy(gb200_context* ctx, const double* G, const double* Sigma1, const double* Sigma_tau, double* e3) {
  return guarded(ctx, [&](Context& c) {
    require(G && Sigma1 && Sigma_tau && e3, GB200_ERR_INVALID, "energy: null pointer");
    cplx *d1, *dt;
    upload_sigmas(c, Sigma1, Sigma_tau, &d1, &dt);
    cplx* dG = (cplx*)c.scratch.get(SL_IO_G, c.g_elems() * sizeof(cplx));
    HostIO::h2d(dG, G, c.g_elems() * sizeof(cplx), c.stream);
    energy(c, dG, d1, dt, e3, c.stream);
  });
}

int gb200_iteration_device(gb200_context* ctx, double* G_dev, double* Sigma1_dev, double* Sigma_dev,
                           double madelung, double nel_target, double tol, double* mu_inout, double* e_out3,
                           void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(G_dev && Sigma1_dev && Sigma_dev && mu_inout, GB200_ERR_INVALID, "iteration: null pointer");
    require(!c.v_subset(), GB200_ERR_STATE,
            "iteration: the GW integrals hold a pair subset (partial self-energy): reduce across ranks and call "
            "the Dyson step separately");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    const gb200_dims& d = c.d;
    cplx* G = reinterpret_cast<cplx*>(G_dev);
    cplx* S1 = reinterpret_cast<cplx*>(Sigma1_dev);
    cplx* St = reinterpret_cast<cplx*>(Sigma_dev);
    const int64_t me = c.mat_elems();
    // dm = spin_prefactor * G(beta) (hf_solver.cpp:9-16)
    cplx* dm = (cplx*)c.scratch.get(SL_DM, me * sizeof(cplx));
    GB_CUDA(cudaMemcpyAsync(dm, G + (int64_t)(d.nts - 1) * me, me * sizeof(cplx), cudaMemcpyDeviceToDevice, st));
    scale_inplace(dm, me, (d.ns == 2 || c.x2c()) ? -1.0 : -2.0, st);
    require(c.have_H, GB200_ERR_STATE, "iteration: Hamiltonian/overlap must be set");
    hf_fock(c, dm, c.S.get(), madelung, S1, st);
    gw_sigma(c, G, St, st);
    double mu = *mu_inout;
    if (nel_target > 0) {
      dyson_prepare_X(c, S1, St, false, st);
      mu = dyson_find_mu(c, mu, nel_target, tol, nullptr, st);
    }
    dyson_compute_G(c, S1, St, mu, G, st);
    *mu_inout = mu;
    if (e_out3) energy(c, G, S1, St, e_out3, st);
    GB_CUDA(cudaStreamSynchronize(st));
  });
}

int gb200_last_timings(const gb200_context* ctx, float* out4) {
  const Context* c = reinterpret_cast<const Context*>(ctx);
  if (!c || !out4) return GB200_ERR_INVALID;
  std::memcpy(out4, c->timings, sizeof(c->timings));
  return GB200_OK;
}

int gb200_set_integrals_device(gb200_context* ctx, int which, const double* V_dev, int64_t pair_begin,
                               int64_t pair_count, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(V_dev != nullptr, GB200_ERR_INVALID, "set_integrals_device: null pointer");
    require(which == GB200_INTEGRALS_GW || which == GB200_INTEGRALS_HF, GB200_ERR_INVALID,
            "set_integrals_device: unknown integral set");
    const int nk = c.d.nk;
    const int64_t npairs = (int64_t)nk * (nk + 1) / 2;
    require(pair_begin >= 0 && pair_count > 0 && pair_begin + pair_count <= npairs, GB200_ERR_INVALID,
            "set_integrals_device: pair range outside [0, nk(nk+1)/2)");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    DevArray<cplx>& dst = which == GB200_INTEGRALS_GW ? c.V : c.Vhf;
    int64_t& done = which == GB200_INTEGRALS_GW ? c.pairs_set_gw : c.pairs_set_hf;
    const int64_t pe = c.pair_elems();
    if (pair_begin == 0) done = 0;
    if (which == GB200_INTEGRALS_GW && c.v_subset()) {
      c.v_slot.clear();  // back to the full pair set
      if (c.have_kq) build_tables(c);
    }
    dst.alloc((size_t)nk * nk * pe);
    scatter_pairs_kernel<<<148 * 16, 256, 0, st>>>(reinterpret_cast<const cplx*>(V_dev), pair_begin, pair_count, dst.p,
                                                   nk, c.d.NQ, c.d.nao);
    GB_CHECK_LAUNCH();
    GB_CUDA(cudaStreamSynchronize(st));
    done += pair_count;
    if (which == GB200_INTEGRALS_GW) {
      c.have_V = done >= npairs;
    } else {
      c.have_Vhf = done >= npairs;
    }
  });
}

int gb200_set_integrals_pairs(gb200_context* ctx, const double* V_pairs, const int64_t* pair_ids, int64_t count,
                              int on_device, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(V_pairs != nullptr && pair_ids != nullptr && count > 0, GB200_ERR_INVALID,
            "set_integrals_pairs: null pointer or empty pair list");
    const int nk = c.d.nk;
    const int64_t npairs = (int64_t)nk * (nk + 1) / 2, pe = c.pair_elems();
    std::vector<int64_t> slot_of((size_t)nk * nk, -1), slots((size_t)2 * count);
    int64_t nblk = 0;
    for (int64_t l = 0; l < count; ++l) {
      const int64_t p = pair_ids[l];
      require(p >= 0 && p < npairs && (l == 0 || p > pair_ids[l - 1]), GB200_ERR_INVALID,
              "set_integrals_pairs: pair indices must increase strictly within [0, nk(nk+1)/2)");
      int64_t k1 = (int64_t)((std::sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
      while (k1 * (k1 + 1) / 2 > p) --k1;
      while ((k1 + 1) * (k1 + 2) / 2 <= p) ++k1;
      const int64_t k2 = p - k1 * (k1 + 1) / 2;
      slots[2 * l] = slot_of[(size_t)(k1 * nk + k2)] = nblk++;
      slots[2 * l + 1] = -1;
      if (k1 != k2) slots[2 * l + 1] = slot_of[(size_t)(k2 * nk + k1)] = nblk++;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    c.V.alloc((size_t)nblk * pe);
    DevArray<int64_t> dslots;
    dslots.upload(slots.data(), slots.size(), st);
    const cplx* src = reinterpret_cast<const cplx*>(V_pairs);
    if (on_device) {
      scatter_pair_slots_kernel<<<148 * 16, 256, 0, st>>>(src, count, dslots.p, c.V.p, c.d.NQ, c.d.nao);
      GB_CHECK_LAUNCH();
    } else {
      // stream the host blocks through a bounded staging buffer
      const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(count, (int64_t)(1e9 / (pe * sizeof(cplx)))));
      DevArray<cplx> stage;
      stage.alloc((size_t)chunk * pe);
      for (int64_t l0 = 0; l0 < count; l0 += chunk) {
        const int64_t cnt = std::min(chunk, count - l0);
        GB_CUDA(cudaMemcpyAsync(stage.p, src + l0 * pe, (size_t)cnt * pe * sizeof(cplx), cudaMemcpyHostToDevice, st));
        scatter_pair_slots_kernel<<<148 * 16, 256, 0, st>>>(stage.p, cnt, dslots.p + 2 * l0, c.V.p, c.d.NQ, c.d.nao);
        GB_CHECK_LAUNCH();
        GB_CUDA(cudaStreamSynchronize(st));
      }
    }
    GB_CUDA(cudaStreamSynchronize(st));
    c.v_slot.swap(slot_of);
    c.pairs_set_gw = count;
    if (c.have_kq) build_tables(c);
    build_subset_tables(c);
    c.have_V = true;
  });
}

int gb200_set_q0_correction(gb200_context* ctx, const double* AqQ, const double* q_abs, double madelung) {
  return guarded(ctx, [&](Context& c) {
    if (!AqQ) {
      c.q0_on = false;
      return;
    }
    require(q_abs != nullptr, GB200_ERR_INVALID, "set_q0_correction: null pointer");
    const int nq = c.d.nk;
    c.AqQ.upload(reinterpret_cast<const cplx*>(AqQ), (size_t)nq * c.d.NQ, c.stream);
    c.q_abs.assign(q_abs, q_abs + nq);
    c.q0_madelung = madelung;
    GB_CUDA(cudaStreamSynchronize(c.stream));
    c.q0_on = true;
  });
}

int gb200_set_q_range(gb200_context* ctx, int q_begin, int q_end) {
  return guarded(ctx, [&](Context& c) {
    require(q_begin >= 0 && q_end <= c.d.nk && q_begin <= q_end, GB200_ERR_INVALID, "set_q_range: need 0 <= begin <= end <= nk");
    c.q_begin = q_begin;
    c.q_end = q_end;
  });
}

int gb200_dyson_solve_device(gb200_context* ctx, double* Sigma1_dev, double* Sigma_dev, double nel_target, double tol,
                             double* mu_inout, double* G_dev, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(Sigma1_dev && Sigma_dev && mu_inout && G_dev, GB200_ERR_INVALID, "dyson_solve_device: null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    cplx* S1 = reinterpret_cast<cplx*>(Sigma1_dev);
    cplx* St = reinterpret_cast<cplx*>(Sigma_dev);
    double mu = *mu_inout;
    if (nel_target > 0) {
      dyson_prepare_X(c, S1, St, false, st);
      mu = dyson_find_mu(c, mu, nel_target, tol, nullptr, st);
    }
    dyson_compute_G(c, S1, St, mu, reinterpret_cast<cplx*>(G_dev), st);
    GB_CUDA(cudaStreamSynchronize(st));
    *mu_inout = mu;
  });
}

int gb200_energy_device(gb200_context* ctx, const double* G_dev, const double* Sigma1_dev, const double* Sigma_dev,
                        double* e_out3, void* stream) {
  return guarded(ctx, [&](Context& c) {
    require(G_dev && Sigma1_dev && Sigma_dev && e_out3, GB200_ERR_INVALID, "energy_device: null pointer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c.stream;
    energy(c, reinterpret_cast<const cplx*>(G_dev), reinterpret_cast<const cplx*>(Sigma1_dev),
           reinterpret_cast<const cplx*>(Sigma_dev), e_out3, st);
  });
}

int gb200_stats_enable(gb200_context* ctx, int on) {
  return guarded(ctx, [&](Context& c) {
    c.stats_on = on != 0;
    c.records_used = 0;
  });
}

int gb200_stats_read(gb200_context* ctx, long long* launches_total, long long* tc_launches, double* tc_ms,
                     double* tc_alg_flops) {
  return guarded(ctx, [&](Context& c) {
    double ms = 0.0, fl = 0.0;
    for (size_t i = 0; i < c.records_used; ++i) {
      GB_CUDA(cudaEventSynchronize(c.records[i].stop));
      float t = 0.f;
      GB_CUDA(cudaEventElapsedTime(&t, c.records[i].start, c.records[i].stop));
      ms += t;
      fl += c.records[i].alg_flops;
    }
    if (launches_total) *launches_total = g_launch_count.load();
    if (tc_launches) *tc_launches = (long long)c.records_used;
    if (tc_ms) *tc_ms = ms;
    if (tc_alg_flops) *tc_alg_flops = fl;
  });
}

}  // extern "C"
