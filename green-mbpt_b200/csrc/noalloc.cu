// Hartree-Fock Fock build that allocates no device memory.
//
// Who needs this: callers that cannot call cudaMalloc once they are running.
// Typical cases are hosts that have handed all free device memory to their own
// pool at start-up (a caching allocator that reserved the HBM, an MPI code with
// registered buffers) and hosts that must not trigger the device-wide
// synchronisation that cudaMalloc and cudaFree imply.  They own every buffer
// they pass in; this entry point's only working memory is the file-scope array
// below, which every GPU that loads the library holds until the process exits.
//
// The computation is the one of gb200_hf_fock_device (hf_cpu_kernels.cpp:25-146)
// with the exchange term taken one k at a time so that its intermediate fits the
// fixed workspace.  Only scalar input (nso = nao) is accepted.  Host code cannot
// use the array's name as a device address, so each call looks the address up
// with cudaGetSymbolAddress for the current device and context.  While the
// stream is being captured into a graph the address recorded by an earlier call
// in the same context is used instead, so the first call in a context should
// come before any stream capture.  All calls share the array and it keeps the
// contents of the last call: calls that overlap on the GPU (two streams, two
// host threads) race on it.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda.h>

#include "context.cuh"

namespace gb200 {
namespace {

// Fixed workspace: 64 MiB.
constexpr size_t NOALLOC_SCRATCH_BYTES = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Address of the workspace per (device, context).  A context that was destroyed
// (cudaDeviceReset) and recreated loads the module again, possibly at another
// address, so the cached value is refreshed on every call that is not being
// captured and is only trusted while a capture is in progress.
constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mutex;
struct AddrEntry {
  CUcontext ctx = nullptr;
  void* ptr = nullptr;
};
AddrEntry g_addr[MAX_DEVICES];

// cuCtxGetCurrent through the runtime's driver entry point, so the library has no link-time
// dependency on the driver library
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(f);
  });
  require(fn != nullptr, GB200_ERR_CUDA, "hf_fock_noalloc: cuCtxGetCurrent unavailable");
  return fn;
}

void* scratch_address(int dev, cudaStream_t st) {
  require(dev >= 0 && dev < MAX_DEVICES, GB200_ERR_INVALID, "hf_fock_noalloc: device index out of range");
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GB_CUDA(cudaStreamIsCapturing(st, &cap));
  std::lock_guard<std::mutex> lk(g_addr_mutex);
  AddrEntry& ent = g_addr[dev];
  void* p = nullptr;
  if (cap == cudaStreamCaptureStatusNone) {
    // the lookup also makes the device's context current if it was not yet
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    require(e == cudaSuccess && p != nullptr, GB200_ERR_CUDA,
            std::string("hf_fock_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
  }
  CUcontext cur = nullptr;
  require(ctx_get_current()(&cur) == CUDA_SUCCESS && cur != nullptr, GB200_ERR_CUDA,
          "hf_fock_noalloc: no current CUDA context");
  if (cap != cudaStreamCaptureStatusNone) {
    require(ent.ctx == cur && ent.ptr != nullptr, GB200_ERR_STATE,
            "hf_fock_noalloc: the first call in this context must come before stream capture");
    return ent.ptr;
  }
  ent.ctx = cur;
  ent.ptr = p;
  return p;
}

__host__ __device__ inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// dmT[k][s][a][b] = dm[s][k][b][a]
__global__ void noalloc_dm_transpose(const cplx* dm, cplx* dmT, int ns, int nk, int n) {
  const int64_t total = (int64_t)ns * nk * n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t m = e / ((int64_t)n * n);
    int r = (int)(e % ((int64_t)n * n));
    int a = r / n, b = r % n;
    int s = (int)(m / nk), k = (int)(m % nk);
    dmT[(((int64_t)k * ns + s) * n + a) * n + b] = dm[e - r + (int64_t)b * n + a];
  }
}

// offset of the diagonal pair (k,k) for the index k*ns+s
__global__ void noalloc_diag_table(int64_t* tab, int nk, int ns, int64_t pe) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nk * ns; i += gridDim.x * blockDim.x) {
    const int k = i / ns;
    tab[i] = ((int64_t)k * nk + k) * pe;
  }
}

ZOperand dense_op(const cplx* p, int64_t ld) {
  ZOperand o;
  o.ptr = p;
  o.row = lin(ld);
  o.col = lin(1);
  return o;
}

// Bytes of the workspace one call uses, with kpb = number of k' values of the
// exchange intermediate held at once (0 when the sizes are invalid).
struct NoallocPlan {
  size_t off_dmT, off_u, off_tab, off_work, work_bytes, total;
  int kpb;
};

NoallocPlan plan_noalloc(const gb200_dims& d) {
  NoallocPlan p{};
  const size_t nao2 = (size_t)d.nao * d.nao, pe = (size_t)d.NQ * nao2;
  const size_t mat = (size_t)d.ns * d.nk * nao2 * sizeof(cplx);
  p.off_dmT = 0;
  p.off_u = align256(mat);
  p.off_tab = p.off_u + align256((size_t)d.NQ * sizeof(cplx));
  p.off_work = p.off_tab + align256((size_t)d.nk * d.ns * sizeof(int64_t));
  // the work area holds the exchange intermediate of one k for kpb values of k'
  // (ns * kpb * NQ * nao^2 elements) and later the Madelung product S dm
  const size_t per_kp = (size_t)d.ns * pe * sizeof(cplx);
  const size_t need_min = std::max(align256(per_kp), align256(mat));
  p.total = p.off_work + need_min;
  if (p.total > NOALLOC_SCRATCH_BYTES) return p;
  const size_t room = NOALLOC_SCRATCH_BYTES - p.off_work;
  p.kpb = (int)std::min<size_t>((size_t)d.nk, room / per_kp);
  p.work_bytes = std::max(align256((size_t)p.kpb * per_kp), align256(mat));
  p.total = p.off_work + p.work_bytes;
  return p;
}

}  // namespace
}  // namespace gb200

using namespace gb200;

extern "C" int gb200_hf_fock_noalloc(const gb200_dims* dims, const double* V_dev, const double* dm_dev,
                                     const double* S_dev, double madelung, double* F_dev, void* stream) {
  try {
    require(dims && V_dev && dm_dev && S_dev && F_dev, GB200_ERR_INVALID, "hf_fock_noalloc: null pointer");
    const gb200_dims d = *dims;
    require(d.nk > 0 && d.nao > 0 && d.NQ > 0 && (d.ns == 1 || d.ns == 2), GB200_ERR_INVALID,
            "hf_fock_noalloc: need nk, nao, NQ > 0 and ns in {1, 2}");
    require(d.nso == 0 || d.nso == d.nao, GB200_ERR_INVALID,
            "hf_fock_noalloc: two-component input (nso = 2*nao) is not supported; only nso = nao (or 0)");
    const NoallocPlan p = plan_noalloc(d);
    if (p.kpb < 1) {
      char msg[400];
      std::snprintf(msg, sizeof msg,
                    "hf_fock_noalloc: sizes need %zu bytes of workspace, above the fixed maximum of %zu bytes "
                    "(16 * (ns*nk*nao^2 + max(ns*NQ*nao^2, ns*nk*nao^2)) bytes plus small tables must fit); "
                    "use gb200_hf_fock_device",
                    p.total, NOALLOC_SCRATCH_BYTES);
      throw Error(GB200_ERR_INVALID, msg);
    }
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char* base = static_cast<unsigned char*>(scratch_address(dev, st));

    const cplx* V = reinterpret_cast<const cplx*>(V_dev);
    const cplx* dm = reinterpret_cast<const cplx*>(dm_dev);
    const cplx* S = reinterpret_cast<const cplx*>(S_dev);
    cplx* F = reinterpret_cast<cplx*>(F_dev);
    cplx* dmT = reinterpret_cast<cplx*>(base + p.off_dmT);
    cplx* u = reinterpret_cast<cplx*>(base + p.off_u);
    int64_t* tab = reinterpret_cast<int64_t*>(base + p.off_tab);
    cplx* W = reinterpret_cast<cplx*>(base + p.off_work);

    const int nk = d.nk, ns = d.ns, NQ = d.NQ;
    const int64_t nao = d.nao, nao2 = nao * nao, pe = (int64_t)NQ * nao2;
    const double pref = (ns == 2) ? 1.0 : 0.5;  // hf_cpu_kernels.cpp:98

    // Every workspace value below is written before it is read within this
    // call (the GEMMs run with beta = 0 on workspace outputs), so the contents
    // left by an earlier call need no clearing.
    {
      unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(((int64_t)nk * ns + 255) / 256, 148));
      noalloc_diag_table<<<g, 256, 0, st>>>(tab, nk, ns, pe);
      GB_CHECK_LAUNCH();
      int64_t total = (int64_t)ns * nk * nao2;
      g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16));
      noalloc_dm_transpose<<<g, 256, 0, st>>>(dm, dmT, ns, nk, (int)nao);
      GB_CHECK_LAUNCH();
    }
    // direct term: u[Q] = (1/nk) sum V(k,k)[Q][a][b] dm[s][k][b][a]; F = sum_Q u[Q] V(k,k)[Q]
    {
      ZGemm g;
      g.M = NQ; g.N = 1; g.K = (int64_t)nk * ns * nao2;
      g.A.ptr = V; g.A.row = lin(nao2); g.A.col = twotab(nao2, 1, tab);
      g.B.ptr = dmT; g.B.row = lin(1); g.B.col = lin(0);
      g.C.ptr = u; g.C.row = lin(1); g.C.col = lin(0);
      g.alpha = cmk(1.0 / nk, 0.0);
      zgemm_fp64(g, st);
    }
    {
      ZGemm g;
      g.M = 1; g.N = nao2; g.K = NQ;
      g.nb0 = nk; g.nb2 = ns;
      g.A.ptr = u; g.A.row = lin(0); g.A.col = lin(1);
      g.B.ptr = V; g.B.row = lin(nao2); g.B.col = lin(1);
      g.B.bat.s0 = ((int64_t)nk + 1) * pe;
      g.C.ptr = F; g.C.row = lin(0); g.C.col = lin(1);
      g.C.bat.s0 = nao2; g.C.bat.s2 = (int64_t)nk * nao2;
      zgemm_fp64(g, st);
    }
    // exchange term, one k and kpb values of k' at a time
    for (int k = 0; k < nk; ++k) {
      for (int q0 = 0; q0 < nk; q0 += p.kpb) {
        const int nq = std::min(p.kpb, nk - q0);
        const cplx* Vk = V + ((int64_t)k * nk + q0) * pe;
        ZGemm y;  // W[s][k'][(Q,i)][a] = sum_b V(k,k')[(Q,i)][b] dm[s][k'][b][a]
        y.M = (int64_t)NQ * nao; y.N = nao; y.K = nao;
        y.nb1 = ns; y.nb2 = nq;
        y.A = dense_op(Vk, nao); y.A.bat.s2 = pe;
        y.B = dense_op(dm + (int64_t)q0 * nao2, nao);
        y.B.bat.s1 = (int64_t)nk * nao2; y.B.bat.s2 = nao2;
        y.C.ptr = W; y.C.row = lin(nao); y.C.col = lin(1);
        y.C.bat.s1 = (int64_t)nq * pe; y.C.bat.s2 = pe;
        zgemm_fp64(y, st);
        ZGemm x;  // F[s][k] -= (c/nk) sum_{(k',Q),a} W[s][(k',Q)][i][a] conj(V(k,k')[(k',Q)][j][a])
        x.M = nao; x.N = nao; x.K = (int64_t)nq * NQ * nao;
        x.nb2 = ns;
        x.A.ptr = W; x.A.row = lin(nao); x.A.col = two(nao, 1, nao2);
        x.A.bat.s2 = (int64_t)nq * pe;
        x.B.ptr = Vk; x.B.row = two(nao, 1, nao2); x.B.col = lin(nao); x.B.conj = true;
        x.C.ptr = F + (int64_t)k * nao2; x.C.row = lin(nao); x.C.col = lin(1);
        x.C.bat.s2 = (int64_t)nk * nao2;
        x.alpha = cmk(-pref / nk, 0.0); x.beta = cmk(1.0, 0.0);
        zgemm_fp64(x, st);
      }
    }
    // Madelung term: F -= c * madelung * S dm S, with S dm in the work area
    if (madelung != 0.0) {
      ZGemm a;
      a.M = nao; a.N = nao; a.K = nao; a.nb2 = (int64_t)ns * nk;
      a.A = dense_op(S, nao); a.A.bat.s2 = nao2;
      a.B = dense_op(dm, nao); a.B.bat.s2 = nao2;
      a.C.ptr = W; a.C.row = lin(nao); a.C.col = lin(1); a.C.bat.s2 = nao2;
      zgemm_fp64(a, st);
      ZGemm b;
      b.M = nao; b.N = nao; b.K = nao; b.nb2 = (int64_t)ns * nk;
      b.A = dense_op(W, nao); b.A.bat.s2 = nao2;
      b.B = dense_op(S, nao); b.B.bat.s2 = nao2;
      b.C.ptr = F; b.C.row = lin(nao); b.C.col = lin(1); b.C.bat.s2 = nao2;
      b.alpha = cmk(-pref * madelung, 0.0); b.beta = cmk(1.0, 0.0);
      zgemm_fp64(b, st);
    }
    set_thread_error(std::string());
    return GB200_OK;
  } catch (const Error& e) {
    set_thread_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_thread_error(e.what());
    return GB200_ERR_INVALID;
  }
}
