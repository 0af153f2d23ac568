// Shared definitions of the gb200 engine: complex helpers, error handling,
// the GEMM descriptor and the context object behind the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cuComplex.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gb200.h"

namespace gb200 {

using cplx = double2;

__host__ __device__ __forceinline__ cplx cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Error carrying a C-ABI status code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define GB_CUDA(call)                                                                                \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) {                                                                         \
      throw ::gb200::Error(e_ == cudaErrorMemoryAllocation ? GB200_ERR_OOM : GB200_ERR_CUDA,         \
                           std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    }                                                                                                \
  } while (0)

// Every kernel launch of the library goes through this check, which also counts it
// (gb200_kernel_stats reports the count).
extern std::atomic<long long> g_launch_count;
#define GB_CHECK_LAUNCH()                                \
  do {                                                   \
    ::gb200::g_launch_count.fetch_add(1, std::memory_order_relaxed); \
    GB_CUDA(cudaGetLastError());                         \
  } while (0)

inline void require(bool cond, int code, const std::string& msg) {
  if (!cond) throw Error(code, msg);
}

// ---------------------------------------------------------------------------
// Index maps of a batched complex GEMM operand.
//
// A logical index i (a row, a column, a K position) maps to a memory offset
//   off(i) = outer(i / n_in) + (i % n_in) * s_in,
//   outer(o) = tab ? tab[o] : o * s_out.
// n_in == 0 means a one-level map off(i) = i * s_in.  This covers every
// operand view of the GW contractions (transposes, (Q,p) row groups, the
// per-k pair offsets of the k +- q maps) without copies.
// ---------------------------------------------------------------------------
struct IdxMap {
  int64_t n_in = 0;
  int64_t s_in = 1;
  int64_t s_out = 0;
  const int64_t* tab = nullptr;  // device array of outer offsets (or nullptr)

  __host__ __device__ __forceinline__ int64_t operator()(int64_t i) const {
    if (n_in == 0) return i * s_in;
    int64_t o, r;
    if (((uint64_t)i | (uint64_t)n_in) < 0x80000000ull) {
      // 32-bit division: several times cheaper than the 64-bit one on the GPU
      const uint32_t q = (uint32_t)i / (uint32_t)n_in;
      o = q;
      r = (int64_t)((uint32_t)i - q * (uint32_t)n_in);
    } else {
      o = i / n_in;
      r = i - o * n_in;
    }
    return (tab ? tab[o] : o * s_out) + r * s_in;
  }
};

inline IdxMap lin(int64_t s) { IdxMap m; m.n_in = 0; m.s_in = s; return m; }
inline IdxMap two(int64_t n_in, int64_t s_in, int64_t s_out) { IdxMap m; m.n_in = n_in; m.s_in = s_in; m.s_out = s_out; return m; }
inline IdxMap twotab(int64_t n_in, int64_t s_in, const int64_t* tab) { IdxMap m; m.n_in = n_in; m.s_in = s_in; m.tab = tab; return m; }

// Batch index b in [0, n0*n1*n2) split as (b0, b1, b2), b2 fastest.
struct BatchMap {
  int64_t s0 = 0, s1 = 0, s2 = 0;
  const int64_t* tab0 = nullptr;  // optional table for the b0 component
  __host__ __device__ __forceinline__ int64_t operator()(int64_t b0, int64_t b1, int64_t b2) const {
    return (tab0 ? tab0[b0] : b0 * s0) + b1 * s1 + b2 * s2;
  }
};

struct ZOperand {
  const cplx* ptr = nullptr;
  IdxMap row, col;     // element (r, c) at ptr[batch + row(r) + col(c)]
  BatchMap bat;
  bool conj = false;
};

struct ZResult {
  cplx* ptr = nullptr;
  IdxMap row, col;
  BatchMap bat;
};

// Split precision: per-row exponents of a later contraction's operand, recorded by the
// contraction that produces that operand.  A result element in column n of batch (b0, b1, b2)
// belongs to entry  c0 b0 + c1 b1 + c2 b2 + ((n / d1) % m1) s1 + (n / d2) s2  of `expo`; every
// result row folds into the same entry.  Aligned groups of 8 columns must share an entry (d1 and
// d2 multiples of 8 where their term is used).
struct ExpoSink {
  int32_t* expo = nullptr;  // nullptr: no sink
  int64_t c0 = 0, c1 = 0, c2 = 0;
  int64_t d1 = 1, m1 = 1, s1 = 0;
  int64_t d2 = 1, s2 = 0;
  int64_t count = 0;  // entries of `expo`
};

// C = alpha * op(A) op(B) + beta * C over a 3-level batch.
struct ZGemm {
  int64_t M = 0, N = 0, K = 0;
  int64_t nb0 = 1, nb1 = 1, nb2 = 1;
  ZOperand A, B;  // A: M x K, B: K x N
  ZResult C;      // M x N
  cplx alpha = {1.0, 0.0};
  cplx beta = {0.0, 0.0};
  // split precision only: `sink` records the exponents of a later contraction's operand from this
  // result (a single K chunk, beta = 0, alpha a real power of two); `B_expo` holds operand B's
  // column exponents, written by such a sink, B_expo_ld apart per reduced batch of B
  ExpoSink sink;
  int32_t* B_expo = nullptr;
  int64_t B_expo_ld = 0;
};

void zgemm_fp64(const ZGemm& g, cudaStream_t st);
void validate(const ZGemm& g);
void set_thread_error(const std::string& msg);

}  // namespace gb200
