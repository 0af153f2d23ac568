// Split-precision complex contractions: Ozaki slicing into INT8, exact INT32
// products on the 5th-generation tensor cores (tcgen05, kind::i8), FP64
// recombination.
//
// Number format.  Every complex row of the left operand (and every complex
// column of the right one) gets a power-of-two exponent e with max|Re|,|Im| <
// 2^(e-1) over the contraction range (one bit of headroom).  Each real part is
// rounded to X = rint(a 2^(7S-e)) and cut into S balanced base-128 digits,
// a = 2^(e-7) (q_0 + q_1 2^-7 + ... + q_{S-1} 2^-7(S-1)) + r with q_s in [-64, 64]
// (split_digits.cuh).  Products of slices s and t share the weight 2^-7(s+t); all
// pairs with s + t = d accumulate into one INT32 accumulator "diagonal" d (pairs
// with s + t >= S are dropped, the usual triangular Ozaki truncation).  Rounding
// and balanced digits keep the representation error and the dropped products
// zero-mean, so they do not add up in phase along the contraction.  The host
// splits the contraction so that no diagonal can overflow INT32.
//
// Complex arithmetic.  A complex product becomes one real product through the
// embedding  [Re A  -Im A; Im A  Re A] x [Re B; Im B]: the left operand is stored
// with two interleaved real rows per complex row (2m: re,-im; 2m+1: im,re,
// interleaved along K), the right operand as (re, im) pairs along K.  Real row
// 2m of the result is Re C, row 2m+1 is Im C.
//
// Tensor-core kernel.  One CTA computes 128 real rows x BN complex columns for
// all S diagonals (S * BN <= 512 TMEM columns).  Warp 0 streams 64-byte K blocks
// of every slice plane with TMA (64-byte swizzle) through a multi-stage mbarrier
// ring, warp 1 issues the tcgen05.mma instructions from one thread, and 16
// epilogue warps read the accumulators from TMEM (tcgen05.ld) and recombine in FP64.  Every
// wait is bounded; on timeout the kernel records an error and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "split.cuh"
#include "split_digits.cuh"

namespace gb200 {

namespace {

constexpr int KBLK = 64;          // bytes of K per pipeline stage (one 64B swizzle atom)
constexpr int TILE_M = 128;       // real rows per CTA (64 complex rows)
constexpr int SMEM_BUDGET = 216 * 1024;  // TMA ring + tables, under the 227 KB opt-in
constexpr int EPI_WARPS = 16;     // four per TMEM sub-partition: enough warps in flight to hide
                                  // the TMEM, FP64 and store latencies of the recombination
constexpr int NWARPS = 2 + EPI_WARPS;  // producer, MMA, epilogue warps
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int EPI_CH = 32;                          // result columns per epilogue step
constexpr int EPI_CG = EPI_CH / (EPI_WARPS / 4);  // columns of a step per epilogue warp
static_assert(EPI_CG == 8, "epilogue column group: one tcgen05.ld of 8 columns");
constexpr long long WAIT_LIMIT = 4000000000LL;  // clock64 cycles (~2 s)

enum SplitErr { SERR_NONE = 0, SERR_TIMEOUT_PRODUCER = 1, SERR_TIMEOUT_MMA = 2, SERR_TIMEOUT_EPILOGUE = 3 };

// ----------------------------------------------------------------------------
// PTX wrappers
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive_local(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, volatile int* abort_flag) {
  long long t0 = clock64();
  while (!mbar_try_wait(bar, phase)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > WAIT_LIMIT) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(smem_dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, int32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(EPI_THREADS) : "memory"); }

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major operand, 64-byte swizzle, rows of
// 64 bytes, 8-row groups 512 bytes apart (SBO), layout version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;   // stride byte offset
  d |= (uint64_t)1 << 46;            // descriptor version
  d |= (uint64_t)4 << 61;            // SWIZZLE_64B
  return d;
}

// Instruction descriptor: S32 accumulate, signed 8-bit A and B, both K-major, M=128, N=bn.
__host__ __device__ constexpr uint32_t idesc_i8(int bn) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

// ----------------------------------------------------------------------------
// parameters
// ----------------------------------------------------------------------------
struct OperandSlices {
  int64_t nrb = 1;             // reduced batch count
  int dep[3] = {0, 0, 0};      // which batch components the operand depends on
  int64_t R = 0;               // complex rows (A: M, B: N)
  int64_t rows_pad = 0;        // real rows per plane
  int64_t kpad = 0;            // bytes per row
  int64_t e_ld = 0;            // exponents per reduced batch
  int8_t* planes = nullptr;    // [nrb][S][rows_pad][kpad]
  int32_t* expo = nullptr;     // [nrb][e_ld]
};

struct GemmParams {
  int S;
  int BN;
  int stages;
  int rows_fast;  // result rows are the unit-stride index (write-out walks rows first)
  int nbuf;       // TMEM accumulator sets (2: epilogue overlaps the next tile's MMAs)
  int tiles_m, tiles_n;
  int nkb;
  int ntiles_n;
  int64_t M, N;
  int64_t nb0, nb1, nb2;
  int depA[3], depB[3];
  int64_t rowsA_pad, rowsB_pad;
  const int32_t* eA;
  const int32_t* eB;
  int64_t eA_ld, eB_ld;
  ZResult C;
  cplx alpha, beta;
  int alpha_pow2;  // alpha is real and a power of two (possibly negative)
  int pair;        // the chunk is short enough that diagonal pairs (0,1), (2,3) fit int32 exactly
  ExpoSink sink;   // exponents of a later contraction's operand, folded from the stored results
  int* err;
  // grouped launch: the problems' entries (tile ranges in order) and the total tile count; the
  // launch-wide fields above (S, BN = the widest tile, stages, nbuf, err) size the shared ring
  const struct GroupEntry* group;
  int ngroup;
  int64_t ntiles;
};

// one problem of a grouped launch: its tensor maps, parameters and first global tile
struct alignas(64) GroupEntry {
  CUtensorMap mA, mB;
  GemmParams p;
  int64_t tile_begin;
};

// a tile of the launch: its problem's parameters and maps, and its index within the problem
struct TileRef {
  const GemmParams* p;
  const CUtensorMap* mA;
  const CUtensorMap* mB;
  int64_t t;
};

template <bool GROUPED>
__device__ __forceinline__ TileRef tile_ref(const GemmParams& p, const CUtensorMap* mA, const CUtensorMap* mB, int64_t t) {
  if constexpr (!GROUPED) {
    return TileRef{&p, mA, mB, t};
  } else {
    int lo = 0, hi = p.ngroup - 1;  // last entry with tile_begin <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (p.group[mid].tile_begin <= t) lo = mid;
      else hi = mid - 1;
    }
    const GroupEntry& e = p.group[lo];
    return TileRef{&e.p, &e.mA, &e.mB, t - e.tile_begin};
  }
}

__device__ __forceinline__ int64_t reduced_batch(const int dep[3], int64_t b0, int64_t b1, int64_t b2, int64_t n1,
                                                 int64_t n2) {
  int64_t rb = 0;
  if (dep[0]) rb = b0;
  if (dep[1]) rb = rb * n1 + b1;
  if (dep[2]) rb = rb * n2 + b2;
  return rb;
}

// ----------------------------------------------------------------------------
// slicing
// ----------------------------------------------------------------------------
struct SliceJob {
  const cplx* ptr;
  IdxMap rmap, kmap;
  BatchMap bat;
  bool conj;
  int64_t R, K, k0;            // rows, K range [k0, k0 + K)
  int64_t n0, n1, n2;          // batch sizes of the GEMM
  int dep[3];
  int embed;                   // 1: left operand (doubled rows), 0: right operand
  int S;
  int64_t rows_pad;            // real rows per plane
  int64_t rpad;                // complex rows covered (rows_pad / 2 for the left operand)
  int64_t kpad, e_ld;
  int8_t* out;
  int32_t* expo;
  bool r_fast;                 // consecutive threads walk rows (else K) when reading
  int single;                  // 1: the whole K range is one tile, exponents found in the same pass
};

constexpr int TR = 32, TK = 64, SL_NT = 256;
// shared tile columns: one spare slot after every 8 complex values, so the 8 threads that
// read consecutive groups of 8 columns of a row hit different banks
constexpr int TKP = TK + TK / 8 + 1;
__device__ __forceinline__ int tcol(int c) { return c + (c >> 3); }
constexpr int EXP_EMPTY = -(1 << 30);

__device__ __forceinline__ void enumerate_batch(const SliceJob& j, int64_t rb, int64_t& b0, int64_t& b1, int64_t& b2) {
  // inverse of reduced_batch with the components the operand does not depend on set to 0
  b0 = b1 = b2 = 0;
  int64_t r = rb;
  if (j.dep[2]) { b2 = r % j.n2; r /= j.n2; }
  if (j.dep[1]) { b1 = r % j.n1; r /= j.n1; }
  if (j.dep[0]) { b0 = r; }
}

// Row and K offsets of a tile (one IdxMap evaluation per row and per K position instead of
// one per element); callers synchronise before using them.
__device__ __forceinline__ void tile_offsets(const SliceJob& j, int64_t r0, int64_t kc, int64_t* roff, int64_t* koff) {
  const int t = threadIdx.x;
  if (t < TR) roff[t] = (r0 + t < j.R) ? j.rmap(r0 + t) : 0;
  else if (t >= 64 && t < 64 + TK) koff[t - 64] = (kc + t - 64 < j.K) ? j.kmap(j.k0 + kc + t - 64) : 0;
}

// Stage a TR x TK tile of the operand in shared memory (zero outside [0,R) x [0,K)); a thread
// issues its loads four at a time before storing them.
__device__ __forceinline__ void load_slice_tile(const SliceJob& j, const cplx* base, const int64_t* roff,
                                                const int64_t* koff, int64_t r0, int64_t kc, cplx (*tile)[TKP]) {
  constexpr int PER = TR * TK / SL_NT, BATCH = 4;
#pragma unroll
  for (int i0 = 0; i0 < PER; i0 += BATCH) {
    cplx v[BATCH];
#pragma unroll
    for (int i = 0; i < BATCH; ++i) {
      const int e = threadIdx.x + (i0 + i) * SL_NT;
      int rl, kl;
      if (j.r_fast) { rl = e % TR; kl = e / TR; } else { kl = e % TK; rl = e / TK; }
      v[i] = cmk(0.0, 0.0);
      if (r0 + rl < j.R && kc + kl < j.K) v[i] = __ldg(base + roff[rl] + koff[kl]);
    }
#pragma unroll
    for (int i = 0; i < BATCH; ++i) {
      const int e = threadIdx.x + (i0 + i) * SL_NT;
      int rl, kl;
      if (j.r_fast) { rl = e % TR; kl = e / TR; } else { kl = e % TK; rl = e / TK; }
      if (j.conj) v[i].y = -v[i].y;
      tile[rl][tcol(kl)] = v[i];
    }
  }
}

// Pass 1: per-row exponent e' = e + 1 (max |Re|,|Im| < 2^e = 2^(e'-1)) by atomicMax over K tiles.
__global__ void __launch_bounds__(SL_NT, 4) slice_expo_kernel(SliceJob j) {
  __shared__ cplx tile[TR][TKP];
  __shared__ int64_t roff[TR], koff[TK];
  const int64_t rb = blockIdx.z, r0 = (int64_t)blockIdx.x * TR, kc = (int64_t)blockIdx.y * TK;
  if (r0 >= j.R || kc >= j.K) return;
  int64_t b0, b1, b2;
  enumerate_batch(j, rb, b0, b1, b2);
  const cplx* base = j.ptr + j.bat(b0, b1, b2);
  tile_offsets(j, r0, kc, roff, koff);
  __syncthreads();
  load_slice_tile(j, base, roff, koff, r0, kc, tile);
  __syncthreads();
  // 8 threads per row, 8 columns each
  const int rl = threadIdx.x / 8, part = threadIdx.x % 8;
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < TK / 8; ++i) {
    cplx v = tile[rl][tcol(part * (TK / 8) + i)];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 4; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (part == 0 && m > 0.0 && r0 + rl < j.R) {
    int e;
    frexp(m, &e);
    atomicMax(&j.expo[rb * j.e_ld + r0 + rl], e + 1);  // |a| < 2^(e'-1): one bit of headroom
  }
}

// Ozaki digits of one real number: balanced base-128 digits of X = rint(a 2^(7S - e)), with one bit
// of headroom in the row exponent e (split_digits.cuh).

// Write the S digit planes of 8 consecutive K positions (from k) of row r with row exponent e,
// including the zero padding of rows and K.  S is a compile-time constant, so every digit shift is
// a constant and one plane's 16 bytes take four packed words (balanced_digit_word).
template <int S>
__device__ __forceinline__ void write_digits(const SliceJob& j, const cplx (&vals)[8], int64_t rb, int64_t r, int64_t k,
                                             int e) {
  if (r >= j.rpad || 2 * k >= j.kpad) return;
  // 2^(7S - e) in two exact power-of-two factors (the exponent can exceed the double range
  // for rows of tiny magnitude)
  const int ex = 7 * S - e;
  const int ex1 = max(-1000, min(1000, ex));
  const double sc1 = __longlong_as_double((long long)(ex1 + 1023) << 52);
  const double sc2 = __longlong_as_double((long long)(max(-1022, min(1023, ex - ex1)) + 1023) << 52);
  // X + bias of the rounded scaled values, (re, im) of the 8 positions in turn
  uint64_t u[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    u[2 * i] = balanced_input((vals[i].x * sc1) * sc2, S);
    u[2 * i + 1] = balanced_input((vals[i].y * sc1) * sc2, S);
  }
  const int64_t plane = j.rows_pad * j.kpad;
  int8_t* outb = j.out + rb * (int64_t)S * plane;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    uint32_t w[4];  // bytes (re, im) of positions 2h and 2h + 1
#pragma unroll
    for (int h = 0; h < 4; ++h) w[h] = balanced_digit_word(u[4 * h], u[4 * h + 1], u[4 * h + 2], u[4 * h + 3], S, s);
    int8_t* p = outb + (int64_t)s * plane;
    if (j.embed) {
      // row 2r: (re, -im) pairs; row 2r+1: (im, re) pairs
      uint32_t w0[4], w1[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        w0[h] = __byte_perm(w[h], negate_bytes(w[h]), 0x7250);
        w1[h] = __byte_perm(w[h], 0u, 0x2301);
      }
      *reinterpret_cast<uint4*>(p + (2 * r) * j.kpad + 2 * k) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
      *reinterpret_cast<uint4*>(p + (2 * r + 1) * j.kpad + 2 * k) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
    } else {
      *reinterpret_cast<uint4*>(p + r * j.kpad + 2 * k) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// Pass 2: slice planes, including the zero padding of rows and K.
template <int S>
__global__ void __launch_bounds__(SL_NT, 4) slice_write_kernel(SliceJob j) {
  __shared__ cplx tile[TR][TKP];
  __shared__ int64_t roff[TR], koff[TK];
  const int64_t rb = blockIdx.z, r0 = (int64_t)blockIdx.x * TR, kc = (int64_t)blockIdx.y * TK;
  int64_t b0, b1, b2;
  enumerate_batch(j, rb, b0, b1, b2);
  const cplx* base = j.ptr + j.bat(b0, b1, b2);
  tile_offsets(j, r0, kc, roff, koff);
  __syncthreads();
  load_slice_tile(j, base, roff, koff, r0, kc, tile);
  __syncthreads();
  const int rl = threadIdx.x / 8, grp = threadIdx.x % 8;
  const int64_t r = r0 + rl;
  const int64_t k = kc + grp * 8;  // first of 8 complex K positions
  cplx vals[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) vals[i] = tile[rl][tcol(grp * 8 + i)];
  int e = 0;
  if (j.single) {
    // the 8 lanes of a row hold all of its K range: reduce the maximum here (before any lane leaves)
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) m = fmax(m, fmax(fabs(vals[i].x), fabs(vals[i].y)));
    for (int o = 4; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (m > 0.0) {
      frexp(m, &e);
      ++e;  // one bit of headroom, as in slice_expo_kernel
    }
    if (grp == 0 && r < j.R) j.expo[rb * j.e_ld + r] = e;
  } else if (r < j.R) {
    e = j.expo[rb * j.e_ld + r];
    if (e == EXP_EMPTY) e = 0;
  }
  write_digits<S>(j, vals, rb, r, k, e);
}

// One pass for contractions of moderate length (K up to 8 tiles): a block stages RB rows over the
// whole contraction range in shared memory, reduces their exponents there and writes the slices,
// so the operand is read from HBM once.  Row layout in shared memory as in the tile kernels (one
// spare slot after every 8 complex values: the 8 threads reading consecutive groups of a row hit
// different banks).
__host__ __device__ inline int resident_ld(int kt) { return kt + kt / 8 + 1; }

inline size_t resident_smem(int rb, int kt) {
  return (size_t)rb * resident_ld(kt) * sizeof(cplx) + (size_t)(rb + kt) * sizeof(int64_t) + rb * sizeof(double);
}

template <int RB, int S>
__global__ void __launch_bounds__(SL_NT) slice_resident_kernel(SliceJob j, int kt) {
  extern __shared__ __align__(16) uint8_t sl_smem[];
  const int ld = resident_ld(kt);
  cplx* rows = reinterpret_cast<cplx*>(sl_smem);
  int64_t* roff = reinterpret_cast<int64_t*>(rows + RB * ld);
  int64_t* koff = roff + RB;
  double* rmax = reinterpret_cast<double*>(koff + kt);
  const int64_t rb = blockIdx.z, r0 = (int64_t)blockIdx.x * RB;
  int64_t b0, b1, b2;
  enumerate_batch(j, rb, b0, b1, b2);
  const cplx* base = j.ptr + j.bat(b0, b1, b2);
  for (int i = threadIdx.x; i < RB + kt; i += SL_NT) {
    if (i < RB) roff[i] = (r0 + i < j.R) ? j.rmap(r0 + i) : 0;
    else koff[i - RB] = (i - RB < j.K) ? j.kmap(j.k0 + i - RB) : 0;
  }
  __syncthreads();
  // stage the block's rows, eight loads in flight per thread
  const int n = RB * kt;
  for (int e0 = 0; e0 < n; e0 += 8 * SL_NT) {
    cplx v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int e = e0 + threadIdx.x + i * SL_NT;
      int rl, kl;
      if (j.r_fast) { rl = e % RB; kl = e / RB; } else { kl = e % kt; rl = e / kt; }
      v[i] = cmk(0.0, 0.0);
      if (e < n && r0 + rl < j.R && kl < j.K) v[i] = __ldg(base + roff[rl] + koff[kl]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int e = e0 + threadIdx.x + i * SL_NT;
      int rl, kl;
      if (j.r_fast) { rl = e % RB; kl = e / RB; } else { kl = e % kt; rl = e / kt; }
      if (j.conj) v[i].y = -v[i].y;
      if (e < n) rows[rl * ld + tcol(kl)] = v[i];
    }
  }
  __syncthreads();
  // row maxima: SL_NT / RB consecutive threads per row
  constexpr int TPR = SL_NT / RB;
  static_assert(TPR <= 32 && (32 % TPR) == 0, "threads of a row within one warp");
  {
    const int rl = threadIdx.x / TPR, part = threadIdx.x % TPR;
    double m = 0.0;
    for (int k = part; k < kt; k += TPR) {
      const cplx v = rows[rl * ld + tcol(k)];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
    for (int o = TPR / 2; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (part == 0) rmax[rl] = m;
  }
  __syncthreads();
  // digits: one thread per (row, 8 consecutive K positions)
  const int groups = kt / 8;
  for (int it = threadIdx.x; it < RB * groups; it += SL_NT) {
    const int rl = it / groups, g = it % groups;
    const int64_t r = r0 + rl;
    int e = 0;
    if (rmax[rl] > 0.0) {
      frexp(rmax[rl], &e);
      ++e;  // one bit of headroom, as in slice_expo_kernel
    }
    if (g == 0 && r < j.R) j.expo[rb * j.e_ld + r] = e;
    cplx vals[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) vals[i] = rows[rl * ld + tcol(g * 8 + i)];
    write_digits<S>(j, vals, rb, r, (int64_t)g * 8, e);
  }
}

// exponent of a row that was entirely zero -> 0 (its slices are zero)
__global__ void fix_empty_expo_kernel(int32_t* e, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (e[i] == EXP_EMPTY) e[i] = 0;
}

// ----------------------------------------------------------------------------
// recombination epilogue (shared by both cores)
// ----------------------------------------------------------------------------
// 2^e as an exact double (e within the normal range)
__device__ __forceinline__ double pow2(int e) {
  e = max(-1022, min(1023, e));
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// int32 -> double on the FP64 pipe: the double with high word 0x43380000 and low word x + 2^31
// is 1.5*2^52 + 2^31 + x exactly (IEEE-754 bit pattern), so one subtraction gives x.
__device__ __forceinline__ double int_to_double(int32_t x) {
  return __hiloint2double(0x43380000, (int)((uint32_t)x ^ 0x80000000u)) - 6755401588539392.0;
}

// Horner sum of the diagonals, sum_d q_d 128^(S-1-d), i.e. the value in units of
// 2^(ea + eb - 7(S+1)).  With |q_d| < 2^31 the first four partial sums are exact (< 2^53), so
// for S <= 5 the result is the exact sum rounded once.  The tensor-core epilogue evaluates the
// same expression, so both engines agree bit for bit.
__device__ __forceinline__ double combine_diagonals(const int32_t* q, int S) {
  double v = int_to_double(q[0]);
  for (int d = 1; d < S; ++d) v = fma(v, 128.0, int_to_double(q[d]));
  return v;
}

// the factor of a result element: 2^ea (row) times 2^(eb - 7(S+1)) (column)
__device__ __forceinline__ double result_scale(int ea, int eb, int S) { return pow2(ea) * pow2(eb - 7 * (S + 1)); }

__device__ __forceinline__ void store_at(const GemmParams& p, cplx* dst, double re, double im, int ea, int eb) {
  const double sc = result_scale(ea, eb, p.S);
  cplx v = cmul(p.alpha, cmk(re * sc, im * sc));
  if (p.beta.x != 0.0 || p.beta.y != 0.0) v = cadd(v, cmul(p.beta, *dst));
  *dst = v;
}

__device__ __forceinline__ void store_result(const GemmParams& p, int64_t b0, int64_t b1, int64_t b2, int64_t m, int64_t n,
                                             double re, double im, int ea, int eb) {
  cplx* Cb = p.C.ptr + p.C.bat(b0, b1, b2);
  store_at(p, Cb + p.C.row(m) + p.C.col(n), re, im, ea, eb);
}

// Horner sum of the S diagonals of W accumulator columns, as combine_diagonals.  With `pair`
// (host check: |q_d| bounded by the chunk length) q_d 128 + q_(d+1) is exact in int32 for the
// pairs (0,1) and (2,3), and the Horner sum over the pairs equals the one over single diagonals,
// since every partial sum below 2^53 is exact.
template <int S, int W>
__device__ __forceinline__ void combine_cols(const int32_t (&q)[S][1][W], bool pair, double (&v)[W]) {
  if constexpr (S <= 5) {
    if (pair) {
#pragma unroll
      for (int j = 0; j < W; ++j) {
        double a = int_to_double(q[0][0][j] * 128 + q[1][0][j]);
        if constexpr (S >= 4) a = fma(a, 16384.0, int_to_double(q[2][0][j] * 128 + q[3][0][j]));
        if constexpr (S == 3) a = fma(a, 128.0, int_to_double(q[2][0][j]));
        if constexpr (S == 5) a = fma(a, 128.0, int_to_double(q[4][0][j]));
        v[j] = a;
      }
      return;
    }
  }
#pragma unroll
  for (int j = 0; j < W; ++j) {
    double a = 0.0;
#pragma unroll
    for (int d = 0; d < S; ++d) a = fma(a, 128.0, int_to_double(q[d][0][j]));
    v[j] = a;
  }
}

// ----------------------------------------------------------------------------
// tcgen05 core
// ----------------------------------------------------------------------------
struct SmemLayout {
  int stage_bytes, a_plane_bytes, b_plane_bytes, stages, ring_bytes, ctile_bytes;
};

__host__ __device__ inline SmemLayout smem_layout(int S, int BN, int stages) {
  SmemLayout L;
  L.a_plane_bytes = TILE_M * KBLK;
  L.b_plane_bytes = BN * KBLK;
  L.stage_bytes = S * (L.a_plane_bytes + L.b_plane_bytes);
  L.stages = stages;
  L.ring_bytes = stages * L.stage_bytes;
  L.ctile_bytes = 0;  // the epilogue stores from registers (no staging tile)
  return L;
}

// one set of per-tile epilogue tables: row and column offsets of C, column factors, row exponents
// and the exponent-sink entries of the column groups (BN / 8 of the BN 4-byte slots at the end)
__host__ __device__ inline int table_set_bytes(int BN) {
  return ((TILE_M / 2) * 8 + BN * 16 + (TILE_M / 2 + BN) * 4 + 15) / 16 * 16;
}

// bytes after the tile ring: barriers, TMEM slot, flags, two sets of per-tile tables
__host__ __device__ inline int misc_bytes(int stages, int BN) {
  return (2 * stages + 4) * 8 + 32 + 2 * table_set_bytes(BN) + 64;
}

struct TileCoord {
  int64_t b0, b1, b2, rbA, rbB, mrow0, ncol0;
};

__device__ __forceinline__ TileCoord tile_coord(const GemmParams& p, int64_t t) {
  // tile and batch counts fit 32 bits (the host checks), so the divisions are 32-bit
  TileCoord c;
  const uint32_t per_batch = (uint32_t)p.tiles_m * (uint32_t)p.tiles_n;
  const uint32_t t32 = (uint32_t)t;
  const uint32_t bz = t32 / per_batch;
  const uint32_t rem = t32 - bz * per_batch;
  const uint32_t by = rem / (uint32_t)p.tiles_n, bx = rem - by * (uint32_t)p.tiles_n;  // N fastest: neighbours share A
  const uint32_t nb2 = (uint32_t)p.nb2, nb1 = (uint32_t)p.nb1;
  const uint32_t bq = bz / nb2;
  c.b2 = bz - bq * nb2;
  c.b1 = bq % nb1;
  c.b0 = bq / nb1;
  c.rbA = reduced_batch(p.depA, c.b0, c.b1, c.b2, p.nb1, p.nb2);
  c.rbB = reduced_batch(p.depB, c.b0, c.b1, c.b2, p.nb1, p.nb2);
  c.mrow0 = (int64_t)by * TILE_M;
  c.ncol0 = (int64_t)bx * p.BN;
  return c;
}

// Persistent tensor-core kernel: every CTA walks tiles blockIdx.x, +gridDim.x, ...
//  warp 0       TMA producer (one thread), a ring of `stages` K blocks that runs across tiles
//  warp 1       MMA issuer (one thread), `nbuf` TMEM accumulator sets of S * BN columns
//  warps 2..    epilogue (EPI_WARPS): TMEM -> registers -> FP64 recombination -> stores to C
// With nbuf = 2 the epilogue of one tile overlaps the MMAs of the next.
template <int SS, bool GROUPED, bool SINK>
__global__ void __launch_bounds__(NWARPS * 32, 1)
    split_gemm_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, GemmParams p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const SmemLayout L = smem_layout(p.S, p.BN, p.stages);
  uint8_t* tiles = smem;
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + L.ring_bytes + L.ctile_bytes);
  uint64_t* empty_bar = full_bar + L.stages;
  uint64_t* accf_bar = empty_bar + L.stages;   // [2]
  uint64_t* acce_bar = accf_bar + 2;           // [2]
  uint8_t* misc = reinterpret_cast<uint8_t*>(acce_bar + 2);
  uint32_t* tmem_base_slot = reinterpret_cast<uint32_t*>(misc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(misc + 4);
  volatile int* epi_ok = reinterpret_cast<volatile int*>(misc + 8);  // [2], per tile parity
  uint8_t* tables = misc + 32;                                          // [2] table sets
  const int tsb = table_set_bytes(p.BN);

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  constexpr int S = SS;
  const int nbuf = p.nbuf;
  const uint32_t acc_cols = (uint32_t)(S * p.BN);
  const uint32_t need = acc_cols * (uint32_t)nbuf;
  const uint32_t ncols_alloc = need <= 32 ? 32 : need <= 64 ? 64 : need <= 128 ? 128 : need <= 256 ? 256 : 512;
  const int64_t ntiles = GROUPED ? p.ntiles : (int64_t)p.tiles_m * p.tiles_n * p.nb0 * p.nb1 * p.nb2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < L.stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf_bar[b], 1);
      mbar_init(&acce_bar[b], EPI_WARPS);  // every epilogue warp releases the set it has read
    }
    *abort_flag = 0;
    epi_ok[0] = epi_ok[1] = 1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(tmem_base_slot, ncols_alloc);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_base_slot;

  int64_t issued = 0;  // producer: K blocks issued in total
  if (warp == 0) {
    if (lane == 0) {
      int64_t it = 0;
      const GemmParams* last_q = nullptr;
      for (int64_t t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        const TileRef tr = tile_ref<GROUPED>(p, &mapA, &mapB, t);
        const GemmParams& q = *tr.p;
        if constexpr (GROUPED) {
          if (tr.p != last_q) {
            // the problem's tensor maps live in global memory that the host rewrites between
            // launches: order those writes before the tensor-map reads of the loads
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tr.mA) : "memory");
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tr.mB) : "memory");
            last_q = tr.p;
          }
        }
        const TileCoord tc = tile_coord(q, tr.t);
        const int bpb = q.BN * KBLK;  // bytes of one B plane of this tile
        const uint32_t tile_stage_bytes = (uint32_t)(S * (L.a_plane_bytes + bpb));
        const int nkb = q.nkb;
        const int64_t rowsA_pad = q.rowsA_pad, rowsB_pad = q.rowsB_pad;
        for (int kb = 0; kb < nkb; ++kb, ++it) {
          const int st = (int)(it % L.stages);
          const uint32_t ph = (uint32_t)((it / L.stages) & 1);
          if (it >= L.stages && !mbar_wait(&empty_bar[st], ph ^ 1, abort_flag)) {
            atomicExch(p.err, SERR_TIMEOUT_PRODUCER);
            *abort_flag = 1;
            break;
          }
          uint8_t* sbase = tiles + (size_t)st * L.stage_bytes;
          mbar_expect_tx(&full_bar[st], tile_stage_bytes);
          for (int s = 0; s < S; ++s) {
            const int ya = (int)((tc.rbA * S + s) * rowsA_pad + tc.mrow0);
            tma_load_2d(sbase + s * L.a_plane_bytes, tr.mA, kb * KBLK, ya, &full_bar[st]);
          }
          uint8_t* bbase = sbase + S * L.a_plane_bytes;
          for (int u = 0; u < S; ++u) {
            const int yb = (int)((tc.rbB * S + u) * rowsB_pad + tc.ncol0);
            tma_load_2d(bbase + u * bpb, tr.mB, kb * KBLK, yb, &full_bar[st]);
          }
          issued = it + 1;
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int64_t it = 0, tcount = 0;
      for (int64_t t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x, ++tcount) {
        const TileRef tr = tile_ref<GROUPED>(p, &mapA, &mapB, t);
        const int tbn = tr.p->BN, nkb = tr.p->nkb;
        const uint32_t idesc = idesc_i8(tbn);
        const int buf = (int)(tcount % nbuf);
        const int64_t use = tcount / nbuf;
        if (use > 0 && !mbar_wait(&acce_bar[buf], (uint32_t)((use - 1) & 1), abort_flag)) {
          atomicExch(p.err, SERR_TIMEOUT_MMA);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem_base + (uint32_t)buf * acc_cols;
        bool ok = true;
        for (int kb = 0; kb < nkb; ++kb, ++it) {
          const int st = (int)(it % L.stages);
          const uint32_t ph = (uint32_t)((it / L.stages) & 1);
          if (!mbar_wait(&full_bar[st], ph, abort_flag)) {
            atomicExch(p.err, SERR_TIMEOUT_MMA);
            *abort_flag = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t* sbase = tiles + (size_t)st * L.stage_bytes;
          uint8_t* bbase = sbase + S * L.a_plane_bytes;
          for (int s = 0; s < S; ++s) {
            const uint64_t ad = smem_desc_sw64(smem_u32(sbase + s * L.a_plane_bytes));
            for (int u = 0; s + u < S; ++u) {
              const uint64_t bd = smem_desc_sw64(smem_u32(bbase + u * tbn * KBLK));
              const uint32_t dt = acc + (uint32_t)((s + u) * tbn);
#pragma unroll
              for (int kk = 0; kk < KBLK / 32; ++kk)
                umma_i8(dt, ad + 2 * kk, bd + 2 * kk, idesc, (kb > 0 || kk > 0 || s > 0) ? 1u : 0u);
            }
          }
          umma_commit(&empty_bar[st]);
        }
        if (!ok) break;
        umma_commit(&accf_bar[buf]);
      }
    }
  } else {
    // epilogue warps: TMEM sub-partition = warp % 4; the EPI_WARPS / 4 warps of a sub-partition
    // take consecutive EPI_CG-column groups of each step.  Lanes 2j and 2j+1 hold the real and
    // imaginary row of one complex result row; one shuffle gives each lane both parts of half of
    // its columns, which it stores straight to C.  The tables of consecutive tiles alternate
    // between two sets, so one named barrier per tile separates their writes from their reads.
    const int sp = warp % 4;
    const int grp = (warp - 2) / 4;
    const int row = sp * 32 + lane;  // real row inside the tile
    const int et = threadIdx.x - 64;  // 0..EPI_THREADS-1
    const int mloc = row / 2;
    const int r = row & 1;
    constexpr int H = EPI_CG / 2;
    int64_t tcount = 0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
      const TileRef tr = tile_ref<GROUPED>(p, &mapA, &mapB, t);
      const GemmParams& q = *tr.p;  // this tile's problem
      const TileCoord tc = tile_coord(q, tr.t);
      const int buf = (int)(tcount % nbuf);
      const int64_t use = tcount / nbuf;
      uint8_t* tb = tables + (tcount & 1) * tsb;
      int64_t* sh_rowC = reinterpret_cast<int64_t*>(tb);
      int64_t* sh_colC = sh_rowC + TILE_M / 2;
      double* sh_csc = reinterpret_cast<double*>(sh_colC + q.BN);  // column factors 2^(eb - 7(S+1))
      int32_t* sh_eA = reinterpret_cast<int32_t*>(sh_csc + q.BN);
      int32_t* sh_key = sh_eA + TILE_M / 2;  // exponent-sink entry per group of 8 columns
      // (filled while the MMAs of this tile run)
      const int ntab = TILE_M / 2 + q.BN + ((SINK && q.sink.expo) ? q.BN / EPI_CG : 0);
      for (int i = et; i < ntab; i += EPI_THREADS) {
        if (i >= TILE_M / 2 + q.BN) {
          const int64_t n = tc.ncol0 + (int64_t)(i - TILE_M / 2 - q.BN) * EPI_CG;
          const ExpoSink& sk = q.sink;
          sh_key[i - TILE_M / 2 - q.BN] = (int32_t)(sk.c0 * tc.b0 + sk.c1 * tc.b1 + sk.c2 * tc.b2 +
                                                    ((n / sk.d1) % sk.m1) * sk.s1 + (n / sk.d2) * sk.s2);
        } else if (i < TILE_M / 2) {
          const int64_t m = tc.mrow0 / 2 + i;
          sh_eA[i] = m < q.M ? q.eA[tc.rbA * q.eA_ld + m] : 0;
          sh_rowC[i] = m < q.M ? q.C.row(m) : 0;
        } else {
          const int64_t n = tc.ncol0 + (i - TILE_M / 2);
          const int eb = n < q.N ? q.eB[tc.rbB * q.eB_ld + n] : 0;
          sh_colC[i - TILE_M / 2] = n < q.N ? q.C.col(n) : 0;
          sh_csc[i - TILE_M / 2] = pow2(eb - 7 * (S + 1));
        }
      }
      if (et == 0) {
        const bool ok = mbar_wait(&accf_bar[buf], (uint32_t)(use & 1), abort_flag);
        if (!ok) {
          atomicExch(p.err, SERR_TIMEOUT_EPILOGUE);
          *abort_flag = 1;
        }
        epi_ok[tcount & 1] = ok ? 1 : 0;
      }
      // every epilogue thread reaches every named barrier, on the error path too
      epi_bar();
      if (!epi_ok[tcount & 1]) break;
      tc_fence_after();
      // a real alpha that is a power of two is folded into the row factor (exact, so the result
      // equals the validation engine's alpha * value); the store is then a plain copy
      const bool alpha_in_tile = q.alpha_pow2 != 0;
      const double rs = alpha_in_tile ? pow2(sh_eA[mloc]) * q.alpha.x : pow2(sh_eA[mloc]);
      // a warp whose 32 rows are all padding skips the accumulator reads
      const bool live = tc.mrow0 + sp * 32 < 2 * q.M;
      const uint32_t acc = tmem_base + (uint32_t)buf * acc_cols + ((uint32_t)(sp * 32) << 16);
      const int64_t mlim = q.M - tc.mrow0 / 2, nlim = q.N - tc.ncol0;
      const bool mok = mloc < mlim;
      cplx* Crow = q.C.ptr + q.C.bat(tc.b0, tc.b1, tc.b2) + sh_rowC[mloc];
      const bool has_beta = q.beta.x != 0.0 || q.beta.y != 0.0;
      for (int c0 = 0; c0 < q.BN; c0 += EPI_CH) {
        const int cw = min(EPI_CH, q.BN - c0);
        const int cc = grp * EPI_CG;
        const bool last = c0 + EPI_CH >= q.BN;
        double v[EPI_CG];
        const bool work = live && cc < cw;
        if (work) {
          // all S diagonals of the warp's 8 columns in one TMEM round trip
          int32_t dq[S][1][EPI_CG];
#pragma unroll
          for (int d = 0; d < S; ++d) tmem_ld8(acc + (uint32_t)(d * q.BN + c0 + cc), dq[d][0]);
          tmem_wait_ld();
          combine_cols<S, EPI_CG>(dq, q.pair != 0, v);
        }
        if (last) {
          // this warp's reads of the accumulator set are complete: release it to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive_local(&acce_bar[buf]);
        }
        if (work) {
#pragma unroll
          for (int j = 0; j < EPI_CG; ++j) v[j] *= rs * sh_csc[c0 + cc + j];
          // the even lane keeps columns [0, H) of the group, the odd lane [H, 2H)
          double other[H];
#pragma unroll
          for (int i = 0; i < H; ++i) other[i] = __shfl_xor_sync(0xffffffffu, r ? v[i] : v[H + i], 1);
          if (mok) {
#pragma unroll
            for (int i = 0; i < H; ++i) {
              const int col = c0 + cc + (r ? H + i : i);
              if (col < nlim) {
                cplx* d = Crow + sh_colC[col];
                cplx val = r ? cmk(other[i], v[H + i]) : cmk(v[i], other[i]);
                if (!alpha_in_tile) val = cmul(q.alpha, val);
                if (has_beta) val = cadd(val, cmul(q.beta, *d));
                *d = val;
              }
            }
          }
          if constexpr (SINK) {
            if (q.sink.expo) {
              // exponent of the largest stored |Re|, |Im| of the warp's 8 columns (one aligned group,
              // one entry), with the convention of slice_expo_kernel; the host allows sinks only
              // where the stored value is v itself (alpha a power of two folded into rs, beta = 0)
              double smax = 0.0;
              if (mok) {
#pragma unroll
                for (int j = 0; j < EPI_CG; ++j)
                  if (c0 + cc + j < nlim) smax = fmax(smax, fabs(v[j]));
              }
              int ev = INT_MIN;
              if (smax > 0.0) {
                const int biased = (int)((__double_as_longlong(smax) >> 52) & 0x7FF);
                int ex = biased - 1022;  // frexp's exponent for a normal number
                if (biased == 0) frexp(smax, &ex);
                ev = ex + 1;
              }
              ev = __reduce_max_sync(0xffffffffu, ev);
              if (lane == 0 && ev != INT_MIN) atomicMax(q.sink.expo + sh_key[(c0 + cc) / EPI_CG], ev);
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  // after an abort, let in-flight TMA loads land before the shared memory is released
  if (warp == 0 && lane == 0 && *abort_flag) {
    for (int64_t k = (issued > L.stages ? issued - L.stages : 0); k < issued; ++k) {
      long long t0 = clock64();
      while (!mbar_try_wait(&full_bar[k % L.stages], (uint32_t)((k / L.stages) & 1))) {
        if (clock64() - t0 > WAIT_LIMIT) break;
      }
    }
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, ncols_alloc);
  }
}

// ----------------------------------------------------------------------------
// CUDA-core validation core: the same diagonal INT32 sums from the same planes.
// ----------------------------------------------------------------------------
__global__ void split_gemm_ref_kernel(const int8_t* Ap, const int8_t* Bp, int64_t kpad, GemmParams p) {
  const int64_t bz = blockIdx.z;
  const int64_t b2 = bz % p.nb2, b1 = (bz / p.nb2) % p.nb1, b0 = bz / (p.nb2 * p.nb1);
  const int64_t rbA = reduced_batch(p.depA, b0, b1, b2, p.nb1, p.nb2);
  const int64_t rbB = reduced_batch(p.depB, b0, b1, b2, p.nb1, p.nb2);
  const int64_t m = (int64_t)blockIdx.y * 16 + threadIdx.y;
  const int64_t n = (int64_t)blockIdx.x * 16 + threadIdx.x;
  if (m >= p.M || n >= p.N) return;
  const int S = p.S;
  int32_t qr[8], qi[8];
  for (int d = 0; d < S; ++d) {
    int32_t accr = 0, acci = 0;
    for (int s = 0; s <= d; ++s) {
      const int t = d - s;
      const int8_t* a0 = Ap + ((rbA * S + s) * p.rowsA_pad + 2 * m) * kpad;
      const int8_t* a1 = a0 + kpad;
      const int8_t* bb = Bp + ((rbB * S + t) * p.rowsB_pad + n) * kpad;
      for (int64_t k = 0; k < kpad; ++k) {
        accr += (int32_t)a0[k] * (int32_t)bb[k];
        acci += (int32_t)a1[k] * (int32_t)bb[k];
      }
    }
    qr[d] = accr;
    qi[d] = acci;
  }
  const double re = combine_diagonals(qr, S), im = combine_diagonals(qi, S);
  store_result(p, b0, b1, b2, m, n, re, im, p.eA[rbA * p.eA_ld + m], p.eB[rbB * p.eB_ld + n]);
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  require(fn != nullptr, GB200_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  return fn;
}

CUtensorMap make_map(const int8_t* base, int64_t kpad, int64_t rows_total, int box_rows) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows_total};
  cuuint64_t strides[1] = {(cuuint64_t)kpad};
  cuuint32_t box[2] = {(cuuint32_t)KBLK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  require((reinterpret_cast<uintptr_t>(base) & 15) == 0 && kpad % 16 == 0, GB200_ERR_INVALID, "TMA alignment");
  CUresult r = get_encode()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  require(r == CUDA_SUCCESS, GB200_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return m;
}

inline int64_t rup(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

void deps_of(const ZOperand& o, int dep[3]) {
  dep[0] = (o.bat.tab0 != nullptr || o.bat.s0 != 0) ? 1 : 0;
  dep[1] = o.bat.s1 != 0 ? 1 : 0;
  dep[2] = o.bat.s2 != 0 ? 1 : 0;
}

int64_t nrb_of(const int dep[3], const ZGemm& g) {
  int64_t n = 1;
  if (dep[0]) n *= g.nb0;
  if (dep[1]) n *= g.nb1;
  if (dep[2]) n *= g.nb2;
  return n;
}

}  // namespace

struct SplitEngine {
  int core = 0;  // 0: tcgen05, 1: CUDA-core validation core
  DevArray<int8_t> planesA, planesB;
  DevArray<int32_t> expA, expB;
  DevArray<int> err;
  DevArray<GroupEntry> group;  // problems of a grouped launch (tensor maps, parameters, tile ranges)
  bool attr_set = false;
};

SplitEngine* split_engine(Context& c) {
  if (!c.split) c.split = new SplitEngine();
  c.split->core = c.split_core;
  return c.split;
}

void split_release(Context& c) {
  delete c.split;
  c.split = nullptr;
}

namespace {

__global__ void fill_int_kernel(int32_t* e, int64_t n, int32_t v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) e[i] = v;
}

// widest column tile for S diagonals in `cols` TMEM columns, a multiple of 16
int max_bn(int S, int cols) {
  int bn = (cols / S) / 16 * 16;
  return std::max(16, std::min(bn, 256));
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// the digit-writing kernels for the job's slice count (a template parameter of the kernels)
void launch_write(const SliceJob& j, dim3 g, cudaStream_t st) {
  switch (j.S) {
    case 2: slice_write_kernel<2><<<g, SL_NT, 0, st>>>(j); break;
    case 3: slice_write_kernel<3><<<g, SL_NT, 0, st>>>(j); break;
    case 4: slice_write_kernel<4><<<g, SL_NT, 0, st>>>(j); break;
    case 5: slice_write_kernel<5><<<g, SL_NT, 0, st>>>(j); break;
    case 6: slice_write_kernel<6><<<g, SL_NT, 0, st>>>(j); break;
    case 7: slice_write_kernel<7><<<g, SL_NT, 0, st>>>(j); break;
    default: slice_write_kernel<8><<<g, SL_NT, 0, st>>>(j); break;
  }
  GB_CHECK_LAUNCH();
}

template <int RB>
void launch_resident(const SliceJob& j, dim3 g, size_t sm, int kt, cudaStream_t st) {
  switch (j.S) {
    case 2: slice_resident_kernel<RB, 2><<<g, SL_NT, sm, st>>>(j, kt); break;
    case 3: slice_resident_kernel<RB, 3><<<g, SL_NT, sm, st>>>(j, kt); break;
    case 4: slice_resident_kernel<RB, 4><<<g, SL_NT, sm, st>>>(j, kt); break;
    case 5: slice_resident_kernel<RB, 5><<<g, SL_NT, sm, st>>>(j, kt); break;
    case 6: slice_resident_kernel<RB, 6><<<g, SL_NT, sm, st>>>(j, kt); break;
    case 7: slice_resident_kernel<RB, 7><<<g, SL_NT, sm, st>>>(j, kt); break;
    default: slice_resident_kernel<RB, 8><<<g, SL_NT, sm, st>>>(j, kt); break;
  }
}

// Opt-in shared memory above 48 KB for the kernels that use it (once per engine).
void set_smem_attrs(SplitEngine& se) {
  if (se.attr_set) return;
  const void* fns[] = {
#define GB_TC_ALL(G, K)                                                                    \
  (const void*)split_gemm_tc_kernel<2, G, K>, (const void*)split_gemm_tc_kernel<3, G, K>, \
      (const void*)split_gemm_tc_kernel<4, G, K>, (const void*)split_gemm_tc_kernel<5, G, K>, \
      (const void*)split_gemm_tc_kernel<6, G, K>, (const void*)split_gemm_tc_kernel<7, G, K>, \
      (const void*)split_gemm_tc_kernel<8, G, K>
      GB_TC_ALL(false, false), GB_TC_ALL(false, true), GB_TC_ALL(true, false), GB_TC_ALL(true, true),
#undef GB_TC_ALL
#define GB_RES_ALL(RB)                                                                        \
  (const void*)slice_resident_kernel<RB, 2>, (const void*)slice_resident_kernel<RB, 3>,       \
      (const void*)slice_resident_kernel<RB, 4>, (const void*)slice_resident_kernel<RB, 5>,   \
      (const void*)slice_resident_kernel<RB, 6>, (const void*)slice_resident_kernel<RB, 7>,   \
      (const void*)slice_resident_kernel<RB, 8>
      GB_RES_ALL(8), GB_RES_ALL(16)
#undef GB_RES_ALL
  };
  for (const void* f : fns) GB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  se.attr_set = true;
}

// Slice one operand (rows x K) into planes + exponents.
void run_slicer(SliceJob& j, int64_t nrb, cudaStream_t st) {
  const int64_t ne = nrb * j.e_ld;
  require(nrb < 65536, GB200_ERR_INVALID, "split: too many operand batches");
  if (j.kpad / 2 <= TK) {
    // the whole contraction range fits one tile: one pass finds the exponents and writes the slices
    j.single = 1;
    dim3 g((unsigned)((j.rpad + TR - 1) / TR), 1, (unsigned)nrb);
    launch_write(j, g, st);
    return;
  }
  j.single = 0;
  const int64_t nkt = (j.kpad / 2 + TK - 1) / TK;  // K tiles covering the padded range
  if (nkt <= 8) {
    // moderate contraction length: the block's rows stay in shared memory for both steps
    const int kt = (int)nkt * TK;
    if (nkt <= 4) {
      const size_t sm = resident_smem(16, kt);
      dim3 g((unsigned)((j.rpad + 15) / 16), 1, (unsigned)nrb);
      launch_resident<16>(j, g, sm, kt, st);
    } else {
      const size_t sm = resident_smem(8, kt);
      dim3 g((unsigned)((j.rpad + 7) / 8), 1, (unsigned)nrb);
      launch_resident<8>(j, g, sm, kt, st);
    }
    GB_CHECK_LAUNCH();
    return;
  }
  fill_int_kernel<<<blocks_for(ne), 256, 0, st>>>(j.expo, ne, EXP_EMPTY);
  GB_CHECK_LAUNCH();
  require(nrb < 65536, GB200_ERR_INVALID, "split: too many operand batches");
  dim3 g1((unsigned)((j.R + TR - 1) / TR), (unsigned)((j.K + TK - 1) / TK), (unsigned)nrb);
  require(g1.y < 65536, GB200_ERR_INVALID, "split: contraction too long for the slicer grid");
  slice_expo_kernel<<<g1, SL_NT, 0, st>>>(j);
  GB_CHECK_LAUNCH();
  dim3 g2((unsigned)((j.rpad + TR - 1) / TR), (unsigned)((j.kpad / 2 + TK - 1) / TK), (unsigned)nrb);
  launch_write(j, g2, st);
  GB_CHECK_LAUNCH();
  fix_empty_expo_kernel<<<blocks_for(ne), 256, 0, st>>>(j.expo, ne);
  GB_CHECK_LAUNCH();
}

// The digit pass alone, with the exponents already in j.expo (empty rows marked EXP_EMPTY).
void run_slicer_known_expo(SliceJob& j, int64_t nrb, cudaStream_t st) {
  require(nrb < 65536, GB200_ERR_INVALID, "split: too many operand batches");
  j.single = 0;
  dim3 g((unsigned)((j.rpad + TR - 1) / TR), (unsigned)((j.kpad / 2 + TK - 1) / TK), (unsigned)nrb);
  require(g.y < 65536, GB200_ERR_INVALID, "split: contraction too long for the slicer grid");
  launch_write(j, g, st);
  GB_CHECK_LAUNCH();
  fix_empty_expo_kernel<<<blocks_for(nrb * j.e_ld), 256, 0, st>>>(j.expo, nrb * j.e_ld);
  GB_CHECK_LAUNCH();
}

}  // namespace

namespace {

// largest K chunk for which no INT32 diagonal can overflow: S * 2K * 127^2 < 2^31
int64_t kmax_for(int S) {
  int64_t kmax = (int64_t)(2147483647.0 / (2.0 * 127.0 * 127.0 * S));
  return kmax / 32 * 32;
}

// Tile width of a problem: one TMEM accumulator set of up to 512 columns and the widest tile it
// allows, or the context's chosen width.  Measured on B200 for every launch shape of the GW
// chain, one set of the widest tile is faster than two sets of half the width (the epilogue of
// one tile overlapping the next tile's MMAs), with one MMA per slice product or with one MMA of
// width (S - s) BN per A slice plane: narrower tiles double the per-tile epilogue work (tables,
// barrier, TMEM round trips) that dominates the short contractions.
int tile_width(const Context& c, int S, int64_t N) {
  int bn = max_bn(S, 512);
  if (c.tile_bn > 0) bn = std::min(bn, std::max(16, c.tile_bn / 16 * 16));
  return std::min<int>(bn, (int)rup(N, 16));
}

struct Prepared {
  GemmParams p{};
  CUtensorMap mA{}, mB{};
  int64_t kpad = 0, ntiles = 0;
  double flops = 0.0;
};

// Slice K chunk [k0, k0 + Kc) of both operands into the engine's planes and fill the problem's
// parameters (and, for the tensor-core engine, its tensor maps).
Prepared prepare_chunk(SplitEngine& se, const ZGemm& g0, int S, int BN, int64_t k0, int64_t Kc, cudaStream_t st) {
  Prepared pr;
  set_smem_attrs(se);
  int depA[3], depB[3];
  deps_of(g0.A, depA);
  deps_of(g0.B, depB);
  const int64_t nrbA = nrb_of(depA, g0), nrbB = nrb_of(depB, g0);
  const int64_t rowsA_pad = rup(2 * g0.M, TILE_M);
  const int64_t rowsB_pad = rup(g0.N, BN);
  if (!se.err.p) {
    se.err.alloc(1);
    GB_CUDA(cudaMemsetAsync(se.err.p, 0, sizeof(int), st));
  }
  const int64_t kpad = rup(2 * Kc, KBLK);
  se.planesA.alloc((size_t)(nrbA * S * rowsA_pad * kpad));
  se.planesB.alloc((size_t)(nrbB * S * rowsB_pad * kpad));
  se.expA.alloc((size_t)(nrbA * rowsA_pad / 2));
  se.expB.alloc((size_t)(nrbB * rowsB_pad));
  {
    SliceJob j{};
    j.ptr = g0.A.ptr; j.rmap = g0.A.row; j.kmap = g0.A.col; j.bat = g0.A.bat; j.conj = g0.A.conj;
    j.R = g0.M; j.K = Kc; j.k0 = k0; j.n0 = g0.nb0; j.n1 = g0.nb1; j.n2 = g0.nb2;
    std::copy(depA, depA + 3, j.dep);
    j.embed = 1; j.S = S; j.rows_pad = rowsA_pad; j.rpad = rowsA_pad / 2; j.kpad = kpad; j.e_ld = rowsA_pad / 2;
    j.out = se.planesA.p; j.expo = se.expA.p;
    j.r_fast = std::abs(g0.A.row.s_in) < std::abs(g0.A.col.s_in);
    run_slicer(j, nrbA, st);
  }
  {
    SliceJob j{};
    // right operand sliced per column: the job's rows are the N columns, K runs along B's rows
    j.ptr = g0.B.ptr; j.rmap = g0.B.col; j.kmap = g0.B.row; j.bat = g0.B.bat; j.conj = g0.B.conj;
    j.R = g0.N; j.K = Kc; j.k0 = k0; j.n0 = g0.nb0; j.n1 = g0.nb1; j.n2 = g0.nb2;
    std::copy(depB, depB + 3, j.dep);
    j.embed = 0; j.S = S; j.rows_pad = rowsB_pad; j.rpad = rowsB_pad; j.kpad = kpad; j.e_ld = rowsB_pad;
    j.out = se.planesB.p; j.expo = se.expB.p;
    j.r_fast = std::abs(g0.B.col.s_in) < std::abs(g0.B.row.s_in);
    if (g0.B_expo) {
      // the producer of B recorded its column exponents (over the whole K range, so every chunk
      // can use them): only the digit pass runs
      require(g0.B_expo_ld >= g0.N, GB200_ERR_INVALID, "split: exponent array of B too short");
      j.expo = g0.B_expo;
      j.e_ld = g0.B_expo_ld;
      run_slicer_known_expo(j, nrbB, st);
    } else {
      run_slicer(j, nrbB, st);
    }
  }
  if (g0.sink.expo) {
    int aexp = 0;
    require(se.core == 0, GB200_ERR_INVALID, "split: exponent sinks need the tensor-core engine");
    require(k0 == 0 && Kc == g0.K, GB200_ERR_INVALID, "split: an exponent sink needs a single K chunk");
    require(g0.beta.x == 0.0 && g0.beta.y == 0.0 && g0.alpha.y == 0.0 && g0.alpha.x != 0.0 &&
                std::fabs(std::frexp(g0.alpha.x, &aexp)) == 0.5,
            GB200_ERR_INVALID, "split: an exponent sink needs beta = 0 and a real power-of-two alpha");
    require((g0.sink.s1 == 0 || g0.sink.d1 % 8 == 0) && (g0.sink.s2 == 0 || g0.sink.d2 % 8 == 0), GB200_ERR_INVALID,
            "split: sink entries must be constant over aligned groups of 8 columns");
    require(g0.sink.count < (1LL << 31), GB200_ERR_INVALID, "split: exponent sink too large");
    fill_int_kernel<<<blocks_for(g0.sink.count), 256, 0, st>>>(g0.sink.expo, g0.sink.count, EXP_EMPTY);
    GB_CHECK_LAUNCH();
  }
  GemmParams& p = pr.p;
  p.S = S; p.BN = BN; p.nkb = (int)(kpad / KBLK);
  p.M = g0.M; p.N = g0.N; p.nb0 = g0.nb0; p.nb1 = g0.nb1; p.nb2 = g0.nb2;
  std::copy(depA, depA + 3, p.depA);
  std::copy(depB, depB + 3, p.depB);
  p.rowsA_pad = rowsA_pad; p.rowsB_pad = rowsB_pad;
  p.eA = se.expA.p; p.eB = se.expB.p; p.eA_ld = rowsA_pad / 2; p.eB_ld = rowsB_pad;
  if (g0.B_expo) {
    p.eB = g0.B_expo;
    p.eB_ld = g0.B_expo_ld;
  }
  p.sink = g0.sink;
  p.C = g0.C; p.alpha = g0.alpha; p.beta = (k0 == 0) ? g0.beta : cmk(1.0, 0.0);
  p.err = se.err.p;
  {
    int aexp = 0;
    p.alpha_pow2 = (g0.alpha.y == 0.0 && g0.alpha.x != 0.0 && std::fabs(std::frexp(g0.alpha.x, &aexp)) == 0.5) ? 1 : 0;
  }
  {
    // |q_d| <= (d + 1) * 2Kc * 64^2 (d + 1 digit pairs per diagonal, balanced digits |q| <= 64):
    // pair (d, d + 1) is exact in int32 when 128 max|q_d| + max|q_(d+1)| < 2^31
    bool ok = S <= 5;
    for (int d = 0; ok && d + 1 < S && d <= 2; d += 2)
      ok = 2.0 * (double)Kc * 4096.0 * (128.0 * (d + 1) + (d + 2)) < 2147483648.0;
    p.pair = ok ? 1 : 0;
  }
  p.rows_fast = std::abs(g0.C.row.s_in) < std::abs(g0.C.col.s_in) ? 1 : 0;
  const int64_t nbatch = g0.nb0 * g0.nb1 * g0.nb2;
  require(nbatch < 65536, GB200_ERR_INVALID, "split: too many batches for one launch");
  p.tiles_m = (int)(rowsA_pad / TILE_M);
  p.tiles_n = (int)(rowsB_pad / BN);
  pr.kpad = kpad;
  pr.ntiles = (int64_t)p.tiles_m * p.tiles_n * nbatch;
  pr.flops = 8.0 * (double)g0.M * (double)g0.N * (double)Kc * (double)nbatch;
  if (se.core == 0) {
    const int64_t rowsA_total = nrbA * S * rowsA_pad;
    const int64_t rowsB_total = nrbB * S * rowsB_pad;
    require(rowsA_total < (1LL << 31) && rowsB_total < (1LL << 31), GB200_ERR_INVALID, "split: operand too large for TMA");
    pr.mA = make_map(se.planesA.p, kpad, rowsA_total, TILE_M);
    pr.mB = make_map(se.planesB.p, kpad, rowsB_total, BN);
  }
  return pr;
}

template <bool G, bool K>
void launch_tc_s(int S, unsigned grid, size_t smem, cudaStream_t st, const CUtensorMap& mA, const CUtensorMap& mB,
                 const GemmParams& p) {
  switch (S) {
    case 2: split_gemm_tc_kernel<2, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    case 3: split_gemm_tc_kernel<3, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    case 4: split_gemm_tc_kernel<4, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    case 5: split_gemm_tc_kernel<5, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    case 6: split_gemm_tc_kernel<6, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    case 7: split_gemm_tc_kernel<7, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
    default: split_gemm_tc_kernel<8, G, K><<<grid, NWARPS * 32, smem, st>>>(mA, mB, p); break;
  }
  GB_CHECK_LAUNCH();
}

// `sink`: some problem of the launch records exponents (otherwise the kernel without that code)
template <bool G>
void launch_tc(int S, bool sink, unsigned grid, size_t smem, cudaStream_t st, const CUtensorMap& mA,
               const CUtensorMap& mB, const GemmParams& p) {
  if (sink) launch_tc_s<G, true>(S, grid, smem, st, mA, mB, p);
  else launch_tc_s<G, false>(S, grid, smem, st, mA, mB, p);
}

// Launch-wide layout for tiles up to BN columns: TMA ring depth (what fits, at most 6 K blocks)
// and the dynamic shared memory.
void ring_layout(int S, int BN, GemmParams& p, size_t& smem) {
  const SmemLayout L1 = smem_layout(S, BN, 1);
  int stages = (SMEM_BUDGET - L1.ctile_bytes - 4096) / L1.stage_bytes;
  stages = std::max(1, std::min(stages, 6));
  p.stages = stages;
  p.nbuf = 1;
  const SmemLayout Ls = smem_layout(S, BN, stages);
  smem = (size_t)Ls.ring_bytes + Ls.ctile_bytes + 1024 /*alignment*/ + misc_bytes(stages, BN);
  require(smem <= 227 * 1024, GB200_ERR_INVALID, "split: shared memory budget exceeded");
}

KernelRecord* begin_record(Context& c, double flops, cudaStream_t st) {
  if (!c.stats_on) return nullptr;
  if (c.records_used == c.records.size()) {
    KernelRecord r;
    GB_CUDA(cudaEventCreate(&r.start));
    GB_CUDA(cudaEventCreate(&r.stop));
    c.records.push_back(r);
  }
  KernelRecord* rec = &c.records[c.records_used++];
  rec->alg_flops = flops;  // FP64-equivalent work: 8 real flops per complex multiply-add
  GB_CUDA(cudaEventRecord(rec->start, st));
  return rec;
}

unsigned persistent_grid(const Context& c, int64_t ntiles) {
  require(ntiles < (1LL << 31), GB200_ERR_INVALID, "split: too many tiles for one launch");
  int nsm = 148;
  GB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device));
  return (unsigned)std::min<int64_t>(ntiles, nsm);  // one CTA per SM walks the tiles
}

}  // namespace

void split_gemm(Context& c, SplitEngine& se, const ZGemm& g0, cudaStream_t st, int slices) {
  if (g0.M <= 0 || g0.N <= 0) return;
  validate(g0);
  const int S = slices > 0 ? slices : c.slices;
  require(S >= 2 && S <= 8, GB200_ERR_INVALID, "split: slices out of range");
  require(g0.K > 0, GB200_ERR_INVALID, "split: empty contraction");
  const int BN = tile_width(c, S, g0.N);
  const int64_t kmax = kmax_for(S);
  for (int64_t k0 = 0; k0 < g0.K; k0 += kmax) {
    const int64_t Kc = std::min(kmax, g0.K - k0);
    Prepared pr = prepare_chunk(se, g0, S, BN, k0, Kc, st);
    const int64_t nbatch = g0.nb0 * g0.nb1 * g0.nb2;
    if (se.core == 1) {
      dim3 grid((unsigned)((g0.N + 15) / 16), (unsigned)((g0.M + 15) / 16), (unsigned)nbatch);
      split_gemm_ref_kernel<<<grid, dim3(16, 16), 0, st>>>(se.planesA.p, se.planesB.p, pr.kpad, pr.p);
      GB_CHECK_LAUNCH();
      continue;
    }
    size_t smem = 0;
    ring_layout(S, BN, pr.p, smem);
    KernelRecord* rec = begin_record(c, pr.flops, st);
    launch_tc<false>(S, pr.p.sink.expo != nullptr, persistent_grid(c, pr.ntiles), smem, st, pr.mA, pr.mB, pr.p);
    if (rec) GB_CUDA(cudaEventRecord(rec->stop, st));
  }
}

int64_t split_max_chunk(int slices) { return kmax_for(slices); }

void split_gemm_group(const std::vector<Context*>& cs, const std::vector<ZGemm>& gs, cudaStream_t st, int slices) {
  require(cs.size() == gs.size() && !cs.empty(), GB200_ERR_INVALID, "split group: one contraction per context");
  const int S = slices;
  require(S >= 2 && S <= 8, GB200_ERR_INVALID, "split: slices out of range");
  const int64_t kmax = kmax_for(S);
  std::vector<SplitEngine*> ses;
  std::vector<int> bns;
  int64_t nch = 0;
  bool tc_engine = true;
  for (size_t i = 0; i < cs.size(); ++i) {
    for (size_t j = 0; j < i; ++j)
      require(cs[j] != cs[i], GB200_ERR_INVALID, "split group: a context appears twice (its slice buffers are shared)");
    validate(gs[i]);
    require(gs[i].K > 0 && gs[i].M > 0 && gs[i].N > 0, GB200_ERR_INVALID, "split group: empty contraction");
    ses.push_back(split_engine(*cs[i]));
    tc_engine = tc_engine && ses.back()->core == 0;
    bns.push_back(tile_width(*cs[i], S, gs[i].N));
    nch = std::max<int64_t>(nch, (gs[i].K + kmax - 1) / kmax);
  }
  if (!tc_engine) {  // the CUDA-core validation engine has no grouped form
    for (size_t i = 0; i < cs.size(); ++i) split_gemm(*cs[i], *ses[i], gs[i], st, S);
    return;
  }
  SplitEngine& se0 = *ses[0];
  // K chunk ch of every problem that has one, all in one grouped launch per chunk
  for (int64_t ch = 0; ch < nch; ++ch) {
    std::vector<GroupEntry> entries;
    int BNmax = 16;
    double flops = 0.0;
    int64_t total = 0;
    bool sink = false;
    for (size_t i = 0; i < cs.size(); ++i) {
      const int64_t k0 = ch * kmax;
      if (k0 >= gs[i].K) continue;
      Prepared pr = prepare_chunk(*ses[i], gs[i], S, bns[i], k0, std::min(kmax, gs[i].K - k0), st);
      GroupEntry e;
      e.mA = pr.mA;
      e.mB = pr.mB;
      e.p = pr.p;
      e.tile_begin = total;
      entries.push_back(e);
      total += pr.ntiles;
      BNmax = std::max(BNmax, bns[i]);
      flops += pr.flops;
      sink = sink || pr.p.sink.expo != nullptr;
    }
    GemmParams p{};
    p.S = S;
    p.BN = BNmax;
    p.err = se0.err.p;
    size_t smem = 0;
    ring_layout(S, BNmax, p, smem);
    se0.group.alloc(entries.size());
    GB_CUDA(cudaMemcpyAsync(se0.group.p, entries.data(), entries.size() * sizeof(GroupEntry), cudaMemcpyHostToDevice, st));
    p.group = se0.group.p;
    p.ngroup = (int)entries.size();
    p.ntiles = total;
    KernelRecord* rec = begin_record(*cs[0], flops, st);
    launch_tc<true>(S, sink, persistent_grid(*cs[0], total), smem, st, entries[0].mA, entries[0].mB, p);
    if (rec) GB_CUDA(cudaEventRecord(rec->stop, st));
  }
}

int split_check_error(Context& c, cudaStream_t st) {
  if (!c.split || !c.split->err.p) return 0;
  int h = 0;
  GB_CUDA(cudaMemcpyAsync(&h, c.split->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  GB_CUDA(cudaStreamSynchronize(st));
  if (h) GB_CUDA(cudaMemsetAsync(c.split->err.p, 0, sizeof(int), st));
  return h;
}

}  // namespace gb200
