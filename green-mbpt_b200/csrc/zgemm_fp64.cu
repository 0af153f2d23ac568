// FP64 batched complex GEMM over general index maps (the parity path).
//
// One CTA computes a 64 x 64 complex tile with 256 threads, each holding a
// 4 x 4 complex accumulator (rows ty + 16 i, cols tx + 16 j).  Operand tiles
// of depth 16 are staged through shared memory; the load pattern follows the
// operand's fastest-varying index so global reads coalesce for row- and
// column-major views alike.  Offsets of the tile's rows / columns are decoded
// once per CTA from the IdxMap, the K offsets once per K step.
#include "common.cuh"

namespace gb200 {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

struct LoadMode {
  bool a_kfast;  // consecutive threads walk K for A (else walk M)
  bool b_kfast;  // consecutive threads walk K for B (else walk N)
};

__global__ void __launch_bounds__(NT) zgemm_fp64_kernel(ZGemm g, LoadMode lm, int64_t nbatch) {
  __shared__ cplx As[BK][BM + 1];
  __shared__ cplx Bs[BK][BN + 1];
  __shared__ int64_t rowA[BM], colB[BN], rowC[BM], colC[BN];
  __shared__ int64_t kA[BK], kB[BK];

  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  const int64_t m0 = (int64_t)blockIdx.y * BM;
  const int64_t n0 = (int64_t)blockIdx.x * BN;

  if (tid < BM) {
    int64_t r = m0 + tid;
    rowA[tid] = r < g.M ? g.A.row(r) : 0;
    rowC[tid] = r < g.M ? g.C.row(r) : 0;
  } else if (tid < BM + BN) {
    int64_t c = n0 + (tid - BM);
    colB[tid - BM] = c < g.N ? g.B.col(c) : 0;
    colC[tid - BM] = c < g.N ? g.C.col(c) : 0;
  }

  for (int64_t b = blockIdx.z; b < nbatch; b += gridDim.z) {
    const int64_t b2 = b % g.nb2;
    const int64_t b1 = (b / g.nb2) % g.nb1;
    const int64_t b0 = b / (g.nb2 * g.nb1);
    const cplx* Ab = g.A.ptr + g.A.bat(b0, b1, b2);
    const cplx* Bb = g.B.ptr + g.B.bat(b0, b1, b2);
    cplx* Cb = g.C.ptr + g.C.bat(b0, b1, b2);

    cplx acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = cmk(0.0, 0.0);

    for (int64_t k0 = 0; k0 < g.K; k0 += BK) {
      __syncthreads();
      if (tid < BK) {
        int64_t k = k0 + tid;
        kA[tid] = k < g.K ? g.A.col(k) : 0;
      } else if (tid < 2 * BK) {
        int64_t k = k0 + tid - BK;
        kB[tid - BK] = k < g.K ? g.B.row(k) : 0;
      }
      __syncthreads();
      // A tile: BM x BK
#pragma unroll
      for (int i = 0; i < (BM * BK) / NT; ++i) {
        int e = tid + i * NT;
        int r, kk;
        if (lm.a_kfast) { kk = e % BK; r = e / BK; } else { r = e % BM; kk = e / BM; }
        cplx v = cmk(0.0, 0.0);
        if (m0 + r < g.M && k0 + kk < g.K) {
          v = Ab[rowA[r] + kA[kk]];
          if (g.A.conj) v.y = -v.y;
        }
        As[kk][r] = v;
      }
      // B tile: BK x BN
#pragma unroll
      for (int i = 0; i < (BN * BK) / NT; ++i) {
        int e = tid + i * NT;
        int c, kk;
        if (lm.b_kfast) { kk = e % BK; c = e / BK; } else { c = e % BN; kk = e / BN; }
        cplx v = cmk(0.0, 0.0);
        if (n0 + c < g.N && k0 + kk < g.K) {
          v = Bb[kB[kk] + colB[c]];
          if (g.B.conj) v.y = -v.y;
        }
        Bs[kk][c] = v;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        cplx a[4], bb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            acc[i][j].x = fma(a[i].x, bb[j].x, acc[i][j].x);
            acc[i][j].x = fma(-a[i].y, bb[j].y, acc[i][j].x);
            acc[i][j].y = fma(a[i].x, bb[j].y, acc[i][j].y);
            acc[i][j].y = fma(a[i].y, bb[j].x, acc[i][j].y);
          }
      }
    }
    const bool has_beta = (g.beta.x != 0.0 || g.beta.y != 0.0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int r = ty + 16 * i;
      if (m0 + r >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int c = tx + 16 * j;
        if (n0 + c >= g.N) continue;
        cplx* p = Cb + rowC[r] + colC[c];
        cplx v = cmul(g.alpha, acc[i][j]);
        if (has_beta) v = cadd(v, cmul(g.beta, *p));
        *p = v;
      }
    }
  }
}

inline int64_t abs64(int64_t v) { return v < 0 ? -v : v; }

}  // namespace

void validate(const ZGemm& g) {
  // an outer index with neither a table nor a stride is a set-up error, not a broadcast
  const IdxMap* maps[] = {&g.A.row, &g.A.col, &g.B.row, &g.B.col, &g.C.row, &g.C.col};
  for (const IdxMap* m : maps)
    require(!(m->n_in > 0 && m->tab == nullptr && m->s_out == 0), GB200_ERR_STATE, "zgemm: index map without outer table");
}

void zgemm_fp64(const ZGemm& g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return;
  validate(g);
  const int64_t nbatch = g.nb0 * g.nb1 * g.nb2;
  if (nbatch <= 0) return;
  LoadMode lm;
  // choose the coalescing direction: the index with the smaller inner stride walks fastest
  lm.a_kfast = abs64(g.A.col.s_in) <= abs64(g.A.row.s_in);
  lm.b_kfast = abs64(g.B.row.s_in) <= abs64(g.B.col.s_in);
  dim3 grid((unsigned)((g.N + BN - 1) / BN), (unsigned)((g.M + BM - 1) / BM),
            (unsigned)(nbatch < 65535 ? nbatch : 65535));
  require(grid.y <= 65535u, GB200_ERR_INVALID, "zgemm: M too large");
  zgemm_fp64_kernel<<<grid, NT, 0, st>>>(g, lm, nbatch);
  GB_CHECK_LAUNCH();
}

}  // namespace gb200
