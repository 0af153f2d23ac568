// FP64 batched complex GEMM over general index maps (the parity path), on the FP64 tensor cores.
//
// One CTA computes a 64 x 64 complex tile with 8 warps.  Each warp owns 16 x 32 complex results as
// 2 x 4 tiles of 8 x 8 and forms them with mma.sync m8n8k4 (FP64 operands, FP64 accumulate): per
// step of 4 along K, Re C += Re A Re B - Im A Im B and Im C += Re A Im B + Im A Re B, four real
// products per tile.  Operand tiles of depth 16 are staged through shared memory as separate real
// and imaginary arrays; a row of 68 doubles puts the 4 K rows x 4 columns that a half-warp's
// fragments read on 16 different bank pairs.  The next depth-16 tile is loaded into registers
// while the current one is multiplied.  Global reads follow the operand's fastest-varying index, so
// row- and column-major views both coalesce; offsets of the tile's rows and columns are decoded once
// per CTA from the IdxMap, the K offsets once per K step.
#include "common.cuh"

namespace gb200 {
namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;
constexpr int LDS = BM + 4;  // shared row length in doubles (BM == BN)

struct LoadMode {
  bool a_kfast;  // consecutive threads walk K for A (else walk M)
  bool b_kfast;  // consecutive threads walk K for B (else walk N)
};

// D = A B + D for one 8 x 8 x 4 FP64 tile (A row-major 8 x 4, B column-major 4 x 8): lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(NT) zgemm_fp64_kernel(ZGemm g, LoadMode lm, int64_t nbatch) {
  __shared__ double Ar[BK][LDS], Ai[BK][LDS], Br[BK][LDS], Bi[BK][LDS];
  __shared__ int64_t rowA[BM], colB[BN], rowC[BM], colC[BN];
  __shared__ int64_t kA[BK], kB[BK];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp >> 1) * 16, wc = (warp & 1) * 32;  // the warp's rows and columns in the tile
  const int fr = lane >> 2, fk = lane & 3;                // fragment row (column for B) and K index
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
  const int nkt = (int)((g.K + BK - 1) / BK);

  for (int64_t b = blockIdx.z; b < nbatch; b += gridDim.z) {
    const int64_t b2 = b % g.nb2;
    const int64_t b1 = (b / g.nb2) % g.nb1;
    const int64_t b0 = b / (g.nb2 * g.nb1);
    const cplx* Ab = g.A.ptr + g.A.bat(b0, b1, b2);
    const cplx* Bb = g.B.ptr + g.B.bat(b0, b1, b2);
    cplx* Cb = g.C.ptr + g.C.bat(b0, b1, b2);

    double cr[2][4][2], ci[2][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;

    cplx va[(BM * BK) / NT], vb[(BN * BK) / NT];  // the next K tile, in registers
    auto k_offsets = [&](int kt) {
      if (tid < BK) {
        const int64_t k = (int64_t)kt * BK + tid;
        kA[tid] = k < g.K ? g.A.col(k) : 0;
      } else if (tid < 2 * BK) {
        const int64_t k = (int64_t)kt * BK + tid - BK;
        kB[tid - BK] = k < g.K ? g.B.row(k) : 0;
      }
    };
    auto load_tile = [&](int kt) {
      const int64_t k0 = (int64_t)kt * BK;
#pragma unroll
      for (int i = 0; i < (BM * BK) / NT; ++i) {
        const int e = tid + i * NT;
        int r, kk;
        if (lm.a_kfast) { kk = e % BK; r = e / BK; } else { r = e % BM; kk = e / BM; }
        va[i] = (m0 + r < g.M && k0 + kk < g.K) ? Ab[rowA[r] + kA[kk]] : cmk(0.0, 0.0);
      }
#pragma unroll
      for (int i = 0; i < (BN * BK) / NT; ++i) {
        const int e = tid + i * NT;
        int c, kk;
        if (lm.b_kfast) { kk = e % BK; c = e / BK; } else { c = e % BN; kk = e / BN; }
        vb[i] = (n0 + c < g.N && k0 + kk < g.K) ? Bb[kB[kk] + colB[c]] : cmk(0.0, 0.0);
      }
    };

    __syncthreads();  // row/column tables (and the previous batch's use of kA/kB)
    k_offsets(0);
    __syncthreads();
    load_tile(0);
    for (int kt = 0; kt < nkt; ++kt) {
      __syncthreads();  // the previous step's fragments have been read; kA/kB were consumed
#pragma unroll
      for (int i = 0; i < (BM * BK) / NT; ++i) {
        const int e = tid + i * NT;
        int r, kk;
        if (lm.a_kfast) { kk = e % BK; r = e / BK; } else { r = e % BM; kk = e / BM; }
        Ar[kk][r] = va[i].x;
        Ai[kk][r] = g.A.conj ? -va[i].y : va[i].y;
      }
#pragma unroll
      for (int i = 0; i < (BN * BK) / NT; ++i) {
        const int e = tid + i * NT;
        int c, kk;
        if (lm.b_kfast) { kk = e % BK; c = e / BK; } else { c = e % BN; kk = e / BN; }
        Br[kk][c] = vb[i].x;
        Bi[kk][c] = g.B.conj ? -vb[i].y : vb[i].y;
      }
      if (kt + 1 < nkt) k_offsets(kt + 1);
      __syncthreads();
      if (kt + 1 < nkt) load_tile(kt + 1);  // in flight while this tile is multiplied
#pragma unroll
      for (int k4 = 0; k4 < BK; k4 += 4) {
        const int kq = k4 + fk;
        double are[2], aim[2], bre[4], bim[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          are[i] = Ar[kq][wr + i * 8 + fr];
          aim[i] = Ai[kq][wr + i * 8 + fr];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          bre[j] = Br[kq][wc + j * 8 + fr];
          bim[j] = Bi[kq][wc + j * 8 + fr];
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            dmma(cr[i][j], are[i], bre[j]);
            dmma(cr[i][j], -aim[i], bim[j]);
            dmma(ci[i][j], are[i], bim[j]);
            dmma(ci[i][j], aim[i], bre[j]);
          }
      }
    }
    const bool has_beta = (g.beta.x != 0.0 || g.beta.y != 0.0);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = wr + i * 8 + fr;
      if (m0 + r >= g.M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = wc + j * 8 + 2 * fk + h;
          if (n0 + c >= g.N) continue;
          cplx* p = Cb + rowC[r] + colC[c];
          cplx v = cmul(g.alpha, cmk(cr[i][j][h], ci[i][j][h]));
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
