// FP64 batched linear algebra: hermitization and Gauss-Jordan inverses.
//
// Small matrices (n <= 64, the Dyson inverses of nso x nso) live entirely in
// shared memory, one CTA per matrix.  Large ones (the NQ x NQ aux-basis
// matrices of the screened interaction) keep the augmented [A | I] in a
// global scratch buffer, one CTA per matrix: blocked by panels of 16 pivots
// when the panel fits shared memory, one pivot at a time otherwise.  All use
// partial (row) pivoting.
#include "context.cuh"

namespace gb200 {
namespace {

__global__ void hermitize_kernel(cplx* X, int64_t nmat, int n, double scale) {
  const int64_t npairs = (int64_t)n * (n + 1) / 2;
  const int64_t total = nmat * npairs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int64_t m = e / npairs;
    int64_t p = e - m * npairs;
    // p -> (i, j) with i >= j
    int i = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > p) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= p) ++i;
    int j = (int)(p - (int64_t)i * (i + 1) / 2);
    cplx* M = X + m * (int64_t)n * n;
    cplx a = cscale(M[(int64_t)i * n + j], scale);
    cplx b = cscale(M[(int64_t)j * n + i], scale);
    cplx h = cscale(cadd(a, cconj(b)), 0.5);
    M[(int64_t)i * n + j] = h;
    M[(int64_t)j * n + i] = cconj(h);
  }
}

__global__ void scale_kernel(cplx* X, int64_t count, double s) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x) {
    X[e] = cscale(X[e], s);
  }
}

__device__ __forceinline__ cplx crecip(cplx a) {
  double d = a.x * a.x + a.y * a.y;
  return make_double2(a.x / d, -a.y / d);
}

// Block-wide argmax of |aug[i][j]|^2 over i in [j, n).
template <int NT>
__device__ int pivot_search(const cplx* aug, int64_t ld, int j, int n, double* sval, int* sidx) {
  double best = -1.0;
  int bi = j;
  for (int i = j + threadIdx.x; i < n; i += NT) {
    double v = cabs2(aug[(int64_t)i * ld + j]);
    if (v > best) { best = v; bi = i; }
  }
  sval[threadIdx.x] = best;
  sidx[threadIdx.x] = bi;
  __syncthreads();
  for (int s = NT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double o = sval[threadIdx.x + s];
      int oi = sidx[threadIdx.x + s];
      if (o > sval[threadIdx.x] || (o == sval[threadIdx.x] && oi < sidx[threadIdx.x])) {
        sval[threadIdx.x] = o;
        sidx[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  int p = sidx[0];
  __syncthreads();
  return p;
}

constexpr int SMALL_NT = 256;

__global__ void __launch_bounds__(SMALL_NT) invert_small_kernel(const cplx* A, cplx* Ainv, int n) {
  extern __shared__ double2 smem_c[];
  cplx* aug = smem_c;                 // n x 2n
  cplx* fac = aug + 2 * n * n;        // n
  __shared__ double sval[SMALL_NT];
  __shared__ int sidx[SMALL_NT];
  const int64_t m = blockIdx.x;
  const cplx* Am = A + m * (int64_t)n * n;
  const int ld = 2 * n;
  for (int e = threadIdx.x; e < n * n; e += SMALL_NT) {
    int i = e / n, c = e % n;
    aug[i * ld + c] = Am[e];
    aug[i * ld + n + c] = (i == c) ? cmk(1.0, 0.0) : cmk(0.0, 0.0);
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    int p = pivot_search<SMALL_NT>(aug, ld, j, n, sval, sidx);
    if (p != j) {
      for (int c = threadIdx.x; c < ld; c += SMALL_NT) {
        cplx t = aug[j * ld + c];
        aug[j * ld + c] = aug[p * ld + c];
        aug[p * ld + c] = t;
      }
      __syncthreads();
    }
    cplx inv = crecip(aug[j * ld + j]);
    __syncthreads();
    for (int c = threadIdx.x; c < ld; c += SMALL_NT) aug[j * ld + c] = cmul(aug[j * ld + c], inv);
    for (int i = threadIdx.x; i < n; i += SMALL_NT) fac[i] = aug[i * ld + j];
    __syncthreads();
    for (int e = threadIdx.x; e < n * (ld - j); e += SMALL_NT) {
      int i = e / (ld - j), c = j + e % (ld - j);
      if (i == j) continue;
      aug[i * ld + c] = csub(aug[i * ld + c], cmul(fac[i], aug[j * ld + c]));
    }
    __syncthreads();
  }
  cplx* Om = Ainv + m * (int64_t)n * n;
  for (int e = threadIdx.x; e < n * n; e += SMALL_NT) {
    int i = e / n, c = e % n;
    Om[e] = aug[i * ld + n + c];
  }
}

constexpr int LARGE_NT = 1024;

__global__ void __launch_bounds__(LARGE_NT) invert_large_kernel(const cplx* A, cplx* Ainv, cplx* augbase, int n,
                                                                 bool herm_from_lower, bool identity_minus) {
  extern __shared__ double2 smem_c[];
  cplx* prow = smem_c;           // 2n (pivot row)
  cplx* fac = prow + 2 * n;      // n
  __shared__ double sval[LARGE_NT];
  __shared__ int sidx[LARGE_NT];
  const int64_t m = blockIdx.x;
  const int ld = 2 * n;
  cplx* aug = augbase + m * (int64_t)n * ld;
  const cplx* Am = A + m * (int64_t)n * n;
  for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += LARGE_NT) {
    int i = (int)(e / n), c = (int)(e % n);
    // B = identity_minus ? I - A : A ; the inverted matrix is B itself or, with
    // herm_from_lower, the Hermitian matrix of B's strict lower triangle and
    // real diagonal (what Eigen's LDLT reads, gw_cpu_kernel.cpp:245-249)
    auto Bel = [&](int x, int y) -> cplx {
      cplx a = Am[(int64_t)x * n + y];
      return identity_minus ? cmk((x == y ? 1.0 : 0.0) - a.x, -a.y) : a;
    };
    cplx v;
    if (herm_from_lower) {
      if (i > c) v = Bel(i, c);
      else if (i < c) v = cconj(Bel(c, i));
      else v = cmk(Bel(i, i).x, 0.0);
    } else {
      v = Bel(i, c);
    }
    aug[(int64_t)i * ld + c] = v;
    aug[(int64_t)i * ld + n + c] = (i == c) ? cmk(1.0, 0.0) : cmk(0.0, 0.0);
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    int p = pivot_search<LARGE_NT>(aug, ld, j, n, sval, sidx);
    if (p != j) {
      for (int c = threadIdx.x; c < ld; c += LARGE_NT) {
        cplx t = aug[(int64_t)j * ld + c];
        aug[(int64_t)j * ld + c] = aug[(int64_t)p * ld + c];
        aug[(int64_t)p * ld + c] = t;
      }
      __syncthreads();
    }
    cplx inv = crecip(aug[(int64_t)j * ld + j]);
    for (int c = threadIdx.x; c < ld; c += LARGE_NT) prow[c] = cmul(aug[(int64_t)j * ld + c], inv);
    for (int i = threadIdx.x; i < n; i += LARGE_NT) fac[i] = aug[(int64_t)i * ld + j];
    __syncthreads();
    for (int c = threadIdx.x; c < ld; c += LARGE_NT) aug[(int64_t)j * ld + c] = prow[c];
    const int w = ld - j;
    for (int64_t e = threadIdx.x; e < (int64_t)n * w; e += LARGE_NT) {
      int i = (int)(e / w), c = j + (int)(e % w);
      if (i == j) continue;
      aug[(int64_t)i * ld + c] = csub(aug[(int64_t)i * ld + c], cmul(fac[i], prow[c]));
    }
    __syncthreads();
  }
  cplx* Om = Ainv + m * (int64_t)n * n;
  for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += LARGE_NT) {
    int i = (int)(e / n), c = (int)(e % n);
    Om[e] = aug[(int64_t)i * ld + n + c];
  }
}

// Blocked Gauss-Jordan with partial pivoting, one CTA per matrix (the aux-basis inverses of the
// screened interaction).  The augmented [B | I] lives in a global scratch buffer; rows are kept in
// a logical order through a permutation instead of being swapped.  Per panel of BLK_NB columns:
//   1. the panel is copied to shared memory and eliminated there to choose the pivot rows J
//      (the same choices as unblocked Gauss-Jordan with partial pivoting);
//   2. D = B[J, panel] (original values) is inverted in shared memory;
//   3. the remaining columns are updated in chunks:  R = D^-1 B[J, :],  B[J, :] = R,
//      B[i, :] -= B[i, panel] R for every other row i  (a rank-BLK_NB update, R in registers).
// The traffic through L2 is one read and one write of the remaining columns per panel instead
// of one per pivot.
constexpr int BLK_NB = 16, BLK_NT = 512, BLK_CH = 128;

__device__ __forceinline__ void block_argmax(double v, int idx, double* sval, int* sidx, int& best_idx) {
  // block-wide argmax of v (ties: smaller idx); every thread gets the result
  sval[threadIdx.x] = v;
  sidx[threadIdx.x] = idx;
  __syncthreads();
  for (int s = BLK_NT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = sval[threadIdx.x + s];
      const int oi = sidx[threadIdx.x + s];
      if (o > sval[threadIdx.x] || (o == sval[threadIdx.x] && oi < sidx[threadIdx.x])) {
        sval[threadIdx.x] = o;
        sidx[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  best_idx = sidx[0];
  __syncthreads();
}

__global__ void __launch_bounds__(BLK_NT) invert_blocked_kernel(const cplx* A, cplx* Ainv, cplx* augbase, int n,
                                                                bool herm_from_lower, bool identity_minus) {
  extern __shared__ double2 smem_c[];
  cplx* pan = smem_c;                        // [n][BLK_NB]: panel copy, then the original panel rows
  cplx* dinv = pan + (size_t)n * BLK_NB;     // [BLK_NB][2*BLK_NB]: D | I -> I | D^-1
  cplx* rch = dinv + 2 * BLK_NB * BLK_NB;    // [BLK_NB][BLK_CH]: R for one column chunk
  int* perm = reinterpret_cast<int*>(rch + BLK_NB * BLK_CH);  // logical row -> physical row
  __shared__ double sval[BLK_NT];
  __shared__ int sidx[BLK_NT];
  const int64_t m = blockIdx.x;
  const int ld = 2 * n;
  cplx* aug = augbase + m * (int64_t)n * ld;
  const cplx* Am = A + m * (int64_t)n * n;
  for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += BLK_NT) {
    const int i = (int)(e / n), c = (int)(e % n);
    auto Bel = [&](int x, int y) -> cplx {
      cplx a = Am[(int64_t)x * n + y];
      return identity_minus ? cmk((x == y ? 1.0 : 0.0) - a.x, -a.y) : a;
    };
    cplx v;
    if (herm_from_lower) {
      if (i > c) v = Bel(i, c);
      else if (i < c) v = cconj(Bel(c, i));
      else v = cmk(Bel(i, i).x, 0.0);
    } else {
      v = Bel(i, c);
    }
    aug[(int64_t)i * ld + c] = v;
    aug[(int64_t)i * ld + n + c] = (i == c) ? cmk(1.0, 0.0) : cmk(0.0, 0.0);
  }
  for (int i = threadIdx.x; i < n; i += BLK_NT) perm[i] = i;
  __syncthreads();
  for (int j0 = 0; j0 < n; j0 += BLK_NB) {
    const int nb = min(BLK_NB, n - j0);
    // 1. panel elimination in shared memory (logical row order) to choose the pivots
    for (int e = threadIdx.x; e < n * BLK_NB; e += BLK_NT) {
      const int li = e / BLK_NB, c = e % BLK_NB;
      pan[e] = c < nb ? aug[(int64_t)perm[li] * ld + j0 + c] : cmk(0.0, 0.0);
    }
    __syncthreads();
    for (int c = 0; c < nb; ++c) {
      const int jr = j0 + c;
      double best = -1.0;
      int bi = jr;
      for (int li = jr + threadIdx.x; li < n; li += BLK_NT) {
        const double v = cabs2(pan[li * BLK_NB + c]);
        if (v > best) { best = v; bi = li; }
      }
      int p;
      block_argmax(best, bi, sval, sidx, p);
      if (p != jr) {
        if (threadIdx.x < BLK_NB) {
          const cplx t = pan[jr * BLK_NB + threadIdx.x];
          pan[jr * BLK_NB + threadIdx.x] = pan[p * BLK_NB + threadIdx.x];
          pan[p * BLK_NB + threadIdx.x] = t;
        }
        if (threadIdx.x == 0) {
          const int t = perm[jr];
          perm[jr] = perm[p];
          perm[p] = t;
        }
      }
      __syncthreads();
      const cplx inv = crecip(pan[jr * BLK_NB + c]);
      __syncthreads();
      if (threadIdx.x < BLK_NB) pan[jr * BLK_NB + threadIdx.x] = cmul(pan[jr * BLK_NB + threadIdx.x], inv);
      __syncthreads();
      for (int e = threadIdx.x; e < n * BLK_NB; e += BLK_NT) {
        const int li = e / BLK_NB, cc = e % BLK_NB;
        if (li == jr || cc <= c) continue;
        pan[e] = csub(pan[e], cmul(pan[li * BLK_NB + c], pan[jr * BLK_NB + cc]));
      }
      __syncthreads();
      for (int li = threadIdx.x; li < n; li += BLK_NT)
        if (li != jr) pan[li * BLK_NB + c] = cmk(0.0, 0.0);
      __syncthreads();
    }

    // 2. original panel values in logical row order (pan) and [D | I] for the pivot block
    for (int e = threadIdx.x; e < n * BLK_NB; e += BLK_NT) {
      const int li = e / BLK_NB, c = e % BLK_NB;
      pan[e] = c < nb ? aug[(int64_t)perm[li] * ld + j0 + c] : cmk(0.0, 0.0);
    }
    for (int e = threadIdx.x; e < BLK_NB * 2 * BLK_NB; e += BLK_NT) {
      const int r = e / (2 * BLK_NB), c = e % (2 * BLK_NB);
      cplx v;
      if (c < BLK_NB) v = (r < nb && c < nb) ? aug[(int64_t)perm[j0 + r] * ld + j0 + c] : cmk(r == c ? 1.0 : 0.0, 0.0);
      else v = cmk(c - BLK_NB == r ? 1.0 : 0.0, 0.0);
      dinv[e] = v;
    }
    __syncthreads();
    // D^-1 by Gauss-Jordan with partial pivoting on [D | I] (512 threads = 16 x 32 entries)
    for (int c = 0; c < BLK_NB; ++c) {
      if (threadIdx.x == 0) {
        int pr = c;
        double b = cabs2(dinv[c * 2 * BLK_NB + c]);
        for (int r = c + 1; r < BLK_NB; ++r) {
          const double v = cabs2(dinv[r * 2 * BLK_NB + c]);
          if (v > b) { b = v; pr = r; }
        }
        sidx[0] = pr;
      }
      __syncthreads();
      const int pr = sidx[0];
      if (pr != c && threadIdx.x < 2 * BLK_NB) {
        const cplx t = dinv[c * 2 * BLK_NB + threadIdx.x];
        dinv[c * 2 * BLK_NB + threadIdx.x] = dinv[pr * 2 * BLK_NB + threadIdx.x];
        dinv[pr * 2 * BLK_NB + threadIdx.x] = t;
      }
      __syncthreads();
      const cplx inv = crecip(dinv[c * 2 * BLK_NB + c]);
      __syncthreads();
      if (threadIdx.x < 2 * BLK_NB) dinv[c * 2 * BLK_NB + threadIdx.x] = cmul(dinv[c * 2 * BLK_NB + threadIdx.x], inv);
      __syncthreads();
      {
        const int r = threadIdx.x / (2 * BLK_NB), cc = threadIdx.x % (2 * BLK_NB);
        const cplx f = (r != c) ? dinv[r * 2 * BLK_NB + c] : cmk(0.0, 0.0);
        __syncthreads();
        if (r != c) dinv[r * 2 * BLK_NB + cc] = csub(dinv[r * 2 * BLK_NB + cc], cmul(f, dinv[c * 2 * BLK_NB + cc]));
      }
      __syncthreads();
    }
    // 3. remaining columns in chunks: R = D^-1 B[J, chunk]; B[J, chunk] = R; other rows -= C R
    for (int col0 = j0 + nb; col0 < ld; col0 += BLK_CH) {
      const int cw = min(BLK_CH, ld - col0);
      for (int e = threadIdx.x; e < BLK_NB * BLK_CH; e += BLK_NT) {
        const int r = e / BLK_CH, cc = e % BLK_CH;
        cplx acc = cmk(0.0, 0.0);
        if (r < nb && cc < cw)
          for (int k = 0; k < nb; ++k)
            acc = cadd(acc, cmul(dinv[r * 2 * BLK_NB + BLK_NB + k], aug[(int64_t)perm[j0 + k] * ld + col0 + cc]));
        rch[e] = acc;
      }
      __syncthreads();
      const int cc = threadIdx.x % BLK_CH, grp = threadIdx.x / BLK_CH;
      if (cc < cw) {
        cplx rr[BLK_NB];
#pragma unroll
        for (int k = 0; k < BLK_NB; ++k) rr[k] = rch[k * BLK_CH + cc];
        for (int li = grp; li < n; li += BLK_NT / BLK_CH) {
          cplx* dst = aug + (int64_t)perm[li] * ld + col0 + cc;
          if (li >= j0 && li < j0 + nb) {
            *dst = rch[(li - j0) * BLK_CH + cc];
            continue;
          }
          cplx v = *dst;
          const cplx* cl = pan + li * BLK_NB;
#pragma unroll
          for (int k = 0; k < BLK_NB; ++k) v = csub(v, cmul(cl[k], rr[k]));
          *dst = v;
        }
      }
      __syncthreads();
    }
  }
  cplx* Om = Ainv + m * (int64_t)n * n;
  for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += BLK_NT) {
    const int i = (int)(e / n), c = (int)(e % n);
    Om[e] = aug[(int64_t)perm[i] * ld + n + c];
  }
}

size_t blocked_smem_bytes(int n) {
  return ((size_t)n * BLK_NB + 2 * BLK_NB * BLK_NB + BLK_NB * BLK_CH) * sizeof(cplx) + (size_t)n * sizeof(int);
}
inline unsigned grid_for(int64_t n, int nt) {
  int64_t g = (n + nt - 1) / nt;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (unsigned)g;
}

}  // namespace

void hermitize_batched(cplx* X, int64_t nmat, int n, double scale, cudaStream_t st) {
  if (nmat <= 0) return;
  int64_t total = nmat * (int64_t)n * (n + 1) / 2;
  hermitize_kernel<<<grid_for(total, 256), 256, 0, st>>>(X, nmat, n, scale);
  GB_CHECK_LAUNCH();
}

void scale_inplace(cplx* X, int64_t count, double s, cudaStream_t st) {
  if (count <= 0) return;
  scale_kernel<<<grid_for(count, 256), 256, 0, st>>>(X, count, s);
  GB_CHECK_LAUNCH();
}

void invert_small_batched(const cplx* A, cplx* Ainv, int64_t nmat, int n, cudaStream_t st) {
  require(n <= 64, GB200_ERR_INVALID, "invert_small_batched: n > 64");
  if (nmat <= 0) return;
  size_t smem = (size_t)(2 * n * n + n) * sizeof(cplx);
  // set on every call: the attribute belongs to the current device, and contexts on other devices
  // or threads call this too (a host-side call of about a microsecond)
  GB_CUDA(cudaFuncSetAttribute(invert_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  for (int64_t off = 0; off < nmat; off += 2147483647LL) {
    int64_t cnt = nmat - off < 2147483647LL ? nmat - off : 2147483647LL;
    invert_small_kernel<<<(unsigned)cnt, SMALL_NT, smem, st>>>(A + off * n * n, Ainv + off * n * n, n);
    GB_CHECK_LAUNCH();
  }
}

void invert_large_batched(const cplx* A, cplx* Ainv, cplx* aug, int64_t nmat, int n, bool herm_from_lower,
                          bool identity_minus, cudaStream_t st) {
  require(n <= 4096, GB200_ERR_INVALID, "invert_large_batched: n > 4096");
  if (nmat <= 0) return;
  GB_CUDA(cudaFuncSetAttribute(invert_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  GB_CUDA(cudaFuncSetAttribute(invert_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
  const size_t bsmem = blocked_smem_bytes(n);
  if (bsmem <= 220 * 1024) {
    // blocked elimination (panel in shared memory) for the sizes whose panel fits
    invert_blocked_kernel<<<(unsigned)nmat, BLK_NT, bsmem, st>>>(A, Ainv, aug, n, herm_from_lower, identity_minus);
  } else {
    const size_t smem = (size_t)(3 * n) * sizeof(cplx);
    invert_large_kernel<<<(unsigned)nmat, LARGE_NT, smem, st>>>(A, Ainv, aug, n, herm_from_lower, identity_minus);
  }
  GB_CHECK_LAUNCH();
}

}  // namespace gb200
