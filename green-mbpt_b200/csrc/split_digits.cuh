// Balanced base-128 digits of the split-precision slices (shared by the slicer kernels and the
// host-side test of the digit arithmetic).
//
// With the row exponent e (|a| < 2^(e-1)) and X = rint(a 2^(7S - e)), |X| < 2^(7S-1) and
// X = sum_p d_p 128^p with d_p in [-64, 63] for p < S - 1 and the top digit in [-64, 64].
// Rounding to nearest and signed digits make both the representation error and the digit products
// left out of the kept diagonals zero-mean, so they do not add up along the contraction the way the
// errors of truncation toward zero do.  Adding H = 64 (128^S - 1) / 127 (64 in every digit) turns
// the balanced digits into the unsigned base-128 digits of X + H >= 0.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define GB_DIGITS_FN __host__ __device__ __forceinline__
#else
#define GB_DIGITS_FN inline
#endif

namespace gb200 {

// H = 64 (128^S - 1) / 127, for 1 <= S <= 8
GB_DIGITS_FN uint64_t balanced_bias(int S) { return ((((uint64_t)1) << (7 * S)) - 1) / 127 * 64; }

// digit s (s = 0 the top one, weight 128^(S-1-s)) of X from U = X + balanced_bias(S) (computed
// modulo 2^64, so U >= 0 for every |X| < 2^(7S-1)), as a byte
GB_DIGITS_FN uint32_t balanced_digit_byte(uint64_t U, int S, int s) {
  const int p = S - 1 - s;
  const int d = (s == 0) ? (int)(U >> (7 * p)) - 64 : (int)((U >> (7 * p)) & 127u) - 64;
  return (uint32_t)d & 0xFFu;
}

}  // namespace gb200
