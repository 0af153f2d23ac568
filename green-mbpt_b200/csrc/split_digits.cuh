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

#ifndef __CUDA_ARCH__
#include <cmath>
#include <cstring>
#endif

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

// X + balanced_bias(S) for X = rint(x) (round to nearest, ties to even), |x| < 2^(7S-1).  For
// S <= 7 (|x| < 2^48) adding 1.5 * 2^52 leaves rint(x) in the low mantissa bits of the sum, so its
// bit pattern minus that of 1.5 * 2^52 is rint(x): one addition instead of a conversion.
GB_DIGITS_FN uint64_t balanced_input(double x, int S) {
  if (S <= 7) {
    const double t = x + 6755399441055744.0;
#ifdef __CUDA_ARCH__
    const uint64_t bits = (uint64_t)__double_as_longlong(t);
#else
    uint64_t bits;
    std::memcpy(&bits, &t, sizeof bits);
#endif
    return bits - 0x4338000000000000ull + balanced_bias(S);
  }
#ifdef __CUDA_ARCH__
  return (uint64_t)__double2ll_rn(x) + balanced_bias(S);
#else
  return (uint64_t)std::llrint(x) + balanced_bias(S);
#endif
}

// Digit s of four values at once: byte i of the word is balanced_digit_byte(U_i, S, s).  The four
// raw digits d in [0, 128] are packed first; d - 64 (mod 256) is d ^ 64 where bit 6 of d is set
// and d | 0xC0 where it is not, which three logic operations apply to all four bytes.
GB_DIGITS_FN uint32_t balanced_digit_word(uint64_t u0, uint64_t u1, uint64_t u2, uint64_t u3, int S, int s) {
  const int sh = 7 * (S - 1 - s);
  const uint32_t t0 = (uint32_t)(u0 >> sh), t1 = (uint32_t)(u1 >> sh), t2 = (uint32_t)(u2 >> sh),
                 t3 = (uint32_t)(u3 >> sh);
#ifdef __CUDA_ARCH__
  uint32_t w = __byte_perm(__byte_perm(t0, t1, 0x0040), __byte_perm(t2, t3, 0x0040), 0x5410);
#else
  uint32_t w = (t0 & 0xFFu) | ((t1 & 0xFFu) << 8) | ((t2 & 0xFFu) << 16) | ((t3 & 0xFFu) << 24);
#endif
  if (s > 0) w &= 0x7F7F7F7Fu;  // the top digit takes all bits above it (at most 128)
  return w ^ 0x40404040u ^ ((~w & 0x40404040u) << 1);
}

// two's complement negation of each byte (no carry between bytes)
GB_DIGITS_FN uint32_t negate_bytes(uint32_t w) { return (0x80808080u - (w & 0x7F7F7F7Fu)) ^ (~w & 0x80808080u); }

}  // namespace gb200
