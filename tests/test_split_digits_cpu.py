"""The balanced digit arithmetic of the split-precision slicer (green-mbpt_b200/csrc/split_digits.cuh),
compiled as host code and checked bit for bit on the CPU against an independent bottom-up
construction: for every slice count 2..8 and values across the whole range |X| < 2^(7S-1),
including both ends, the digits lie in [-64, 63] (the top one in [-64, 64]) and
sum_p d_p 128^p = X."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#include "split_digits.cuh"
int main() {
  int S; long long X;
  while (std::scanf("%d %lld", &S, &X) == 2) {
    const unsigned long long U = (unsigned long long)X + gb200::balanced_bias(S);
    for (int s = 0; s < S; ++s) std::printf("%d ", (int)(signed char)gb200::balanced_digit_byte(U, S, s));
    std::printf("\n");
  }
  return 0;
}
'''


def bottom_up(X, S):
    """Balanced base-128 digits from the least significant one (top digit = what remains)."""
    d = []
    for _ in range(S - 1):
        r = ((X + 64) % 128) - 64
        d.append(r)
        X = (X - r) // 128
    d.append(X)
    return d[::-1]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not installed")
    d = tmp_path_factory.mktemp("digits")
    src, exe = d / "h.cpp", d / "h"
    src.write_text(HARNESS)
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "green-mbpt_b200", "csrc"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def test_balanced_digits_match_bottom_up_construction(harness):
    rng = np.random.default_rng(0)
    cases = []
    for S in range(2, 9):
        lim = (1 << (7 * S - 1))
        vals = [0, 1, -1, 63, 64, -64, -65, 127, 128, lim - 1, -(lim - 1), lim // 2, -(lim // 2)]
        vals += [int(v) for v in rng.integers(-(lim - 1), lim, 200, dtype=np.int64)]
        cases += [(S, v) for v in vals]
    inp = "".join(f"{S} {v}\n" for S, v in cases)
    out = subprocess.run([harness], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    for (S, X), line in zip(cases, out):
        got = [int(t) for t in line.split()]
        assert got == bottom_up(X, S), (S, X, got)
        assert all(-64 <= g <= 63 for g in got[1:]) and -64 <= got[0] <= 64
        assert sum(g * 128 ** (S - 1 - i) for i, g in enumerate(got)) == X


def test_rounded_scaling_stays_in_range():
    """With the exponent one above frexp's, rint(a 2^(7S - e)) stays within |X| <= 2^(7S-1), the
    range the digits cover (the top digit reaches 64 only at the bound itself)."""
    for S in range(2, 9):
        for a in (1.0 - 2.0 ** -53, -(1.0 - 2.0 ** -53), 0.75, 2.0 ** -30, 1e-300):
            _, e = np.frexp(abs(a))
            X = int(np.rint(np.ldexp(a, 7 * S - (int(e) + 1))))
            assert abs(X) <= (1 << (7 * S - 1))
            if abs(X) < (1 << 62):
                d = bottom_up(X, S)
                assert -64 <= d[0] <= 64


PACKED = r'''
#include <cstdio>
#include "split_digits.cuh"
using namespace gb200;
int main() {
  int S; double x[4];
  while (std::scanf("%d %lf %lf %lf %lf", &S, &x[0], &x[1], &x[2], &x[3]) == 5) {
    unsigned long long u[4];
    for (int i = 0; i < 4; ++i) {
      u[i] = balanced_input(x[i], S);
      std::printf("%lld ", (long long)(u[i] - balanced_bias(S)));
    }
    for (int s = 0; s < S; ++s) {
      const unsigned w = balanced_digit_word(u[0], u[1], u[2], u[3], S, s);
      unsigned ref = 0;
      for (int i = 0; i < 4; ++i) ref |= balanced_digit_byte(u[i], S, s) << (8 * i);
      unsigned neg = 0;
      for (int i = 0; i < 4; ++i) neg |= ((0u - ((ref >> (8 * i)) & 0xFFu)) & 0xFFu) << (8 * i);
      std::printf("%u %u %u %u ", w, ref, negate_bytes(w), neg);
    }
    std::printf("\n");
  }
  return 0;
}
'''


def test_packed_digit_words_match_single_digits(tmp_path):
    """The slicers' fast path (split_digits.cuh, compiled here as host code): balanced_input rounds
    x to nearest, ties to even, through the 1.5 * 2^52 addition (as np.rint does);
    balanced_digit_word packs the digits of four values into the same bytes as four calls of
    balanced_digit_byte; negate_bytes negates each byte without carries, for every slice count
    and values across the whole range, both ends included."""
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not installed")
    src, exe = tmp_path / "p.cpp", tmp_path / "p"
    src.write_text(PACKED)
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "green-mbpt_b200", "csrc"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    rng = np.random.default_rng(3)
    cases = []
    for S in range(2, 9):
        lim = float(1 << (7 * S - 1))
        edge = [0.0, 0.5, -0.5, 1.5, -2.5, lim - 1.0, -(lim - 1.0), 63.5, -64.5]
        vals = edge + [float(v) for v in rng.uniform(-(lim - 1.0), lim - 1.0, 400)]
        vals += [float(v) for v in rng.uniform(-300, 300, 40)]
        vals += [float(v) for v in rng.integers(-200, 200, 40)]
        while len(vals) % 4:
            vals.append(0.0)
        cases += [(S, vals[i:i + 4]) for i in range(0, len(vals), 4)]
    inp = "".join(f"{S} " + " ".join(repr(v) for v in x) + "\n" for S, x in cases)
    out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    for (S, x), line in zip(cases, out):
        t = [int(v) for v in line.split()]
        assert t[:4] == [int(np.rint(v)) for v in x], (S, x, t[:4])
        for s in range(S):
            w, ref, neg_w, neg_ref = t[4 + 4 * s: 8 + 4 * s]
            assert w == ref and neg_w == neg_ref, (S, s, x, w, ref, neg_w, neg_ref)
