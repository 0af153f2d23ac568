// Test stand-in for green-mbpt's df_integral_t: the irreducible k-pair chunk of an integral
// directory (here <path>/V_chunk.bin, [npairs_irreducible][NQ][nao][nao]), read_integrals(k1, k2)
// and symmetrize(v, k1, k2) restating df_integral_t.h:64-84,162-203 (stored pair k1 >= k2, the
// conjugate transpose for k1 < k2, then the conj / trans pair symmetry) for the test.
#pragma once
#include <complex>
#include <string>
#include <vector>

#include "../stub_io.h"
#include "../symmetry/symmetry.h"
#include "kernels.h"

namespace green::mbpt {

class df_integral_t {
  using cd = std::complex<double>;

 public:
  df_integral_t(const std::string& path, int nao, int NQ, const symmetry::brillouin_zone_utils& bz)
      : V_(stub::load<cd>(path + "/V_chunk")), nao_(nao), NQ_(NQ), bz_(bz) {}
  void read_integrals(size_t, size_t) {}
  template <typename prec>
  void symmetrize(tensor<prec, 3>& v, size_t k1, size_t k2) {
    size_t idx = k1 >= k2 ? k1 * (k1 + 1) / 2 + k2 : k2 * (k2 + 1) / 2 + k1;
    int kind = 0;  // 0 direct, 1 conjugated, 2 transposed
    const auto ks = bz_.k_symmetry();
    if ((size_t)ks.conj_kpair_list()[idx] != idx) {
      idx = ks.conj_kpair_list()[idx];
      kind = 1;
    } else if ((size_t)ks.trans_kpair_list()[idx] != idx) {
      idx = ks.trans_kpair_list()[idx];
      kind = 2;
    }
    const long red = ks.irre_pos_kpair(idx);
    const size_t n = nao_, n2 = n * n;
    const cd* src = V_.data() + (size_t)red * NQ_ * n2;
    for (int Q = 0; Q < NQ_; ++Q)
      for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
          cd x = k1 < k2 ? std::conj(src[Q * n2 + j * n + i]) : src[Q * n2 + i * n + j];
          v.data()[Q * n2 + i * n + j] = x;
        }
    if (kind == 1)
      for (size_t e = 0; e < (size_t)NQ_ * n2; ++e) v.data()[e] = std::conj(v.data()[e]);
    if (kind == 2)
      for (int Q = 0; Q < NQ_; ++Q)
        for (size_t i = 0; i < n; ++i)
          for (size_t j = i + 1; j < n; ++j) std::swap(v.data()[Q * n2 + i * n + j], v.data()[Q * n2 + j * n + i]);
  }

 private:
  std::vector<cd> V_;
  int nao_, NQ_;
  const symmetry::brillouin_zone_utils& bz_;
};

}  // namespace green::mbpt
