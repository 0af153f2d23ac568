// Test stand-in for green::symmetry::brillouin_zone_utils with the members the B200 plug-in and
// the df_integral_t stand-in use: nk(), ink(), k_q_map() (k1_from_k2q, k2_from_k1q) and
// k_symmetry() (value_AO, full_point, the k-pair symmetry lists).  value_AO restates the
// green-symmetry operation the reference applies (U_k X_red U_k^H, conjugated for time-reversal
// partners) for the test.  Test infrastructure only.
#pragma once
#include <complex>
#include <string>
#include <vector>

#include "../ndarray/ndarray.h"
#include "../stub_io.h"

namespace green::symmetry {

class brillouin_zone_utils {
  using cd = std::complex<double>;

 public:
  struct kq_map_t {
    const brillouin_zone_utils* bz;
    size_t k1_from_k2q(size_t k2, size_t q) const { return (size_t)bz->kplus_[k2 * bz->nk_ + q]; }
    size_t k2_from_k1q(size_t k1, size_t q) const { return (size_t)bz->kminus_[k1 * bz->nk_ + q]; }
  };
  struct mat {
    size_t n;
    std::vector<cd> v;
    cd operator()(size_t i, size_t j) const { return v[i * n + j]; }
  };
  struct k_symmetry_t {
    const brillouin_zone_utils* bz;
    size_t full_point(size_t ik) const { return (size_t)bz->ibz2bz_[ik]; }
    const std::vector<int64_t>& conj_kpair_list() const { return bz->conj_; }
    const std::vector<int64_t>& trans_kpair_list() const { return bz->trans_; }
    long irre_pos_kpair(size_t idx) const {
      for (size_t i = 0; i < bz->irre_.size(); ++i)
        if ((size_t)bz->irre_[i] == idx) return (long)i;
      return -1;
    }
    mat value_AO(const ndarray::ndarray<cd, 3>& X, size_t k) const {
      const size_t n = X.shape()[1];
      size_t red = 0;
      for (size_t i = 0; i < bz->ibz2bz_.size(); ++i)
        if (bz->ibz2bz_[i] == bz->bz2ibz_[k]) red = i;
      const cd* Y = X.data() + red * n * n;
      const cd* U = bz->U_.data() + k * n * n;
      mat T{n, std::vector<cd>(n * n)}, R{n, std::vector<cd>(n * n)};
      for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
          cd s = 0.0;
          for (size_t a = 0; a < n; ++a) s += U[i * n + a] * Y[a * n + j];
          T.v[i * n + j] = s;
        }
      for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
          cd s = 0.0;
          for (size_t a = 0; a < n; ++a) s += T.v[i * n + a] * std::conj(U[j * n + a]);
          R.v[i * n + j] = bz->tr_[k] ? std::conj(s) : s;
        }
      return R;
    }
  };

  explicit brillouin_zone_utils(const std::string& dir)
      : kplus_(stub::load<int64_t>(dir + "/kplus")), kminus_(stub::load<int64_t>(dir + "/kminus")),
        bz2ibz_(stub::load<int64_t>(dir + "/bz2ibz")), ibz2bz_(stub::load<int64_t>(dir + "/ibz2bz")),
        tr_(stub::load<int64_t>(dir + "/tr_conj")), conj_(stub::load<int64_t>(dir + "/conj_pairs_list")),
        trans_(stub::load<int64_t>(dir + "/trans_pairs_list")), irre_(stub::load<int64_t>(dir + "/kpair_irre_list")),
        U_(stub::load<cd>(dir + "/k_sym_transform_ao")) {
    nk_ = bz2ibz_.size();
  }
  size_t nk() const { return nk_; }
  size_t ink() const { return ibz2bz_.size(); }
  kq_map_t k_q_map() const { return kq_map_t{this}; }
  k_symmetry_t k_symmetry() const { return k_symmetry_t{this}; }

 private:
  std::vector<int64_t> kplus_, kminus_, bz2ibz_, ibz2bz_, tr_, conj_, trans_, irre_;
  std::vector<cd> U_;
  size_t nk_ = 0;
};

}  // namespace green::symmetry
