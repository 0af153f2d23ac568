// Test stand-in for green::grids::transformer_t: the transforms the B200 plug-in applies
// (tau_to_omega, omega_to_tau, tau_f_to_w_b, w_b_to_tau_f, wsample_fermi, sd().repn_*()), here
// dense matrices loaded from files and applied along the leading (time) dimension.  Test
// infrastructure only.
#pragma once
#include <complex>
#include <string>
#include <vector>

#include "../ndarray/ndarray.h"
#include "../stub_io.h"

namespace green::grids {

class transformer_t {
  using cd = std::complex<double>;
  struct repn {
    size_t nts_, nw_;
    size_t nts() const { return nts_; }
    size_t nw() const { return nw_; }
  };
  struct sparse_data {
    repn f, b;
    const repn& repn_fermi() const { return f; }
    const repn& repn_bose() const { return b; }
  };
  struct wvec {
    const std::vector<double>* w;
    double operator()(size_t i) const { return (*w)[i]; }
  };

 public:
  explicit transformer_t(const std::string& dir)
      : Tnt_f_(stub::load<cd>(dir + "/Tnt_f")), Ttn_f_(stub::load<cd>(dir + "/Ttn_f")),
        Tnt_b_(stub::load<cd>(dir + "/Tnt_b")), Ttn_b_(stub::load<cd>(dir + "/Ttn_b")),
        wf_(stub::load<double>(dir + "/wsample_f")) {
    const auto s = stub::shape_of(dir + "/Tnt_f");
    const auto sb = stub::shape_of(dir + "/Tnt_b");
    sd_.f = {s[1], s[0]};
    sd_.b = {sb[1], sb[0]};
  }
  const sparse_data& sd() const { return sd_; }
  wvec wsample_fermi() const { return wvec{&wf_}; }

  template <size_t N>
  void tau_to_omega(const ndarray::ndarray<cd, N>& X, ndarray::ndarray<cd, N>& Y, int) const {
    apply(Tnt_f_, sd_.f.nw_, sd_.f.nts_, X, Y);
  }
  template <size_t N>
  void omega_to_tau(const ndarray::ndarray<cd, N>& X, ndarray::ndarray<cd, N>& Y, int) const {
    apply(Ttn_f_, sd_.f.nts_, sd_.f.nw_, X, Y);
  }
  template <size_t N>
  void tau_f_to_w_b(const ndarray::ndarray<cd, N>& X, ndarray::ndarray<cd, N>& Y, size_t, size_t, bool) const {
    apply(Tnt_b_, sd_.b.nw_, sd_.f.nts_, X, Y);
  }
  template <size_t N>
  void w_b_to_tau_f(const ndarray::ndarray<cd, N>& X, ndarray::ndarray<cd, N>& Y, size_t, size_t, bool) const {
    apply(Ttn_b_, sd_.f.nts_, sd_.b.nw_, X, Y);
  }

 private:
  // Y[i][...] = sum_j T[i][j] X[j][...]
  template <size_t N>
  static void apply(const std::vector<cd>& T, size_t ni, size_t nj, const ndarray::ndarray<cd, N>& X,
                    ndarray::ndarray<cd, N>& Y) {
    const size_t inner = X.size() / X.shape()[0];
    for (size_t i = 0; i < ni; ++i)
      for (size_t r = 0; r < inner; ++r) {
        cd s = 0.0;
        for (size_t j = 0; j < nj; ++j) s += T[i * nj + j] * X.data()[j * inner + r];
        Y.data()[i * inner + r] = s;
      }
  }
  std::vector<cd> Tnt_f_, Ttn_f_, Tnt_b_, Ttn_b_;
  std::vector<double> wf_;
  sparse_data sd_{};
};

}  // namespace green::grids
