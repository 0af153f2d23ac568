// green-mbpt custom-kernel plug-in for the B200 library: the GW and HF kernel callbacks of
// kernel_factory.h on top of the C ABI of include/gb200.h.
//
// What the shim does on the host, with green-mbpt's own objects:
//  * the k+q / k-q tables of bz.k_q_map() (call sites gw_cpu_kernel.cpp:90,117);
//  * the imaginary-time transforms as dense matrices: the transformer applied to unit vectors with
//    the calls the CPU kernels make (gw_cpu_kernel.cpp:234,264; dyson.cpp:205,213);
//  * the integrals of every stored pair k1 >= k2, read and symmetrized by green-mbpt's
//    df_integral_t (read_integrals / symmetrize, df_integral_t.h:64-84,162-177);
//  * k-point symmetry: G, the density matrix and S at the irreducible points are expanded to the
//    full zone with value_AO (the expansion gw_cpu_kernel.cpp:177,337 makes per k-pair), the
//    results are returned at the irreducible points (k_symmetry().full_point).
// The device work is one gb200_gw_sigma / gb200_hf_fock call per callback.
#include "gb200_green_kernel.h"

#include <gb200.h>

#include <complex>
#include <string>
#include <vector>

#include <green/mbpt/df_integral_t.h>
#include <green/mbpt/except.h>

namespace gb200_green {
namespace {

using cd = std::complex<double>;
using green::mbpt::ztensor;
using bz_utils_t = green::symmetry::brillouin_zone_utils;

// status code -> the reference's exception classes (except.h:28-46)
void check(int rc, gb200_context* c) {
  if (rc == GB200_OK) return;
  const std::string m = gb200_last_error(c);
  if (rc == GB200_ERR_WRONG_GRID) throw green::mbpt::mbpt_wrong_grid(m);
  if (rc == GB200_ERR_MU_SEARCH) throw green::mbpt::mbpt_chemical_potential_search_failure(m);
  if (rc == GB200_ERR_OUTDATED_INPUT) throw green::mbpt::mbpt_outdated_input(m);
  throw green::mbpt::mbpt_kernel_error(m);
}

struct handle {
  gb200_context* c = nullptr;
  handle() = default;
  handle(const handle&) = delete;
  handle& operator=(const handle&) = delete;
  ~handle() {
    if (c) gb200_destroy(c);
  }
};

void upload_maps(gb200_context* c, const bz_utils_t& bz) {
  const size_t nk = bz.nk();
  std::vector<int32_t> kp(nk * nk), km(nk * nk);
  for (size_t k = 0; k < nk; ++k)
    for (size_t q = 0; q < nk; ++q) {
      kp[k * nk + q] = (int32_t)bz.k_q_map().k1_from_k2q(k, q);
      km[k * nk + q] = (int32_t)bz.k_q_map().k2_from_k1q(k, q);
    }
  check(gb200_set_kq_maps(c, kp.data(), km.data()), c);
}

ztensor<2> unit(size_t n) {
  ztensor<2> I(n, n);
  I.set_zero();
  for (size_t i = 0; i < n; ++i) I.data()[i * n + i] = cd(1.0, 0.0);
  return I;
}

// Columns of the identity through each transform of the CPU kernels: Tnt_f [nw][nts] (tau_to_omega,
// dyson.cpp:205), Ttn_f [nts][nw] (omega_to_tau, dyson.cpp:213), Tnt_b [nw_b][nts] and Ttn_b
// [nts][nw_b] (tau_f_to_w_b / w_b_to_tau_f with the arguments of gw_cpu_kernel.cpp:234,264; the
// polarization they act on is symmetric in tau, as the GPU's is).
void upload_grid(gb200_context* c, const green::grids::transformer_t& ft) {
  const size_t nts = ft.sd().repn_fermi().nts(), nw = ft.sd().repn_fermi().nw(), nwb = ft.sd().repn_bose().nw();
  const ztensor<2> It = unit(nts), Iw = unit(nw), Iwb = unit(nwb);
  ztensor<2> Tnt_f(nw, nts), Ttn_f(nts, nw), Tnt_b(nwb, nts), Ttn_b(nts, nwb);
  ft.tau_to_omega(It, Tnt_f, 1);
  ft.omega_to_tau(Iw, Ttn_f, 1);
  ft.tau_f_to_w_b(It, Tnt_b, 0, nwb, true);
  ft.w_b_to_tau_f(Iwb, Ttn_b, 0, nts, true);
  std::vector<double> wf(nw);
  for (size_t i = 0; i < nw; ++i) wf[i] = ft.wsample_fermi()(i);
  check(gb200_set_grid(c, reinterpret_cast<const double*>(Tnt_f.data()), reinterpret_cast<const double*>(Ttn_f.data()),
                       reinterpret_cast<const double*>(Tnt_b.data()), reinterpret_cast<const double*>(Ttn_b.data()),
                       wf.data()),
        c);
}

// Every stored pair k1 >= k2 of the full zone from the irreducible chunks on disk, in the layout
// gb200_set_integrals takes ([nk(nk+1)/2][NQ][nao][nao], pair index k1 (k1 + 1) / 2 + k2).
void upload_integrals(gb200_context* c, const std::string& path, int which, size_t nao, size_t NQ,
                      const bz_utils_t& bz) {
  const size_t nk = bz.nk(), pe = NQ * nao * nao, npairs = nk * (nk + 1) / 2;
  green::mbpt::df_integral_t ints(path, (int)nao, (int)NQ, bz);
  std::vector<cd> half(npairs * pe);
  ztensor<3> v(NQ, nao, nao);
  for (size_t k1 = 0; k1 < nk; ++k1)
    for (size_t k2 = 0; k2 <= k1; ++k2) {
      ints.read_integrals(k1, k2);
      ints.symmetrize(v, k1, k2);
      const cd* src = v.data();
      std::copy(src, src + pe, half.begin() + (k1 * (k1 + 1) / 2 + k2) * pe);
    }
  check(gb200_set_integrals(c, which, reinterpret_cast<const double*>(half.data()), (int64_t)npairs), c);
}

// [lead..., ink, n, n] at the irreducible points -> [lead..., nk, n, n] (value_AO of each full-zone
// point); `lead` is the product of the leading dimensions of X viewed as [lead][ink][n][n]
template <size_t D>
std::vector<cd> full_zone(const ztensor<D>& X, const bz_utils_t& bz) {
  static_assert(D == 4 || D == 5, "objects are [ns][ink][n][n] or [nts][ns][ink][n][n]");
  const size_t nk = bz.nk(), n = X.shape()[D - 1];
  const size_t d0 = X.shape()[0], d1 = D == 5 ? X.shape()[1] : 1;
  std::vector<cd> out(d0 * d1 * nk * n * n);
  for (size_t a = 0; a < d0; ++a)
    for (size_t b = 0; b < d1; ++b) {
      const ztensor<3> Xab = [&] {
        if constexpr (D == 5) return X(a, b);
        else return X(a);
      }();
      for (size_t k = 0; k < nk; ++k) {
        const auto M = bz.k_symmetry().value_AO(Xab, k);
        cd* dst = out.data() + ((a * d1 + b) * nk + k) * n * n;
        for (size_t i = 0; i < n; ++i)
          for (size_t j = 0; j < n; ++j) dst[i * n + j] = M(i, j);
      }
    }
  return out;
}

// [lead][nk][n][n] -> the irreducible points of Y ([lead][ink][n][n])
void to_irreducible(const std::vector<cd>& full, const bz_utils_t& bz, size_t lead, size_t n, cd* Y) {
  const size_t nk = bz.nk(), ink = bz.ink(), n2 = n * n;
  for (size_t a = 0; a < lead; ++a)
    for (size_t ik = 0; ik < ink; ++ik) {
      const cd* src = full.data() + (a * nk + bz.k_symmetry().full_point(ik)) * n2;
      std::copy(src, src + n2, Y + (a * ink + ik) * n2);
    }
}

}  // namespace

void custom_kernel_parameters(green::params::params& p) {
  p.define<int>("gb200_device", "CUDA device of the B200 kernel", 0);
  p.define<int>("gb200_split_slices", "INT8 slices per operand for split precision (0: FP64)", 0);
}

std::tuple<std::shared_ptr<void>, gw_callback> custom_gw_kernel(bool X2C, const green::params::params& p, size_t nao,
                                                                size_t nso, size_t ns, size_t NQ,
                                                                const green::grids::transformer_t& ft,
                                                                const bz_utils_t& bz, const ztensor<4>&) {
  if (X2C && bz.ink() != bz.nk())
    throw green::mbpt::mbpt_kernel_error("B200 kernel: two-component input with k-point symmetry is not supported");
  if (p["q0_treatment"].as<std::string>() != "IGNORE_G0")
    throw green::mbpt::mbpt_kernel_error(
        "B200 kernel plug-in: only q0_treatment IGNORE_G0 (the library's gb200_set_q0_correction takes AqQ directly)");
  gb200_dims d{(int32_t)bz.nk(), (int32_t)nao, (int32_t)nso, (int32_t)ns, (int32_t)NQ,
               (int32_t)ft.sd().repn_fermi().nts(), (int32_t)ft.sd().repn_fermi().nw(),
               (int32_t)ft.sd().repn_bose().nw(), p["BETA"].as<double>()};
  auto h = std::make_shared<handle>();
  check(gb200_create(&d, p["gb200_device"].as<int>(), &h->c), nullptr);
  upload_maps(h->c, bz);
  upload_grid(h->c, ft);
  upload_integrals(h->c, p["dfintegral_file"].as<std::string>(), GB200_INTEGRALS_GW, nao, NQ, bz);
  const int S = p["gb200_split_slices"].as<int>();
  check(gb200_set_precision(h->c, S ? GB200_PREC_SPLIT : GB200_PREC_FP64, S ? S : 4), h->c);
  const size_t nts = d.nts;
  // callback (G, Sigma) at the irreducible points: the library zeroes, accumulates and divides
  // Sigma by nk (gw_cpu_kernel.cpp:41,55); node rank 0 computes, the others wait at the fences
  gw_callback cb = [h, &bz, nts, ns, nso](green::utils::shared_object<ztensor<5>>& G,
                                          green::utils::shared_object<ztensor<5>>& Sigma) {
    Sigma.fence();
    if (!green::utils::context().node_rank) {
      const std::vector<cd> Gf = full_zone(G.object(), bz);
      std::vector<cd> Sf(Gf.size());
      check(gb200_gw_sigma(h->c, reinterpret_cast<const double*>(Gf.data()), reinterpret_cast<double*>(Sf.data())),
            h->c);
      to_irreducible(Sf, bz, nts * ns, nso, Sigma.object().data());
    }
    Sigma.fence();
  };
  return {h, cb};
}

std::tuple<std::shared_ptr<void>, hf_callback> custom_hf_kernel(bool X2C, const green::params::params& p, size_t nao,
                                                                size_t nso, size_t ns, size_t NQ, double madelung,
                                                                const bz_utils_t& bz, const ztensor<4>& S_k) {
  if (X2C && bz.ink() != bz.nk())
    throw green::mbpt::mbpt_kernel_error("B200 kernel: two-component input with k-point symmetry is not supported");
  // the HF context needs no imaginary-time grid: any even nts
  gb200_dims d{(int32_t)bz.nk(), (int32_t)nao, (int32_t)nso, (int32_t)ns, (int32_t)NQ, 2, 2, 3, 1.0};
  auto h = std::make_shared<handle>();
  check(gb200_create(&d, p["gb200_device"].as<int>(), &h->c), nullptr);
  upload_maps(h->c, bz);
  upload_integrals(h->c, p["dfintegral_hf_file"].as<std::string>(), GB200_INTEGRALS_HF, nao, NQ, bz);
  auto Sf = std::make_shared<std::vector<cd>>(full_zone(S_k, bz));
  // callback dm -> F at the irreducible points (hf_cpu_kernels.cpp:25-146); dm is already
  // spin_prefactor * G(beta) (hf_solver.cpp:9-16)
  hf_callback cb = [h, Sf, madelung, &bz, ns, nso](const ztensor<4>& dm) {
    const std::vector<cd> dmf = full_zone(dm, bz);
    std::vector<cd> Ff(dmf.size());
    check(gb200_hf_fock(h->c, reinterpret_cast<const double*>(dmf.data()), reinterpret_cast<const double*>(Sf->data()),
                        madelung, reinterpret_cast<double*>(Ff.data())),
          h->c);
    ztensor<4> F(dm.shape());
    to_irreducible(Ff, bz, ns, nso, F.data());
    return F;
  };
  return {h, cb};
}

}  // namespace gb200_green
