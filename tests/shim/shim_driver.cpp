// Test driver for the green-mbpt plug-in (green-mbpt_b200/shim): builds the stand-in objects of
// a case directory written by tests/test_shim.py, obtains the kernels from custom_hf_kernel /
// custom_gw_kernel as green-mbpt's kernel factories do, runs one callback and writes its result.
//   shim_driver <dir> hf   -> <dir>/F.bin      (Fock matrix at the irreducible points)
//   shim_driver <dir> gw   -> <dir>/Sigma.bin  (self-energy at the irreducible points)
#include <cstdio>
#include <fstream>
#include <string>

#include "gb200_green_kernel.h"

using namespace green;
using cd = std::complex<double>;

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: shim_driver <dir> hf|gw\n");
    return 2;
  }
  const std::string dir = argv[1], mode = argv[2];
  try {
    std::ifstream f(dir + "/dims.txt");
    size_t nao, nso, ns, NQ;
    double madelung, beta;
    std::string q0;
    f >> nao >> nso >> ns >> NQ >> madelung >> beta >> q0;
    params::params p;
    gb200_green::custom_kernel_parameters(p);
    p.set("BETA", std::to_string(beta));
    p.set("dfintegral_file", dir);
    p.set("dfintegral_hf_file", dir);
    p.set("q0_treatment", q0);
    symmetry::brillouin_zone_utils bz(dir);
    const size_t ink = bz.ink();
    mbpt::ztensor<4> S(ns, ink, nso, nso);
    {
      auto v = stub::load<cd>(dir + "/S_ibz");
      std::copy(v.begin(), v.end(), S.data());
    }
    const bool X2C = nso == 2 * nao;
    if (mode == "hf") {
      auto [kernel, cb] = gb200_green::custom_hf_kernel(X2C, p, nao, nso, ns, NQ, madelung, bz, S);
      mbpt::ztensor<4> dm(ns, ink, nso, nso);
      auto v = stub::load<cd>(dir + "/dm");
      std::copy(v.begin(), v.end(), dm.data());
      mbpt::ztensor<4> F = cb(dm);
      stub::save(dir + "/F", F.data(), F.size());
    } else {
      grids::transformer_t ft(dir);
      const size_t nts = ft.sd().repn_fermi().nts();
      auto [kernel, cb] = gb200_green::custom_gw_kernel(X2C, p, nao, nso, ns, NQ, ft, bz, S);
      utils::shared_object<mbpt::ztensor<5>> G(mbpt::ztensor<5>(nts, ns, ink, nso, nso));
      utils::shared_object<mbpt::ztensor<5>> Sig(mbpt::ztensor<5>(nts, ns, ink, nso, nso));
      auto v = stub::load<cd>(dir + "/G");
      std::copy(v.begin(), v.end(), G.object().data());
      cb(G, Sig);
      stub::save(dir + "/Sigma", Sig.object().data(), Sig.object().size());
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "shim_driver: %s\n", e.what());
    return 1;
  }
  return 0;
}
