// green-mbpt custom-kernel plug-in for the B200 library (libgb200.so, include/gb200.h).
//
// A plug-in provides a header, an enum value appended to kernel_type, a namespace with three
// functions and a library to link (cmake/AddGreenKernel.cmake:1-24, custom_kernels.h:24-38,
// common_defs.h:139-180).  green-mbpt's kernel factories call
//   custom_gw_kernel(X2C, p, nao, nso, ns, NQ, ft, bz_utils, S_k)   (kernel_factory.h:86-108)
//   custom_hf_kernel(X2C, p, nao, nso, ns, NQ, madelung, bz_utils, S_k)   (kernel_factory.h:28-36,42-69)
// and keep the returned handle alive next to the callback, exactly as for the CPU kernels.
#pragma once

#include <functional>
#include <memory>
#include <tuple>

#include <green/mbpt/kernels.h>

namespace gb200_green {

using gw_callback = std::function<void(green::utils::shared_object<green::mbpt::ztensor<5>>&,
                                       green::utils::shared_object<green::mbpt::ztensor<5>>&)>;
using hf_callback = std::function<green::mbpt::ztensor<4>(const green::mbpt::ztensor<4>&)>;

void custom_kernel_parameters(green::params::params& p);

std::tuple<std::shared_ptr<void>, gw_callback> custom_gw_kernel(bool X2C, const green::params::params& p, size_t nao,
                                                                size_t nso, size_t ns, size_t NQ,
                                                                const green::grids::transformer_t& ft,
                                                                const green::symmetry::brillouin_zone_utils& bz,
                                                                const green::mbpt::ztensor<4>& S_k);

std::tuple<std::shared_ptr<void>, hf_callback> custom_hf_kernel(bool X2C, const green::params::params& p, size_t nao,
                                                                size_t nso, size_t ns, size_t NQ, double madelung,
                                                                const green::symmetry::brillouin_zone_utils& bz,
                                                                const green::mbpt::ztensor<4>& S_k);

}  // namespace gb200_green
