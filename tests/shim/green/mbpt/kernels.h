// Test stand-in for <green/mbpt/kernels.h>: the types a custom-kernel plug-in sees (params,
// shared_object, transformer_t, brillouin_zone_utils, ztensor<N>).  Test infrastructure only.
#pragma once
#include <complex>

#include "../grids/transformer_t.h"
#include "../ndarray/ndarray.h"
#include "../params/params.h"
#include "../symmetry/symmetry.h"
#include "../utils/mpi_shared.h"

namespace green::mbpt {
template <typename prec, size_t Dim>
using tensor = green::ndarray::ndarray<prec, Dim>;
template <size_t Dim>
using ztensor = green::ndarray::ndarray<std::complex<double>, Dim>;
}  // namespace green::mbpt
