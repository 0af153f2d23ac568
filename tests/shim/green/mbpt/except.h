// Test stand-in for green-mbpt's exception classes (except.h).  Test infrastructure only.
#pragma once
#include <stdexcept>

namespace green::mbpt {
struct mbpt_kernel_error : std::runtime_error { using std::runtime_error::runtime_error; };
struct mbpt_wrong_grid : std::runtime_error { using std::runtime_error::runtime_error; };
struct mbpt_chemical_potential_search_failure : std::runtime_error { using std::runtime_error::runtime_error; };
struct mbpt_outdated_input : std::runtime_error { using std::runtime_error::runtime_error; };
}  // namespace green::mbpt
