// Shared handle type of the oracle/_ref library: the reference's own C++
// potentials and optimisers (compiled unchanged from the reference tree)
// behind a small C interface for ctypes.  Test infrastructure only.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "base_potential.hpp"  // source/fresco/base_potential.hpp

struct RefPotential {
  std::shared_ptr<fresco::BasePotential> p;
};

inline std::vector<double> ref_vec(const double* p, int64_t n) { return std::vector<double>(p, p + n); }
