// Potential families not yet built on the device.
#include <stdexcept>

#include "potential.cuh"

namespace fb {

PotentialPtr make_uwnu(const std::vector<int>&, const std::vector<double>&, const std::vector<double>&,
                       const std::vector<double>&, const std::vector<double>&, double, int) {
  throw std::runtime_error("UwNU is not available in this build");
}
PotentialPtr make_nuwnu(const std::vector<double>&, const std::vector<double>&, const std::vector<double>&,
                        const std::vector<double>&, const std::vector<double>&, double, int) {
  throw std::runtime_error("NUwNU is not available in this build");
}
}  // namespace fb
