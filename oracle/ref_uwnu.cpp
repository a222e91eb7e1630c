// UwNU of the reference (source/fresco/uwnu.hpp), compiled unchanged.  Its
// get_energy prints every |rho(k)| (uwnu.hpp:301); callers use the gradient.
#include "uwnu.hpp"
#include "ref_glue.h"

extern "C" void* ref_uwnu_create(const int* grid, int ndim, const double* kpts, int64_t nk, const double* sk,
                                 const double* v, const double* L, double eps) {
  std::vector<int> g(grid, grid + ndim);
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(
      new fresco::UwNU(g, ref_vec(kpts, nk * ndim), ref_vec(sk, nk), ref_vec(v, nk), ref_vec(L, ndim), eps))};
}
