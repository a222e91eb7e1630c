// UwU of the reference (source/fresco/uwu.hpp), compiled unchanged.
#include "uwu.hpp"
#include "ref_glue.h"

extern "C" void* ref_uwu_create(const int* grid, int ndim, double K, const double* sk, const double* v, int64_t nsk,
                                const double* L, double eps) {
  std::vector<int> g(grid, grid + ndim);
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(
      new fresco::UwU(g, K, ref_vec(sk, nsk), ref_vec(v, nsk), ref_vec(L, ndim), eps))};
}
