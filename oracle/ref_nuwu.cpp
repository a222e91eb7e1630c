// NUwU of the reference (source/fresco/nuwu.hpp), compiled unchanged.
#include "nuwu.hpp"
#include "ref_glue.h"

extern "C" void* ref_nuwu_create(const double* radii, int64_t n, double K, const double* sk, const double* v,
                                 int64_t nsk, const double* L, int ndim, double eps) {
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(
      new fresco::NUwU(ref_vec(radii, n), K, ref_vec(sk, nsk), ref_vec(v, nsk), ref_vec(L, ndim), eps))};
}
