// NUwNU of the reference (source/fresco/nuwnu.hpp), compiled unchanged.
#include "nuwnu.hpp"
#include "ref_glue.h"

extern "C" void* ref_nuwnu_create(const double* radii, int64_t n, const double* kpts, int64_t nk, const double* sk,
                                  const double* v, const double* L, int ndim, double eps) {
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(new fresco::NUwNU(
      ref_vec(radii, n), ref_vec(kpts, nk * ndim), ref_vec(sk, nk), ref_vec(v, nk), ref_vec(L, ndim), eps))};
}
