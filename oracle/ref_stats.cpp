// Reference point-pattern statistics (source/fresco/point_pattern_statistics.hpp)
// and overlap checks (check_overlap.hpp, check_overlap_cell_lists.hpp),
// compiled unchanged.  This file is built without OpenMP: the reference's
// window count adds to one shared counter inside `omp parallel for`
// (point_pattern_statistics.hpp:82-89), a race that a serial build removes.
// Built with -ffp-contract=off, so products and sums round one by one.
#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "fresco/check_overlap.hpp"
#include "fresco/check_overlap_cell_lists.hpp"
#include "fresco/point_pattern_statistics.hpp"

namespace {

struct RefPPS {
  int ndim = 0;
  std::unique_ptr<fresco::PointPatternStatistics<1>> p1;
  std::unique_ptr<fresco::PointPatternStatistics<2>> p2;
  std::unique_ptr<fresco::PointPatternStatistics<3>> p3;
};

template <class T>
std::vector<size_t> overlap_of(T& chk, const std::vector<double>& x, std::vector<long>* changed) {
  if (changed && !changed->empty()) return chk.get_overlapping_particles_ca(x, *changed);
  return chk.get_overlapping_particles(x);
}

template <size_t D>
std::vector<size_t> overlap_dim(const std::vector<double>& r, const std::vector<double>& b, int periodic,
                                int cell_lists, double scale, const std::vector<double>& x,
                                std::vector<long>* changed) {
  if (periodic && cell_lists) {
    fresco::CheckOverlapPeriodicCellLists<D> c(r, b, scale);
    return overlap_of(c, x, changed);
  }
  if (periodic) {
    fresco::CheckOverlapPeriodic<D> c(r, b);
    return overlap_of(c, x, changed);
  }
  fresco::CheckOverlapCartesian<D> c(r);
  return overlap_of(c, x, changed);
}

}  // namespace

extern "C" {

void* ref_pps_create(const double* x, int64_t n_points, int ndim, const double* boxv, double radius, uint64_t seed) {
  std::vector<double> c(x, x + n_points * ndim), b(boxv, boxv + ndim);
  auto* h = new RefPPS;
  h->ndim = ndim;
  if (ndim == 1) h->p1.reset(new fresco::PointPatternStatistics<1>(c, b, radius, seed));
  else if (ndim == 2) h->p2.reset(new fresco::PointPatternStatistics<2>(c, b, radius, seed));
  else if (ndim == 3) h->p3.reset(new fresco::PointPatternStatistics<3>(c, b, radius, seed));
  else {
    delete h;
    return nullptr;
  }
  return h;
}

void ref_pps_run(void* hp, int64_t n) {
  auto* h = static_cast<RefPPS*>(hp);
  if (h->p1) h->p1->run(n);
  if (h->p2) h->p2->run(n);
  if (h->p3) h->p3->run(n);
}

void ref_pps_set_seed(void* hp, uint64_t seed) {
  auto* h = static_cast<RefPPS*>(hp);
  if (h->p1) h->p1->set_generator_seed(seed);
  if (h->p2) h->p2->set_generator_seed(seed);
  if (h->p3) h->p3->set_generator_seed(seed);
}

void ref_pps_get(void* hp, double* mean, double* var, uint64_t* count) {
  auto* h = static_cast<RefPPS*>(hp);
  if (h->p1) *mean = h->p1->get_mean(), *var = h->p1->get_variance(), *count = h->p1->get_count();
  if (h->p2) *mean = h->p2->get_mean(), *var = h->p2->get_variance(), *count = h->p2->get_count();
  if (h->p3) *mean = h->p3->get_mean(), *var = h->p3->get_variance(), *count = h->p3->get_count();
}

void ref_pps_destroy(void* hp) { delete static_cast<RefPPS*>(hp); }

// Sorted overlapping indices into out (room for n); returns their number, or
// -1 when the reference raised (its message in ref_last_error()).
static std::string g_ref_error;
const char* ref_last_error(void) { return g_ref_error.c_str(); }

int64_t ref_overlap(const double* radii, int64_t n, const double* boxv, int ndim, int periodic, int cell_lists,
                    double ncellx_scale, const double* x, const int64_t* changed, int64_t n_changed, uint64_t* out) {
  std::vector<double> r(radii, radii + n), b(boxv, boxv + ndim), c(x, x + n * ndim);
  std::vector<long> ch(changed, changed + n_changed);
  std::vector<size_t> v;
  try {
    if (ndim == 1) v = overlap_dim<1>(r, b, periodic, cell_lists, ncellx_scale, c, &ch);
    else if (ndim == 2) v = overlap_dim<2>(r, b, periodic, cell_lists, ncellx_scale, c, &ch);
    else if (ndim == 3) v = overlap_dim<3>(r, b, periodic, cell_lists, ncellx_scale, c, &ch);
  } catch (const std::exception& e) {
    g_ref_error = e.what();
    return -1;
  }
  std::sort(v.begin(), v.end());
  for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
  return int64_t(v.size());
}

}  // extern "C"
