// Point-pattern utilities on the device: the hard-core overlap check
// (fresco.distances.CheckOverlap: source/fresco/check_overlap.hpp:24-130,
// check_overlap_cell_lists.hpp:87-180) and the number-variance window counts
// (fresco.utils.PointPatternStatistics: point_pattern_statistics.hpp:36-111;
// fresco.utils.BatchPPS: batch_pointstats.hpp:29-150).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

namespace fb {

class OverlapCheck {
 public:
  virtual ~OverlapCheck() = default;
  // Indices, ascending, of the particles whose hard cores (radius r_i) overlap
  // another one: |r_ij|^2 < (r_i + r_j)^2.  With changed atoms, only the pairs
  // that hold a changed atom count (get_overlapping_particles_ca).  x: host
  // coordinates (ndof = N * ndim); out: room for N indices.  Returns the count.
  virtual int64_t find(const double* x, int64_t ndof, const int64_t* changed, int64_t n_changed, uint64_t* out) = 0;
  virtual int64_t natoms() const = 0;
};

// periodic: minimum-image distances in the box boxv; otherwise Cartesian
// (boxv only gives the dimension).  ndim 1, 2 or 3.
std::unique_ptr<OverlapCheck> make_overlap_check(const std::vector<double>& radii, const std::vector<double>& boxv,
                                                 bool periodic);

class WindowCounts {
 public:
  virtual ~WindowCounts() = default;
  // n more windows: centres drawn from the std::mt19937_64 stream, and for each
  // radius the running moments of the number of points within it.
  virtual void run(int64_t n) = 0;
  virtual void set_seed(uint64_t seed) = 0;
  virtual uint64_t seed() const = 0;
  virtual int nradii() const = 0;
  // mean, variance (E[n^2] - E[n]^2) and sample count per radius
  virtual void moments(double* mean, double* var, uint64_t* count) const = 0;
};

// x: n_points * ndim host coordinates; radii ascending (one for
// PointPatternStatistics, several for BatchPPS).
std::unique_ptr<WindowCounts> make_window_counts(const double* x, int64_t n_points, const std::vector<double>& boxv,
                                                 const std::vector<double>& radii, uint64_t seed);

}  // namespace fb
