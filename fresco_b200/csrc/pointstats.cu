// Point-pattern utilities on the device: the hard-core overlap check
// (CheckOverlap*, source/fresco/check_overlap.hpp:24-130 and
// check_overlap_cell_lists.hpp:87-180) and the number-variance window counts
// (PointPatternStatistics, point_pattern_statistics.hpp:36-111; BatchPPS,
// batch_pointstats.hpp:29-150).
//
// Both sort the points into a uniform cell grid (count, scan, scatter) and
// test distances with the reference's arithmetic: r_ij = r1 - r2, minus
// round(r_ij / L) * L per periodic axis (distance.hpp:170-192, ibox = 1 / L),
// squared and summed in axis order with every operation rounded on its own (no
// fused multiply-add), so each comparison (d2 < (r_i + r_j)^2, d2 <= r^2)
// decides as the reference's does.
//
// Window counts: the window centres come from the same std::mt19937_64 and
// std::uniform_real_distribution<double>(0, L) calls as the reference, on the
// host, in the same order; one thread block per window walks the cells of the
// window's bounding box, adds whole cells that lie inside a radius (with a
// slack of 1e-9 of the box above rounding), skips cells outside it, and tests
// the points of the cells the circle crosses one by one.  The integer counts
// are therefore the reference's; the running moments (moments.hpp:28-37) are
// updated on the host in the reference's sample order.
#include <algorithm>
#include <cmath>
#include <random>
#include <string>

#include "common.cuh"
#include "pointstats.cuh"
#include "scan.cuh"

namespace fb {

namespace {

constexpr int kPsThreads = 256;
constexpr int64_t kWindowChunk = 65536;  // windows per launch
constexpr int kMaxRadii = 8192;          // shared-memory difference array per window

struct CellGrid {
  double lo[3] = {0, 0, 0};    // grid origin (0 on periodic axes)
  double L[3] = {1, 1, 1};     // period (periodic) or grid extent (Cartesian)
  double ibox[3] = {1, 1, 1};  // 1 / L, as the reference's distance computes it
  double cw[3] = {1, 1, 1};    // cell width
  double inv_cw[3] = {1, 1, 1};
  int nc[3] = {1, 1, 1};
  int periodic = 1;
};

template <int D>
struct Pt {
  double x[D];
};

// Cell of a coordinate along axis a; a non-finite one goes to cell 0.
__device__ __forceinline__ int axis_cell(double v, const CellGrid& g, int a) {
  double u = v - g.lo[a];
  if (g.periodic) u = u - floor(u * g.ibox[a]) * g.L[a];
  const double t = u * g.inv_cw[a];
  return t >= 0.0 ? (t < double(g.nc[a]) ? int(t) : g.nc[a] - 1) : 0;
}

template <int D>
__device__ __forceinline__ int cell_index(const double* p, const CellGrid& g) {
  int cell = 0, stride = 1;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    cell += axis_cell(p[a], g, a) * stride;
    stride *= g.nc[a];
  }
  return cell;
}

// |r1 - r2|^2 with the reference's rounding (periodic_distance::get_rij, then
// std::inner_product / dot from 0).
template <int D>
__device__ __forceinline__ double dist2(const double* r1, const double* r2, const CellGrid& g) {
  double s = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    double d = __dsub_rn(r1[a], r2[a]);
    if (g.periodic) d = __dsub_rn(d, __dmul_rn(rint(__dmul_rn(d, g.ibox[a])), g.L[a]));
    s = __dadd_rn(s, __dmul_rn(d, d));
  }
  return s;
}

template <int D>
__global__ void __launch_bounds__(kPsThreads) ps_count_kernel(const double* __restrict__ x, int64_t N, CellGrid g,
                                                              int* cell_count, uint32_t* rank) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    double p[D];
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = x[j * D + a];
    rank[j] = uint32_t(atomicAdd(&cell_count[cell_index<D>(p, g)], 1));
  }
}

template <int D>
__global__ void __launch_bounds__(kPsThreads) ps_scatter_kernel(const double* __restrict__ x, int64_t N, CellGrid g,
                                                                const uint32_t* __restrict__ rank,
                                                                const int* __restrict__ cell_start, Pt<D>* xs,
                                                                uint32_t* ids) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    Pt<D> p;
#pragma unroll
    for (int a = 0; a < D; ++a) p.x[a] = x[j * D + a];
    const int64_t pos = int64_t(cell_start[cell_index<D>(p.x, g)]) + rank[j];
    xs[pos] = p;
    ids[pos] = uint32_t(j);
  }
}

// Neighbour cell offsets along an axis: {-1, 0, 1}, or the distinct cells when
// a periodic axis has fewer than three; Cartesian axes drop cells off the grid.
__device__ __forceinline__ int axis_offsets(const CellGrid& g, int a, int c, int* out) {
  const int nc = g.nc[a];
  int n = 0;
  if (g.periodic) {
    if (nc == 1) {
      out[n++] = 0;
    } else if (nc == 2) {
      out[n++] = c;
      out[n++] = 1 - c;
    } else {
      out[n++] = (c + nc - 1) % nc;
      out[n++] = c;
      out[n++] = (c + 1) % nc;
    }
  } else {
    for (int o = -1; o <= 1; ++o)
      if (c + o >= 0 && c + o < nc) out[n++] = c + o;
  }
  return n;
}

// Visits the records of the cells around position p: f(q) for each record q.
// Returns early when f returns true.
template <int D, class F>
__device__ __forceinline__ bool for_neighbours(const double* p, const CellGrid& g, const int* __restrict__ cell_start,
                                               F f) {
  int cells[3][3], nn[3] = {1, 1, 1};
#pragma unroll
  for (int a = 0; a < D; ++a) nn[a] = axis_offsets(g, a, axis_cell(p[a], g, a), cells[a]);
  for (int i2 = 0; i2 < (D > 2 ? nn[2] : 1); ++i2)
    for (int i1 = 0; i1 < (D > 1 ? nn[1] : 1); ++i1)
      for (int i0 = 0; i0 < nn[0]; ++i0) {
        int cell = cells[0][i0];
        if (D > 1) cell += cells[1][i1] * g.nc[0];
        if (D > 2) cell += cells[2][i2] * g.nc[0] * g.nc[1];
        const int end = cell_start[cell + 1];
        for (int q = cell_start[cell]; q < end; ++q)
          if (f(q)) return true;
      }
  return false;
}

// Every point: is any other point closer than the sum of the radii?  The
// relation is symmetric, so flagging the point itself covers both members of
// each pair (check_overlap.hpp:84-97 inserts i and j).
template <int D>
__global__ void __launch_bounds__(kPsThreads) overlap_all_kernel(const Pt<D>* __restrict__ xs,
                                                                 const uint32_t* __restrict__ ids,
                                                                 const double* __restrict__ radii,
                                                                 const int* __restrict__ cell_start, int64_t N,
                                                                 CellGrid g, uint8_t* flags) {
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < N; p += int64_t(gridDim.x) * blockDim.x) {
    const Pt<D> pi = xs[p];
    const double ri = radii[ids[p]];
    const bool hit = for_neighbours<D>(pi.x, g, cell_start, [&](int q) {
      if (q == p) return false;
      const Pt<D> pj = xs[q];
      const double s = __dadd_rn(ri, radii[ids[q]]);
      return dist2<D>(pi.x, pj.x, g) < __dmul_rn(s, s);
    });
    if (hit) flags[ids[p]] = 1;
  }
}

// Changed atoms only (check_overlap.hpp:66-82): every pair (i changed, j != i)
// closer than r_i + r_j flags both.
template <int D>
__global__ void __launch_bounds__(kPsThreads) overlap_changed_kernel(const double* __restrict__ x,
                                                                     const int64_t* __restrict__ changed, int64_t nc,
                                                                     const Pt<D>* __restrict__ xs,
                                                                     const uint32_t* __restrict__ ids,
                                                                     const double* __restrict__ radii,
                                                                     const int* __restrict__ cell_start, CellGrid g,
                                                                     uint8_t* flags) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < nc; k += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = changed[k];
    double pi[D];
#pragma unroll
    for (int a = 0; a < D; ++a) pi[a] = x[i * D + a];
    const double ri = radii[i];
    for_neighbours<D>(pi, g, cell_start, [&](int q) {
      const uint32_t j = ids[q];
      if (int64_t(j) == i) return false;
      const Pt<D> pj = xs[q];
      const double s = __dadd_rn(ri, radii[j]);
      if (dist2<D>(pi, pj.x, g) < __dmul_rn(s, s)) {
        flags[i] = 1;
        flags[j] = 1;
      }
      return false;
    });
  }
}

// One block per window: counts[w * R + i] = number of points with
// |centre - x|^2 <= r2[i] (r2 ascending).  Per cell of the window's bounding
// box, the radii split into three ranges: [0, ilo) miss the cell, [ihi, R)
// hold all of it, [ilo, ihi) cross it, and those test each point.  Contributions
// go into a shared difference array over the radius index (a point inside
// radius i is inside every larger one), summed at the end.
template <int D>
__global__ void __launch_bounds__(kPsThreads) window_count_kernel(const Pt<D>* __restrict__ xs,
                                                                  const int* __restrict__ cell_start, CellGrid g,
                                                                  int local, double slack,
                                                                  const double* __restrict__ centres,
                                                                  const double* __restrict__ r2,
                                                                  const double* __restrict__ rr, int R, int* counts) {
  extern __shared__ int diff[];  // R + 1
  for (int i = threadIdx.x; i <= R; i += blockDim.x) diff[i] = 0;
  __syncthreads();
  double c[D], cu[D];
  int kmin[D], span[D];
  int64_t total = 1;
  const double rmax = rr[R - 1];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    c[a] = centres[int64_t(blockIdx.x) * D + a];
    cu[a] = c[a] - floor(c[a] * g.ibox[a]) * g.L[a];  // wrapped into [0, L)
    if (local) {
      kmin[a] = int(floor((cu[a] - rmax - slack) * g.inv_cw[a]));
      span[a] = int(floor((cu[a] + rmax + slack) * g.inv_cw[a])) - kmin[a] + 1;
      if (span[a] > g.nc[a]) local = 0;
    }
  }
#pragma unroll
  for (int a = 0; a < D; ++a) {
    if (!local) {
      kmin[a] = 0;
      span[a] = g.nc[a];
    }
    total *= span[a];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int64_t t = warp; t < total; t += nwarps) {
    int64_t rem = t;
    int cell = 0, stride = 1;
    double dmin2 = 0.0, dmax2 = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int k = kmin[a] + int(rem % span[a]);
      rem /= span[a];
      const int kw = ((k % g.nc[a]) + g.nc[a]) % g.nc[a];
      cell += kw * stride;
      stride *= g.nc[a];
      // faces of the cell relative to the centre, unwrapped (valid when local)
      const double lo = k * g.cw[a] - cu[a], hi = (k + 1) * g.cw[a] - cu[a];
      const double nearest = lo > 0.0 ? lo : (hi < 0.0 ? -hi : 0.0);
      const double farthest = fmax(fabs(lo), fabs(hi));
      dmin2 += nearest * nearest;
      dmax2 += farthest * farthest;
    }
    int ilo = 0, ihi = R;
    if (local) {
      const double dmin = sqrt(dmin2), dmax = sqrt(dmax2);
      int lo = 0, hi = R;  // first radius with dmax + slack < rr
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (dmax + slack < rr[m]) hi = m;
        else lo = m + 1;
      }
      ihi = lo;
      lo = 0;
      hi = ihi;  // first radius with dmin - slack <= rr (the cell may hold points within it)
      while (lo < hi) {
        const int m = (lo + hi) >> 1;
        if (dmin - slack <= rr[m]) hi = m;
        else lo = m + 1;
      }
      ilo = lo;
    }
    const int beg = cell_start[cell], end = cell_start[cell + 1];
    if (lane == 0 && ihi < R && end > beg) atomicAdd(&diff[ihi], end - beg);
    if (ilo < ihi) {
      for (int q = beg + lane; q < end; q += 32) {
        const Pt<D> p = xs[q];
        const double d2 = dist2<D>(c, p.x, g);  // get_rij(dr, centre, x_i)
        int lo = ilo, hi = ihi;
        while (lo < hi) {
          const int m = (lo + hi) >> 1;
          if (d2 <= r2[m]) hi = m;
          else lo = m + 1;
        }
        if (lo < ihi) {
          atomicAdd(&diff[lo], 1);
          if (ihi < R) atomicAdd(&diff[ihi], -1);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < R; ++i) {
      acc += diff[i];
      counts[int64_t(blockIdx.x) * R + i] = acc;
    }
  }
}

int launch_grid(int64_t n) { return int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, kPsThreads), sm_count() * 8LL))); }

// Uniform cell grid of about one cell per point at most, cells at least
// min_width wide (0: as many as that allows).
CellGrid make_grid(int D, const double* lo, const double* extent, bool periodic, double min_width, int64_t N,
                   double cells_per_point) {
  CellGrid g;
  g.periodic = periodic ? 1 : 0;
  const double cap = std::max(1.0, std::floor(std::pow(std::max(1.0, double(N) * cells_per_point), 1.0 / D)));
  for (int a = 0; a < D; ++a) {
    g.lo[a] = lo[a];
    g.L[a] = extent[a];
    g.ibox[a] = 1.0 / extent[a];
    double nc = min_width > 0.0 ? std::floor(extent[a] / (min_width * (1.0 + 1e-9))) : cap;
    nc = std::max(1.0, std::min(nc, cap));
    g.nc[a] = int(nc);
    g.cw[a] = extent[a] / g.nc[a];
    g.inv_cw[a] = g.nc[a] / extent[a];
  }
  return g;
}

// Cell sort of N device points on stream s into xs / ids / cell_start.
template <int D>
struct CellSort {
  DevBuf<int> count, start, tmp;
  DevBuf<uint32_t> rank, ids;
  DevBuf<Pt<D>> xs;
  int64_t ncells = 0;

  void sort(const double* x, int64_t N, const CellGrid& g, cudaStream_t s) {
    int64_t nc = 1;
    for (int a = 0; a < D; ++a) nc *= g.nc[a];
    if (nc + 1 > int64_t(count.n)) {
      count.alloc(nc + 1);
      start.alloc(nc + 1);
      tmp.alloc(scan_tmp_size(nc + 1));
    }
    if (N > int64_t(rank.n)) {
      rank.alloc(N);
      ids.alloc(N);
      xs.alloc(N);
    }
    ncells = nc;
    FB_CUDA(cudaMemsetAsync(count.p, 0, sizeof(int) * (nc + 1), s));
    if (N > 0) {
      ps_count_kernel<D><<<launch_grid(N), kPsThreads, 0, s>>>(x, N, g, count.p, rank.p);
      FB_LAUNCH_CHECK();
    }
    exclusive_scan(count.p, start.p, tmp.p, nc + 1, s);
    if (N > 0) {
      ps_scatter_kernel<D><<<launch_grid(N), kPsThreads, 0, s>>>(x, N, g, rank.p, start.p, xs.p, ids.p);
      FB_LAUNCH_CHECK();
    }
  }
};

template <int D>
class OverlapCheckImpl final : public OverlapCheck {
 public:
  OverlapCheckImpl(const std::vector<double>& radii, const std::vector<double>& boxv, bool periodic)
      : N_(int64_t(radii.size())), periodic_(periodic), box_(boxv) {
    if (radii.empty()) throw std::runtime_error("CheckOverlap: illegal input: radii");
    if (N_ >= (int64_t(1) << 31)) throw InvalidArgument("CheckOverlap: more than 2^31 - 1 particles");
    if (periodic)
      for (double L : boxv)
        if (!(L > 0.0) || !std::isfinite(L)) throw InvalidArgument("CheckOverlap: box lengths must be positive");
    rcut_ = 2.0 * *std::max_element(radii.begin(), radii.end());
    FB_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    radii_.alloc(N_);
    x_.alloc(N_ * D);
    flags_.alloc(N_);
    FB_CUDA(cudaMemcpy(radii_.p, radii.data(), sizeof(double) * N_, cudaMemcpyHostToDevice));
    host_flags_.resize(N_);
  }
  ~OverlapCheckImpl() override {
    if (s_) {
      cudaStreamSynchronize(s_);
      cudaStreamDestroy(s_);
    }
  }

  int64_t natoms() const override { return N_; }

  int64_t find(const double* x, int64_t ndof, const int64_t* changed, int64_t n_changed, uint64_t* out) override {
    if (ndof % D) throw std::runtime_error("CheckOverlap::conf_test: illegal input");
    if (ndof / D != N_) throw std::runtime_error("CheckOverlap::conf_test: illegal input");
    for (int64_t k = 0; k < n_changed; ++k)
      if (changed[k] < 0 || changed[k] >= N_) throw InvalidArgument("CheckOverlap: changed atom index out of range");
    double lo[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    if (periodic_) {
      for (int a = 0; a < D; ++a) ext[a] = box_[a];
    } else {  // the grid spans the points' bounding box
      for (int a = 0; a < D; ++a) {
        double mn = INFINITY, mx = -INFINITY;
        for (int64_t j = 0; j < N_; ++j) {
          const double v = x[j * D + a];
          if (std::isfinite(v)) {
            mn = std::min(mn, v);
            mx = std::max(mx, v);
          }
        }
        if (!(mn <= mx)) mn = mx = 0.0;
        const double w = (mx - mn) * (1.0 + 1e-9) + 1e-300 + 1e-12 * std::max(std::fabs(mn), std::fabs(mx));
        lo[a] = mn;
        ext[a] = std::max(w, 1e-300);
      }
    }
    const CellGrid g = make_grid(D, lo, ext, periodic_, rcut_, N_, 1.0);
    FB_CUDA(cudaMemcpyAsync(x_.p, x, sizeof(double) * N_ * D, cudaMemcpyHostToDevice, s_));
    cells_.sort(x_.p, N_, g, s_);
    FB_CUDA(cudaMemsetAsync(flags_.p, 0, N_, s_));
    if (changed && n_changed > 0) {
      if (n_changed > int64_t(changed_.n)) changed_.alloc(n_changed);
      FB_CUDA(cudaMemcpyAsync(changed_.p, changed, sizeof(int64_t) * n_changed, cudaMemcpyHostToDevice, s_));
      overlap_changed_kernel<D><<<launch_grid(n_changed), kPsThreads, 0, s_>>>(
          x_.p, changed_.p, n_changed, cells_.xs.p, cells_.ids.p, radii_.p, cells_.start.p, g, flags_.p);
    } else {
      overlap_all_kernel<D><<<launch_grid(N_), kPsThreads, 0, s_>>>(cells_.xs.p, cells_.ids.p, radii_.p,
                                                                     cells_.start.p, N_, g, flags_.p);
    }
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaMemcpyAsync(host_flags_.data(), flags_.p, N_, cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    int64_t n = 0;
    for (int64_t j = 0; j < N_; ++j)
      if (host_flags_[j]) out[n++] = uint64_t(j);
    return n;
  }

 private:
  int64_t N_;
  bool periodic_;
  std::vector<double> box_;
  double rcut_ = 0.0;
  cudaStream_t s_ = nullptr;
  DevBuf<double> radii_, x_;
  DevBuf<uint8_t> flags_;
  DevBuf<int64_t> changed_;
  CellSort<D> cells_;
  std::vector<uint8_t> host_flags_;
};

// Running mean of n and n^2 (moments.hpp:28-37), in the reference's
// expression order.
struct Moments {
  double mean = 0.0, mean2 = 0.0;
  uint64_t count = 0;
  void update(double v) {
    mean = (mean * double(count) + v) / double(count + 1);
    mean2 = (mean2 * double(count) + v * v) / double(count + 1);
    ++count;
  }
};

template <int D>
class WindowCountsImpl final : public WindowCounts {
 public:
  WindowCountsImpl(const double* x, int64_t N, const std::vector<double>& boxv, const std::vector<double>& radii,
                   uint64_t seed)
      : N_(N), box_(boxv), seed_(seed), gen_(seed), mom_(radii.size()) {
    const int R = int(radii.size());
    if (R < 1) throw InvalidArgument("at least one window radius is needed");
    if (R > kMaxRadii) throw InvalidArgument("at most " + std::to_string(kMaxRadii) + " window radii");
    if (N < 0 || N >= (int64_t(1) << 31)) throw InvalidArgument("the number of points must be below 2^31");
    for (double L : boxv)
      if (!(L > 0.0) || !std::isfinite(L)) throw InvalidArgument("box lengths must be positive");
    std::vector<double> r2(R), rr(R);
    for (int i = 0; i < R; ++i) {
      r2[i] = radii[i] * radii[i];  // batch_pointstats.hpp:50-52, point_pattern_statistics.hpp:79
      if (!std::isfinite(r2[i])) throw InvalidArgument("window radii must be finite");
      if (i && r2[i] < r2[i - 1])
        throw InvalidArgument("window radii must be in ascending order (batch_pointstats.hpp:85-109 assumes it)");
      rr[i] = std::sqrt(r2[i]);
    }
    double lo[3] = {0, 0, 0}, ext[3];
    double Lmax = 0.0;
    for (int a = 0; a < D; ++a) {
      ext[a] = box_[a];
      Lmax = std::max(Lmax, box_[a]);
    }
    slack_ = 1e-9 * Lmax;
    // cells of a quarter of the largest radius, at most about four per point
    g_ = make_grid(D, lo, ext, true, rr[R - 1] / 4.0, N_, 4.0);
    local_ = 1;
    for (int a = 0; a < D; ++a)
      if (!(rr[R - 1] + g_.cw[a] + slack_ < 0.5 * box_[a])) local_ = 0;
    FB_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    r2_.alloc(R);
    rr_.alloc(R);
    FB_CUDA(cudaMemcpy(r2_.p, r2.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
    FB_CUDA(cudaMemcpy(rr_.p, rr.data(), sizeof(double) * R, cudaMemcpyHostToDevice));
    DevBuf<double> xd(std::max<int64_t>(N_ * D, 1));
    if (N_) FB_CUDA(cudaMemcpy(xd.p, x, sizeof(double) * N_ * D, cudaMemcpyHostToDevice));
    cells_.sort(xd.p, N_, g_, s_);
    FB_CUDA(cudaStreamSynchronize(s_));
  }
  ~WindowCountsImpl() override {
    if (s_) {
      cudaStreamSynchronize(s_);
      cudaStreamDestroy(s_);
    }
  }

  int nradii() const override { return int(mom_.size()); }
  uint64_t seed() const override { return seed_; }
  void set_seed(uint64_t s) override {
    seed_ = s;
    gen_.seed(s);
  }

  void run(int64_t n) override {
    const int R = nradii();
    while (n > 0) {
      const int64_t w = std::min(n, kWindowChunk);
      // point_pattern_statistics.hpp:72-77 / batch_pointstats.hpp:76-80
      hc_.resize(w * D);
      for (int64_t k = 0; k < w; ++k)
        for (int a = 0; a < D; ++a) {
          std::uniform_real_distribution<double> real_dist(0, box_[a]);
          hc_[k * D + a] = real_dist(gen_) - box_[a] / 2;
        }
      if (int64_t(centres_.n) < w * D) {
        centres_.alloc(kWindowChunk * D);
        counts_.alloc(kWindowChunk * int64_t(R));
      }
      FB_CUDA(cudaMemcpyAsync(centres_.p, hc_.data(), sizeof(double) * w * D, cudaMemcpyHostToDevice, s_));
      window_count_kernel<D><<<int(w), kPsThreads, sizeof(int) * (R + 1), s_>>>(
          cells_.xs.p, cells_.start.p, g_, local_, slack_, centres_.p, r2_.p, rr_.p, R, counts_.p);
      FB_LAUNCH_CHECK();
      hcount_.resize(w * R);
      FB_CUDA(cudaMemcpyAsync(hcount_.data(), counts_.p, sizeof(int) * w * R, cudaMemcpyDeviceToHost, s_));
      FB_CUDA(cudaStreamSynchronize(s_));
      for (int64_t k = 0; k < w; ++k)
        for (int i = 0; i < R; ++i) mom_[i].update(double(hcount_[k * R + i]));
      n -= w;
    }
  }

  void moments(double* mean, double* var, uint64_t* count) const override {
    for (size_t i = 0; i < mom_.size(); ++i) {
      if (mean) mean[i] = mom_[i].mean;
      if (var) var[i] = mom_[i].mean2 - mom_[i].mean * mom_[i].mean;
      if (count) count[i] = mom_[i].count;
    }
  }

 private:
  int64_t N_;
  std::vector<double> box_;
  uint64_t seed_;
  std::mt19937_64 gen_;
  std::vector<Moments> mom_;
  CellGrid g_;
  int local_ = 0;
  double slack_ = 0.0;
  cudaStream_t s_ = nullptr;
  DevBuf<double> r2_, rr_, centres_;
  DevBuf<int> counts_;
  CellSort<D> cells_;
  std::vector<double> hc_;
  std::vector<int> hcount_;
};

}  // namespace

std::unique_ptr<OverlapCheck> make_overlap_check(const std::vector<double>& radii, const std::vector<double>& boxv,
                                                 bool periodic) {
  const int D = int(boxv.size());
  if (D == 1) return std::unique_ptr<OverlapCheck>(new OverlapCheckImpl<1>(radii, boxv, periodic));
  if (D == 2) return std::unique_ptr<OverlapCheck>(new OverlapCheckImpl<2>(radii, boxv, periodic));
  if (D == 3) return std::unique_ptr<OverlapCheck>(new OverlapCheckImpl<3>(radii, boxv, periodic));
  throw std::runtime_error("CheckOverlap: dimension " + std::to_string(D) + " is not supported on the device");
}

std::unique_ptr<WindowCounts> make_window_counts(const double* x, int64_t n_points, const std::vector<double>& boxv,
                                                 const std::vector<double>& radii, uint64_t seed) {
  const int D = int(boxv.size());
  if (D == 1) return std::unique_ptr<WindowCounts>(new WindowCountsImpl<1>(x, n_points, boxv, radii, seed));
  if (D == 2) return std::unique_ptr<WindowCounts>(new WindowCountsImpl<2>(x, n_points, boxv, radii, seed));
  if (D == 3) return std::unique_ptr<WindowCounts>(new WindowCountsImpl<3>(x, n_points, boxv, radii, seed));
  throw std::runtime_error("point pattern statistics: dimension " + std::to_string(D) +
                           " is not supported on the device");
}

}  // namespace fb
