// Soft-sphere repulsion E = sum_{pairs, r < d_ij} eps/a (1 - r/d_ij)^a,
// d_ij = r_i + r_j: the device counterpart of InversePowerPeriodicCellLists /
// InversePowerPeriodic / InversePowerCartesian
// (source/fresco/inversepower_potential.hpp:18-124).
//
// Periodic boxes with at least 3 cells per dimension use a cell list built by
// a counting sort (cell edge >= r_cut = 2 max(r_i), inversepower_potential.
// hpp:115) into packed 32-byte point records, then one thread per
// (cell-sorted) point gathers its neighbours from the 3^d surrounding cells;
// the three cells of a row along x are one contiguous range of records.  No
// atomics on the gradient, and each pair's energy is counted once (by its
// lower original index), as in EnergyGradientAccumulator::insert_atom_pair
// (cell_list_potential.hpp:154-181).  Smaller periodic boxes and the Cartesian distance use a tiled
// all-pairs kernel.  Distances follow periodic_distance::get_rij
// (distance.hpp:179-185): dr = x_i - x_j, dr -= round(dr / L) L.
#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

#include "potential.cuh"
#include "scan.cuh"

namespace fb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double pair_energy_gradient(double r2, double dsum, double a, double eps, double* gij) {
  if (r2 >= dsum * dsum) {
    *gij = 0.0;
    return 0.0;
  }
  // inversepower_potential.hpp:52-55
  const double r = sqrt(r2);
  const double base = 1.0 - r / dsum;
  const double factor = (a == 2.0 ? base * base : pow(base, a)) * eps;
  *gij = -factor / ((r - dsum) * r);
  return factor / a;
}

__device__ __forceinline__ double min_image(double d, double L, double invL, bool periodic) {
  // round_fast rounds half to even (distance.hpp:32-36); rint does the same
  return periodic ? d - rint(d * invL) * L : d;
}

struct Box {
  double L[3] = {1, 1, 1};
  double invL[3] = {1, 1, 1};
  int nc[3] = {1, 1, 1};
  double cw[3] = {1, 1, 1};     // cell width
  double inv_cw[3] = {1, 1, 1};
  float Lf[3] = {1, 1, 1}, invLf[3] = {1, 1, 1};
  float reject2 = 0.f;  // squared FP32 distance beyond which no pair can interact (r_cut with a margin)
};

// A cell-sorted point (32 bytes in 2D): position, an FP32 copy of the position
// wrapped into the box (for a cheap distance pre-check), original index (the
// radius is read from the radius array by it) and cell.
template <int D>
struct alignas(16) PairRec {
  double x[D];
  float xf[D];
  uint32_t idx;
  int cell;
};

// Cell of a position (the same expression in the counting and the scattering
// pass, so both agree); false for a non-finite coordinate (cell 0).
template <int D>
__device__ __forceinline__ bool cell_of(const double* __restrict__ p, const Box& b, int& cell) {
  bool ok = true;
  int stride = 1;
  cell = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double v = p[a];
    int c = 0;
    if (isfinite(v)) {
      const double u = v - floor(v * b.invL[a]) * b.L[a];
      c = min(max(int(u * b.inv_cw[a]), 0), b.nc[a] - 1);
    } else {
      ok = false;
    }
    cell += c * stride;
    stride *= b.nc[a];
  }
  return ok;
}

constexpr int kCellBatch = 4;  // points per thread per round: their loads overlap

template <int D>
__global__ void __launch_bounds__(kThreads) cell_count_kernel(const double* __restrict__ x, int64_t N, Box b,
                                                              int* cell_count, uint32_t* rank, int* status) {
  bool bad = false;
  const int64_t step = int64_t(gridDim.x) * blockDim.x;
  for (int64_t j0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j0 < N; j0 += kCellBatch * step) {
    double p[kCellBatch][D];
#pragma unroll
    for (int u = 0; u < kCellBatch; ++u)
#pragma unroll
      for (int a = 0; a < D; ++a) p[u][a] = j0 + u * step < N ? x[(j0 + u * step) * D + a] : 0.0;
    int cell[kCellBatch];
#pragma unroll
    for (int u = 0; u < kCellBatch; ++u) {
      bad |= !cell_of<D>(p[u], b, cell[u]);
      if (j0 + u * step < N) rank[j0 + u * step] = uint32_t(atomicAdd(&cell_count[cell[u]], 1));
    }
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
}

template <int D>
__global__ void __launch_bounds__(kThreads) cell_scatter_kernel(const double* __restrict__ x,
                                                                const double* __restrict__ radii, int64_t N, Box b,
                                                                const uint32_t* __restrict__ rank,
                                                                const int* __restrict__ cell_start, PairRec<D>* recs,
                                                                const uint32_t* __restrict__ gidx) {
  const int64_t step = int64_t(gridDim.x) * blockDim.x;
  for (int64_t j0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j0 < N; j0 += kCellBatch * step) {
    PairRec<D> r[kCellBatch];
    uint32_t rk[kCellBatch];
#pragma unroll
    for (int u = 0; u < kCellBatch; ++u) {
      const int64_t j = j0 + u * step;
      if (j < N) {
#pragma unroll
        for (int a = 0; a < D; ++a) r[u].x[a] = x[j * D + a];
        rk[u] = rank[j];
      }
    }
#pragma unroll
    for (int u = 0; u < kCellBatch; ++u) {
      const int64_t j = j0 + u * step;
      if (j >= N) break;
      cell_of<D>(r[u].x, b, r[u].cell);
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const double v = r[u].x[a];
        r[u].xf[a] = isfinite(v) ? float(v - floor(v * b.invL[a]) * b.L[a]) : 0.f;
      }
      r[u].idx = gidx ? gidx[j] : uint32_t(j);  // the pattern's index of the point
      recs[int64_t(cell_start[r[u].cell]) + rk[u]] = r[u];
    }
  }
}

// One thread per cell-sorted point; neighbours from the 3^D surrounding cells.
// cell_start has ncells + 1 entries (the last is N), so cells c..c+2 of a row
// are the records [cell_start[c], cell_start[c + 3]).
//
// Two phases per warp.  (1) Each lane scans its candidates with an FP32
// distance test on the wrapped positions and queues the ones within reach in
// a per-lane shared list (candidate counts differ between lanes, but this
// test is cheap); in 2D the warp first stages the union of its lanes' ranges
// of each neighbour row in shared memory with coalesced loads.  (2) The warp
// evaluates all queued pairs in FP64 with every lane busy (32 pairs at a
// time; a lane finds its pair by a search over the lanes' queue prefix sums)
// and adds the pair force to the owner's gradient slot in shared memory.
// Survivors beyond a full list are evaluated afterwards by a rescan of that
// point alone.  Only points whose pattern index lies in [own_lo, own_lo +
// own_n) take part as the first point of a pair and get a gradient (at
// index - own_lo); the others (a halo) are neighbours only.
constexpr int kPairQueue = 16;  // queued pairs per point

template <int D>
struct PairOut {
  double g[D];
  double e;
};

template <int D>
__device__ __forceinline__ PairOut<D> pair_term(const PairRec<D>& me, double my_r, const PairRec<D>& o, double o_r,
                                                const Box& b, double a_pow, double eps) {
  PairOut<D> out;
  double dr[D], r2 = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    dr[a] = min_image(me.x[a] - o.x[a], b.L[a], b.invL[a], true);
    r2 += dr[a] * dr[a];
  }
  double gij;
  const double e = pair_energy_gradient(r2, my_r + o_r, a_pow, eps, &gij);
#pragma unroll
  for (int a = 0; a < D; ++a) out.g[a] = gij != 0.0 ? -dr[a] * gij : 0.0;
  out.e = o.idx > me.idx ? e : 0.0;
  return out;
}

// Radius of original point k: radii[k], or the common value when radii is null.
__device__ __forceinline__ double radius_of(const double* __restrict__ radii, double r_uniform, uint32_t k) {
  return radii ? radii[k] : r_uniform;
}

template <int D>
__device__ __forceinline__ bool within_reach(const float (&a)[D], const float (&c)[D], const Box& b) {
  float r2 = 0.f;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    float d = a[k] - c[k];
    d -= rintf(d * b.invLf[k]) * b.Lf[k];
    r2 += d * d;
  }
  return r2 <= b.reject2;
}

// Record ranges of the 3^(D-1) neighbour rows of a cell (two ranges per row
// when x wraps; the second is empty otherwise), in scan order.
template <int D>
struct RowRanges {
  static constexpr int R = D == 1 ? 1 : (D == 2 ? 3 : 9);
  int lo[2 * R], hi[2 * R];
};

template <int D>
__device__ __forceinline__ RowRanges<D> row_ranges(int cell, const Box& b, const int* __restrict__ cell_start) {
  RowRanges<D> rr;
  int ci[3] = {0, 0, 0};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    ci[a] = cell % b.nc[a];
    cell /= b.nc[a];
  }
  const int nc0 = b.nc[0];
#pragma unroll
  for (int r = 0; r < RowRanges<D>::R; ++r) {
    int row = 0;
    if (D >= 2) {
      int c1 = ci[1] + (r % 3) - 1;
      c1 += c1 < 0 ? b.nc[1] : (c1 >= b.nc[1] ? -b.nc[1] : 0);
      row = c1 * nc0;
    }
    if (D >= 3) {
      int c2 = ci[2] + (r / 3) - 1;
      c2 += c2 < 0 ? b.nc[2] : (c2 >= b.nc[2] ? -b.nc[2] : 0);
      row += c2 * nc0 * b.nc[1];
    }
    const int c0 = ci[0];
    if (c0 >= 1 && c0 <= nc0 - 2) {
      rr.lo[2 * r] = cell_start[row + c0 - 1];
      rr.hi[2 * r] = cell_start[row + c0 + 2];
      rr.lo[2 * r + 1] = rr.hi[2 * r + 1] = 0;
    } else if (c0 == 0) {  // x wraps on the left
      rr.lo[2 * r] = cell_start[row];
      rr.hi[2 * r] = cell_start[row + 2];
      rr.lo[2 * r + 1] = cell_start[row + nc0 - 1];
      rr.hi[2 * r + 1] = cell_start[row + nc0];
    } else {  // x wraps on the right
      rr.lo[2 * r] = cell_start[row + nc0 - 2];
      rr.hi[2 * r] = cell_start[row + nc0];
      rr.lo[2 * r + 1] = cell_start[row];
      rr.hi[2 * r + 1] = cell_start[row + 1];
    }
  }
  return rr;
}

// Rescan of one point whose list overflowed: evaluates its survivors from the
// (skip)-th on, in the scan order of the first phase.
template <int D>
__device__ __forceinline__ PairOut<D> overflow_pairs(const PairRec<D>* __restrict__ recs, const double* __restrict__ radii,
                                                  double r_uniform, const int* __restrict__ cell_start, int64_t i,
                                                  const Box& b, double a_pow, double eps, int skip) {
  PairOut<D> acc;
#pragma unroll
  for (int a = 0; a < D; ++a) acc.g[a] = 0.0;
  acc.e = 0.0;
  const PairRec<D> me = recs[i];
  const double my_r = radius_of(radii, r_uniform, me.idx);
  const RowRanges<D> rr = row_ranges<D>(me.cell, b, cell_start);
  int seen = 0;
  for (int q = 0; q < 2 * RowRanges<D>::R; ++q)
    for (int j = rr.lo[q]; j < rr.hi[q]; ++j) {
      if (j == int(i) || !within_reach<D>(me.xf, recs[j].xf, b)) continue;
      if (seen++ < skip) continue;
      const PairOut<D> t = pair_term<D>(me, my_r, recs[j], radius_of(radii, r_uniform, recs[j].idx), b, a_pow, eps);
#pragma unroll
      for (int a = 0; a < D; ++a) acc.g[a] += t.g[a];
      acc.e += t.e;
    }
  return acc;
}

template <int D>
__global__ void __launch_bounds__(kThreads) cell_pair_kernel(const PairRec<D>* __restrict__ recs,
                                                             const double* __restrict__ radii, double r_uniform,
                                                             const int* __restrict__ cell_start, int64_t N, Box b,
                                                             double a_pow, double eps, double* grad, double* energy,
                                                             int accumulate, const int* __restrict__ status,
                                                             uint32_t own_lo, uint32_t own_n) {
  constexpr int NW = kThreads / 32;
  constexpr int kSpan = 96;  // 2D: staged records per neighbour row and warp
  __shared__ int queue[NW][32][kPairQueue];
  __shared__ double gsm[NW][32][D];
  __shared__ float2 span_xf[D == 2 ? NW : 1][3][kSpan];
  const bool bad = (*status) & STATUS_NONFINITE_INPUT;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double e_loc = 0.0;
  const int nc0 = b.nc[0];
  // whole warps iterate together (the pair phase needs every lane)
  const int64_t nwarps_total = int64_t(gridDim.x) * NW;
  for (int64_t wbase = (int64_t(blockIdx.x) * NW + warp) * 32; wbase < N; wbase += nwarps_total * 32) {
    const int64_t i = wbase + lane;
    PairRec<D> me;
    int nq = 0;
    if (i < N) me = recs[i];
    const bool active = i < N && me.idx - own_lo < own_n;
    // a warp of halo records only has nothing to do (and no range to stage:
    // its empty min/max would overflow the span test below)
    if (!__any_sync(0xffffffffu, active)) continue;
    // phase 1: candidates within reach -> queue
    bool staged = false;
    if constexpr (D == 2) {
      int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
      bool ok = true;
      if (active) {
        const int c0 = me.cell % nc0, c1 = me.cell / nc0;
        ok = c0 >= 1 && c0 <= nc0 - 2;
        if (ok) {
#pragma unroll
          for (int o1 = 0; o1 < 3; ++o1) {
            int r1 = c1 + o1 - 1;
            r1 += r1 < 0 ? b.nc[1] : (r1 >= b.nc[1] ? -b.nc[1] : 0);
            lo[o1] = cell_start[r1 * nc0 + c0 - 1];
            hi[o1] = cell_start[r1 * nc0 + c0 + 2];
          }
        }
      }
      int smin[3], smax[3];
#pragma unroll
      for (int o1 = 0; o1 < 3; ++o1) {
        int mn = active && ok ? lo[o1] : INT_MAX, mx = active && ok ? hi[o1] : INT_MIN;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
          mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        smin[o1] = mn;
        smax[o1] = mx;
      }
      staged = __all_sync(0xffffffffu, !active || ok) && smax[0] - smin[0] <= kSpan &&
               smax[1] - smin[1] <= kSpan && smax[2] - smin[2] <= kSpan;
      if (staged) {
#pragma unroll
        for (int o1 = 0; o1 < 3; ++o1)
          for (int k = lane; k < smax[o1] - smin[o1]; k += 32) {
            const PairRec<D>& rj = recs[smin[o1] + k];
            span_xf[warp][o1][k] = make_float2(rj.xf[0], rj.xf[1]);
          }
        __syncwarp();
        if (active) {
          const float mine_f[2] = {me.xf[0], me.xf[1]};
#pragma unroll
          for (int o1 = 0; o1 < 3; ++o1)
            for (int j = lo[o1]; j < hi[o1]; ++j) {
              const float2 q = span_xf[warp][o1][j - smin[o1]];
              const float other_f[2] = {q.x, q.y};
              if (j != int(i) && within_reach<2>(mine_f, other_f, b)) {
                if (nq < kPairQueue) queue[warp][lane][nq] = j;
                ++nq;
              }
            }
        }
      }
    }
    if (active && !staged) {
      const RowRanges<D> rr = row_ranges<D>(me.cell, b, cell_start);
#pragma unroll
      for (int q = 0; q < 2 * RowRanges<D>::R; ++q)
        for (int j = rr.lo[q]; j < rr.hi[q]; ++j)
          if (j != int(i) && within_reach<D>(me.xf, recs[j].xf, b)) {
            if (nq < kPairQueue) queue[warp][lane][nq] = j;
            ++nq;
          }
    }
    // phase 2: the queued pairs, every lane busy
    const int nql = min(nq, kPairQueue);
#pragma unroll
    for (int a = 0; a < D; ++a) gsm[warp][lane][a] = 0.0;
    int inc = nql;  // inclusive prefix sum of the queue lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    const int total = __shfl_sync(0xffffffffu, inc, 31);
    const int excl = inc - nql;
    __syncwarp();  // the queues and gradient slots are visible to the whole warp
    for (int t0 = 0; t0 < total; t0 += 32) {
      const int t = t0 + lane;
      // owner of item t: the number of lanes whose inclusive prefix is <= t
      int owner = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int pre = __shfl_sync(0xffffffffu, inc, owner + step - 1);
        if (pre <= t) owner += step;
      }
      const int first = __shfl_sync(0xffffffffu, excl, owner);
      if (t < total) {
        const int j = queue[warp][owner][t - first];
        const PairRec<D> mine = recs[wbase + owner];
        const PairOut<D> po = pair_term<D>(mine, radius_of(radii, r_uniform, mine.idx), recs[j],
                                           radius_of(radii, r_uniform, recs[j].idx), b, a_pow, eps);
        e_loc += po.e;
#pragma unroll
        for (int a = 0; a < D; ++a)
          if (po.g[a] != 0.0) atomicAdd(&gsm[warp][owner][a], po.g[a]);
      }
    }
    __syncwarp();
    if (active) {
      double gi[D];
#pragma unroll
      for (int a = 0; a < D; ++a) gi[a] = gsm[warp][lane][a];
      if (nq > kPairQueue) {  // rare: survivors beyond the list
        const PairOut<D> extra = overflow_pairs<D>(recs, radii, r_uniform, cell_start, i, b, a_pow, eps, kPairQueue);
#pragma unroll
        for (int a = 0; a < D; ++a) gi[a] += extra.g[a];
        e_loc += extra.e;
      }
      const double nan = __longlong_as_double(0x7ff8000000000000ULL);
#pragma unroll
      for (int a = 0; a < D; ++a) {
        double* dst = grad + int64_t(me.idx - own_lo) * D + a;
        const double v = bad ? nan : gi[a];
        *dst = accumulate ? *dst + v : v;
      }
    }
    __syncwarp();
  }
  block_sum_atomic(e_loc, energy);
  if (blockIdx.x == 0 && threadIdx.x == 0 && bad) atomicAdd(energy, __longlong_as_double(0x7ff8000000000000ULL));
}

// All pairs, tiled through shared memory (Cartesian distance or < 3 cells per dimension).
template <int D>
__global__ void __launch_bounds__(kThreads) allpairs_kernel(const double* __restrict__ x,
                                                            const double* __restrict__ radii, int64_t N, Box b,
                                                            bool periodic, double a_pow, double eps, double* grad,
                                                            double* energy, int accumulate, int* status) {
  __shared__ double tx[kThreads * D];
  __shared__ double tr[kThreads];
  double e_loc = 0.0;
  bool bad_local = false;
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < N; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const bool active = i < N;
    double xi[D], gi[D];
    double ri = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      xi[a] = active ? x[i * D + a] : 0.0;
      gi[a] = 0.0;
      if (active && !isfinite(xi[a])) bad_local = true;
    }
    if (active) ri = radii[i];
    for (int64_t t0 = 0; t0 < N; t0 += kThreads) {
      __syncthreads();
      const int64_t jl = t0 + threadIdx.x;
      if (jl < N) {
#pragma unroll
        for (int a = 0; a < D; ++a) tx[threadIdx.x * D + a] = x[jl * D + a];
        tr[threadIdx.x] = radii[jl];
      }
      __syncthreads();
      const int cnt = int((N - t0) < int64_t(kThreads) ? (N - t0) : int64_t(kThreads));
      if (active) {
        for (int jj = 0; jj < cnt; ++jj) {
          const int64_t j = t0 + jj;
          if (j == i) continue;
          double dr[D], r2 = 0.0;
#pragma unroll
          for (int a = 0; a < D; ++a) {
            dr[a] = min_image(xi[a] - tx[jj * D + a], b.L[a], b.invL[a], periodic);
            r2 += dr[a] * dr[a];
          }
          double gij;
          const double e = pair_energy_gradient(r2, ri + tr[jj], a_pow, eps, &gij);
          if (gij != 0.0) {
#pragma unroll
            for (int a = 0; a < D; ++a) gi[a] -= dr[a] * gij;
          }
          if (j > i) e_loc += e;
        }
      }
    }
    if (active) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        double* dst = grad + i * D + a;
        *dst = accumulate ? *dst + gi[a] : gi[a];
      }
    }
  }
  if (bad_local) raise_status(status, STATUS_NONFINITE_INPUT);
  block_sum_atomic(e_loc, energy);
}

__global__ void nan_fill_kernel(const int* __restrict__ status, double* grad, int64_t n, double* energy) {
  if (!((*status) & STATUS_NONFINITE_INPUT)) return;
  const double nan = __longlong_as_double(0x7ff8000000000000ULL);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    if (grad) grad[i] = nan;
  if (blockIdx.x == 0 && threadIdx.x == 0) *energy = nan;
}

// Box and cell grid of a pattern: cells of edge >= r_cut = 2 max(r_i)
// (inversepower_potential.hpp:115), at most about one cell per point (results
// do not depend on the cell size; the reference picks its own via
// ncellx_scale).  Returns the cell count; use_cells is false without a
// periodic box of at least 3 cells per dimension.
int64_t make_box(int D, const std::vector<double>& radii, const std::vector<double>& boxv, bool periodic, Box& box,
                 bool& use_cells) {
  const int64_t N = int64_t(radii.size());
  double rmax = 0.0;
  for (double r : radii) rmax = std::max(rmax, r);
  const double rcut = 2.0 * rmax;
  use_cells = periodic;
  int64_t ncells = 1;
  for (int a = 0; a < D; ++a) {
    box.L[a] = periodic ? boxv[a] : 1.0;
    box.invL[a] = 1.0 / box.L[a];
  }
  if (periodic) {
    const double target = std::max(1.0, std::floor(std::pow(double(std::max<int64_t>(N, 1)), 1.0 / D)));
    for (int a = 0; a < D; ++a) {
      // the margin keeps every cell at least r_cut wide after rounding
      int nc = rcut > 0 ? int(std::floor(box.L[a] / (rcut * (1.0 + 1e-9)))) : 1;
      nc = std::max(1, std::min(nc, int(target)));
      if (nc < 3) use_cells = false;
      box.nc[a] = nc;
      box.cw[a] = box.L[a] / nc;
      box.inv_cw[a] = nc / box.L[a];
      box.Lf[a] = float(box.L[a]);
      box.invLf[a] = float(box.invL[a]);
      ncells *= nc;
    }
  }
  // FP32 positions (wrapped into the box) are within a few ulp of the exact
  // ones; a 0.1% margin on r_cut never rejects an interacting pair
  const double rej = rcut * (1.0 + 1e-3) + 1e-6 * std::max({box.L[0], box.L[1], box.L[2]});
  box.reject2 = float(rej * rej);
  return ncells;
}

template <int D>
class InversePowerImpl final : public Potential {
 public:
  InversePowerImpl(double a, double eps, const std::vector<double>& radii, const std::vector<double>& boxv,
                   bool periodic)
      : N_(int64_t(radii.size())), a_(a), eps_(eps), periodic_(periodic) {
    init_status();
    if (periodic && int(boxv.size()) != D) throw InvalidArgument("box.size() must be equal to ndim");
    // equal radii (the usual case) are passed as one value instead of gathered
    uniform_r_ = !radii.empty() && std::all_of(radii.begin(), radii.end(), [&](double r) { return r == radii[0]; });
    r0_ = radii.empty() ? 0.0 : radii[0];
    const int64_t ncells = make_box(D, radii, boxv, periodic, box_, use_cells_);
    radii_.alloc(std::max<int64_t>(N_, 1));
    scratch_grad_.alloc(std::max<int64_t>(N_ * D, 1));
    if (N_) FB_CUDA(cudaMemcpy(radii_.p, radii.data(), sizeof(double) * N_, cudaMemcpyHostToDevice));
    if (use_cells_) {
      ncells_ = ncells;
      cell_count_.alloc(ncells + 1);  // the extra zero count makes cell_start[ncells] = N
      cell_start_.alloc(ncells + 1);
      block_sums_.alloc(scan_tmp_size(ncells + 1));
      rank_.alloc(std::max<int64_t>(N_, 1));
      recs_.alloc(std::max<int64_t>(N_, 1));
    }
  }

  int64_t ndof() const override { return N_ * D; }
  std::string kind() const override { return "InversePower"; }
  std::string describe() const override {
    std::string s = "InversePower D=" + std::to_string(D) + " N=" + std::to_string(N_) + " a=" + std::to_string(a_) +
                    (periodic_ ? " periodic" : " cartesian");
    if (use_cells_) {
      s += " cells=";
      for (int a = 0; a < D; ++a) s += (a ? "x" : "") + std::to_string(box_.nc[a]);
    } else {
      s += " all-pairs";
    }
    return s;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override {
    run(x, scratch_grad_.p, e, false, acc, s);
  }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, acc, s);
  }

 private:
  void run(const double* x, double* g, double* e, bool acc_grad, bool acc_e, cudaStream_t s) {
    timer_begin(s);
    begin_eval_status(s);
    if (!acc_e) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    if (N_ == 0) return;
    const int grid = int(std::min<int64_t>(ceil_div(N_, kThreads), int64_t(sm_count()) * 8));
    if (!use_cells_) {
      allpairs_kernel<D><<<grid, kThreads, 0, s>>>(x, radii_.p, N_, box_, periodic_, a_, eps_, g, e,
                                                  acc_grad ? 1 : 0, status_.p);
      FB_LAUNCH_CHECK();
    } else {
      FB_CUDA(cudaMemsetAsync(cell_count_.p, 0, sizeof(int) * (ncells_ + 1), s));
      cell_count_kernel<D><<<grid, kThreads, 0, s>>>(x, N_, box_, cell_count_.p, rank_.p, status_.p);
      exclusive_scan(cell_count_.p, cell_start_.p, block_sums_.p, ncells_ + 1, s);
      cell_scatter_kernel<D><<<grid, kThreads, 0, s>>>(x, radii_.p, N_, box_, rank_.p, cell_start_.p, recs_.p,
                                                       nullptr);
      FB_LAUNCH_CHECK();
      timer_mark("cell_sort", s);
      cell_pair_kernel<D><<<grid, kThreads, 0, s>>>(recs_.p, uniform_r_ ? nullptr : radii_.p, r0_, cell_start_.p, N_,
                                                    box_, a_, eps_, g, e, acc_grad ? 1 : 0, status_.p, 0u,
                                                    uint32_t(N_));
      FB_LAUNCH_CHECK();
    }
    nan_fill_kernel<<<grid, kThreads, 0, s>>>(status_.p, g, N_ * D, e);
    FB_LAUNCH_CHECK();
    timer_mark("pairs", s);
  }

  int64_t N_;
  double a_, eps_;
  bool periodic_;
  bool use_cells_ = false;
  Box box_;
  int64_t ncells_ = 0;
  bool uniform_r_ = false;
  double r0_ = 0.0;
  DevBuf<double> radii_, scratch_grad_;
  DevBuf<int> cell_count_, cell_start_, block_sums_;
  DevBuf<uint32_t> rank_;
  DevBuf<PairRec<D>> recs_;
};

}  // namespace

namespace {

// g (+)= full[0..n)
__global__ void take_slab_kernel(const double* __restrict__ full, double* __restrict__ g, int64_t n, int acc) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    g[i] = acc ? g[i] + full[i] : full[i];
}

class InversePowerShard final : public Potential {
 public:
  InversePowerShard(double a, double eps, const std::vector<double>& radii_all, const std::vector<double>& boxv,
                    bool periodic, int64_t lo, int64_t hi, GatherFn gather, ReduceFn reduce, void* ctx)
      : D_(int(boxv.size())), N_(int64_t(radii_all.size())), lo_(lo), hi_(hi), gather_(gather), reduce_(reduce),
        ctx_(ctx) {
    if (!gather || !reduce) throw InvalidArgument("a repulsion shard needs a gather and a reduce function");
    if (lo < 0 || hi < lo || hi > N_) throw InvalidArgument("the slab [lo, hi) must lie within the pattern");
    inner_ = make_inversepower(a, eps, radii_all, boxv, periodic, true, 1.0);
    init_status();
    xall_.alloc(std::max<int64_t>(N_ * D_, 1));
    gall_.alloc(std::max<int64_t>(N_ * D_, 1));
    et_.alloc(1);
  }

  int64_t ndof() const override { return (hi_ - lo_) * D_; }
  std::string kind() const override { return "InversePowerShard"; }
  bool host_steps() const override { return true; }  // the gather and the energy sum
  std::string describe() const override {
    return "InversePowerShard points [" + std::to_string(lo_) + ", " + std::to_string(hi_) + ") of " +
           std::to_string(N_) + "; " + inner_->describe();
  }
  void set_gradient_mode(int mode) override {
    grad_mode_ = mode;
    inner_->set_gradient_mode(mode);
  }
  int read_and_clear_status(cudaStream_t s) override {
    return Potential::read_and_clear_status(s) | inner_->read_and_clear_status(s);
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override {
    run(x, nullptr, e, acc, s);
  }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    gather_(x, (hi_ - lo_) * D_, xall_.p, N_ * D_, s, ctx_);
    if (g) inner_->energy_gradient(xall_.p, N_ * D_, gall_.p, et_.p, false, s);
    else inner_->energy(xall_.p, N_ * D_, et_.p, false, s);
    // every process evaluates the whole pattern; the one whose slab starts at
    // point 0 contributes the energy, so the sum holds it once, with the same
    // bits on every process
    if (!(lo_ == 0 && hi_ > 0)) FB_CUDA(cudaMemsetAsync(et_.p, 0, sizeof(double), s));
    reduce_(et_.p, 1, s, ctx_);
    if (acc) {
      add_scalar(et_.p, e, s);
    } else {
      FB_CUDA(cudaMemcpyAsync(e, et_.p, sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    const int64_t n = (hi_ - lo_) * D_;
    if (g && n > 0) {
      const int grid = int(std::min<int64_t>(ceil_div(n, 256), int64_t(sm_count()) * 8));
      take_slab_kernel<<<grid, 256, 0, s>>>(gall_.p + lo_ * D_, g, n, acc ? 1 : 0);
      FB_LAUNCH_CHECK();
    }
  }

  int D_;
  int64_t N_, lo_, hi_;
  GatherFn gather_;
  ReduceFn reduce_;
  void* ctx_;
  PotentialPtr inner_;
  DevBuf<double> xall_, gall_, et_;
};


// ---------------------------------------------------------------------------
// Repulsion over spatially compact index slabs, with a halo exchange.
//
// This process owns points [lo, hi) of the pattern.  The columns are the cell
// list's cells along axis 0 (each at least r_cut wide), so a point interacts
// only with points in its own column and the two beside it.  Per evaluation:
//  1. each process marks the columns that hold its points; the marks are
//     gathered from every process;
//  2. `need` = the columns next to another process's marked columns, `reach`
//     = the columns next to this process's own (periodic);
//  3. this process's points in `need` columns are exported (coordinates and
//     pattern index) and gathered from every process (the sizes differ);
//  4. the points received from other processes that lie in `reach` columns
//     join the own points as a halo; one cell list over both gives each own
//     point its complete gradient and the energy of the pairs whose lower
//     pattern index is an own point (each pair once, as
//     cell_list_potential.hpp:154-181 counts it);
//  5. one sum over the processes gives every process the pattern's energy; a
//     NaN energy (a non-finite coordinate on any process) makes the gradient
//     NaN.
// With the points ordered along axis 0 before the split, each slab is a
// spatial slab and only the points of the columns at its two ends travel;
// any other order stays correct and exports more.
// ---------------------------------------------------------------------------

// Column of a coordinate along axis 0 (the expression cell_of uses).
__device__ __forceinline__ int column_of(double v, const Box& b) {
  if (!isfinite(v)) return 0;
  const double u = v - floor(v * b.invL[0]) * b.L[0];
  return min(max(int(u * b.inv_cw[0]), 0), b.nc[0] - 1);
}

__device__ __forceinline__ bool column_bit(const uint32_t* __restrict__ m, int c) { return (m[c >> 5] >> (c & 31)) & 1u; }

// Own points: their copy at the head of the combined set and, if mask is not
// null, their columns' marks.  The lanes of a warp that mark the same word
// combine their bits first (points in spatial order share a few columns), so
// a warp issues one atomic per distinct word.
template <int D>
__global__ void halo_own_kernel(const double* __restrict__ x, int64_t n, Box b, uint32_t lo, uint32_t* mask,
                                double* comb_x, uint32_t* comb_idx) {
  const int lane = threadIdx.x & 31;
  for (int64_t b0 = int64_t(blockIdx.x) * blockDim.x; b0 < n; b0 += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = b0 + threadIdx.x;  // the whole warp iterates together
    const bool valid = i < n;
    int word = -1;
    uint32_t bit = 0u;
    if (valid) {
      const int c = column_of(x[i * D], b);
      word = c >> 5;
      bit = 1u << (c & 31);
#pragma unroll
      for (int a = 0; a < D; ++a) comb_x[i * D + a] = x[i * D + a];
      comb_idx[i] = lo + uint32_t(i);
    }
    if (mask) {
      const unsigned grp = __match_any_sync(0xffffffffu, word);
      const uint32_t bits = __reduce_or_sync(grp, bit);
      if (word >= 0 && lane == __ffs(grp) - 1) atomicOr(mask + word, bits);
    }
  }
}

__global__ void mask_to_double_kernel(const uint32_t* __restrict__ mask, int nwords, double* out) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += gridDim.x * blockDim.x) out[w] = double(mask[w]);
}

// need / reach from every process's marks (one block).
__global__ void halo_columns_kernel(const double* __restrict__ marks, int nranks, int rank, int nwords, int ncol,
                                    uint32_t* need, uint32_t* reach) {
  for (int w = threadIdx.x; w < nwords; w += blockDim.x) {
    need[w] = 0u;
    reach[w] = 0u;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    const int cm = c == 0 ? ncol - 1 : c - 1, cp = c == ncol - 1 ? 0 : c + 1;
    bool nd = false, rc = false;
    for (int q = 0; q < nranks; ++q) {
      const double* m = marks + int64_t(q) * nwords;
      const uint32_t bits = ((uint32_t(m[cm >> 5]) >> (cm & 31)) | (uint32_t(m[c >> 5]) >> (c & 31)) |
                             (uint32_t(m[cp >> 5]) >> (cp & 31))) & 1u;
      if (q == rank) rc = bits != 0u;
      else nd |= bits != 0u;
    }
    if (nd) atomicOr(need + (c >> 5), 1u << (c & 31));
    if (rc) atomicOr(reach + (c >> 5), 1u << (c & 31));
  }
}

// Own points in `need` columns -> export records (D coordinates, pattern index).
template <int D>
__global__ void halo_export_kernel(const double* __restrict__ x, int64_t n, Box b, uint32_t lo,
                                   const uint32_t* __restrict__ need, double* out, int* count) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    if (!column_bit(need, column_of(x[i * D], b))) continue;
    double* r = out + int64_t(atomicAdd(count, 1)) * (D + 1);  // at most n records
#pragma unroll
    for (int a = 0; a < D; ++a) r[a] = x[i * D + a];
    r[D] = double(lo + uint32_t(i));
  }
}

// Received records of the other processes in `reach` columns -> the halo,
// after the n_own own points of the combined set.
template <int D>
__global__ void halo_keep_kernel(const double* __restrict__ recv, int64_t n_recv, int64_t skip_lo, int64_t skip_hi,
                                 Box b, const uint32_t* __restrict__ reach, int64_t n_own, int64_t cap,
                                 int64_t n_total, double* comb_x, uint32_t* comb_idx, int* count, int* status) {
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n_recv; k += int64_t(gridDim.x) * blockDim.x) {
    if (k >= skip_lo && k < skip_hi) continue;  // this process's own export
    const double* r = recv + k * (D + 1);
    if (!column_bit(reach, column_of(r[0], b))) continue;
    const double gi = r[D];
    if (!(gi >= 0.0 && gi < double(n_total))) {  // not a point of the pattern
      raise_status(status, STATUS_OVERFLOW);
      continue;
    }
    const int s = atomicAdd(count, 1);
    if (s >= cap) {  // more than the other processes' points: some were sent twice
      raise_status(status, STATUS_OVERFLOW);
      continue;
    }
#pragma unroll
    for (int a = 0; a < D; ++a) comb_x[(n_own + s) * D + a] = r[a];
    comb_idx[n_own + s] = uint32_t(gi);
  }
}

__global__ void nan_if_nan_energy_kernel(const double* __restrict__ e, double* g, int64_t n) {
  if (!isnan(*e)) return;
  const double nan = __longlong_as_double(0x7ff8000000000000ULL);
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    g[i] = nan;
}

template <int D>
class InversePowerHalo final : public Potential {
 public:
  InversePowerHalo(double a, double eps, const std::vector<double>& radii_all, const std::vector<double>& boxv,
                   int64_t lo, int64_t hi, int rank, int nranks, GatherVFn gatherv, ReduceFn reduce, void* ctx)
      : N_(int64_t(radii_all.size())), lo_(lo), hi_(hi), rank_(rank), nranks_(nranks), a_(a), eps_(eps),
        gatherv_(gatherv), reduce_(reduce), ctx_(ctx) {
    if (!gatherv || !reduce) throw InvalidArgument("a repulsion halo shard needs a gatherv and a reduce function");
    if (lo < 0 || hi < lo || hi > N_) throw InvalidArgument("the slab [lo, hi) must lie within the pattern");
    if (nranks < 1 || rank < 0 || rank >= nranks) throw InvalidArgument("rank must lie in [0, nranks)");
    if (N_ >= (int64_t(1) << 31)) throw InvalidArgument("a halo shard holds fewer than 2^31 points");
    if (int(boxv.size()) != D) throw InvalidArgument("box.size() must be equal to ndim");
    init_status();
    bool use_cells = false;
    ncells_ = make_box(D, radii_all, boxv, true, box_, use_cells);
    if (!use_cells)
      throw InvalidArgument("the halo exchange needs cell lists: a periodic box of at least 3 cells per dimension");
    uniform_r_ = !radii_all.empty() &&
                 std::all_of(radii_all.begin(), radii_all.end(), [&](double r) { return r == radii_all[0]; });
    r0_ = radii_all.empty() ? 0.0 : radii_all[0];
    ncol_ = box_.nc[0];
    nwords_ = (ncol_ + 31) / 32;
    const int64_t n = hi - lo, cap = std::max<int64_t>(N_, 1);
    radii_.alloc(cap);
    if (N_) FB_CUDA(cudaMemcpy(radii_.p, radii_all.data(), sizeof(double) * N_, cudaMemcpyHostToDevice));
    mask_.alloc(nwords_);
    need_.alloc(nwords_);
    reach_.alloc(nwords_);
    mask_d_.alloc(nwords_);
    marks_.alloc(int64_t(nranks) * nwords_);
    exp_.alloc(std::max<int64_t>(n, 1) * (D + 1));
    recv_.alloc(cap * (D + 1));
    comb_x_.alloc(cap * D);
    comb_idx_.alloc(cap);
    counts_dev_.alloc(2);
    e_part_.alloc(1);
    scratch_g_.alloc(std::max<int64_t>(n, 1) * D);
    cell_count_.alloc(ncells_ + 1);  // the extra zero count makes cell_start[ncells] = the point count
    cell_start_.alloc(ncells_ + 1);
    block_sums_.alloc(scan_tmp_size(ncells_ + 1));
    rank_buf_.alloc(cap);
    recs_.alloc(cap);
    FB_CUDA(cudaMallocHost(&host_counts_, 2 * sizeof(int)));
    counts_.assign(size_t(nranks), 0);
  }
  ~InversePowerHalo() override {
    if (host_counts_) cudaFreeHost(host_counts_);
  }

  int64_t ndof() const override { return (hi_ - lo_) * D; }
  std::string kind() const override { return "InversePowerHalo"; }
  bool host_steps() const override { return true; }  // the gathers, the sizes read back and the energy sum
  std::string describe() const override {
    std::string s = "InversePowerHalo points [" + std::to_string(lo_) + ", " + std::to_string(hi_) + ") of " +
                    std::to_string(N_) + " process " + std::to_string(rank_) + "/" + std::to_string(nranks_) +
                    " D=" + std::to_string(D) + " cells=";
    for (int a = 0; a < D; ++a) s += (a ? "x" : "") + std::to_string(box_.nc[a]);
    return s;
  }
  bool halo_stats(int64_t* exported, int64_t* halo) const override {
    if (exported) *exported = exported_;
    if (halo) *halo = halo_;
    return true;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override { run(x, nullptr, e, acc, s); }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  int grid_for(int64_t n) const {
    return int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, kThreads), int64_t(sm_count()) * 8)));
  }

  int read_count(int which, cudaStream_t s) {
    FB_CUDA(cudaMemcpyAsync(host_counts_ + which, counts_dev_.p + which, sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    return host_counts_[which];
  }

  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    const int64_t n = hi_ - lo_;
    double* gout = g ? g : scratch_g_.p;
    const bool acc_g = g != nullptr && acc;
    begin_eval_status(s);
    FB_CUDA(cudaMemsetAsync(mask_.p, 0, sizeof(uint32_t) * nwords_, s));
    FB_CUDA(cudaMemsetAsync(counts_dev_.p, 0, 2 * sizeof(int), s));
    FB_CUDA(cudaMemsetAsync(e_part_.p, 0, sizeof(double), s));
    if (n > 0) {
      halo_own_kernel<D><<<grid_for(n), kThreads, 0, s>>>(x, n, box_, uint32_t(lo_), nranks_ > 1 ? mask_.p : nullptr,
                                                          comb_x_.p, comb_idx_.p);
      FB_LAUNCH_CHECK();
    }
    exported_ = 0;
    halo_ = 0;
    if (nranks_ > 1) {  // one process has no other process to exchange with
      mask_to_double_kernel<<<1, 256, 0, s>>>(mask_.p, nwords_, mask_d_.p);
      FB_LAUNCH_CHECK();
      // 1. every process's column marks
      gatherv_(mask_d_.p, nwords_, marks_.p, int64_t(nranks_) * nwords_, counts_.data(), s, ctx_);
      for (int q = 0; q < nranks_; ++q)
        if (counts_[size_t(q)] != nwords_)
          throw CudaError("halo exchange: the processes disagree on the column grid");
      // 2. need / reach, 3. the export
      halo_columns_kernel<<<1, 1024, 0, s>>>(marks_.p, nranks_, rank_, nwords_, ncol_, need_.p, reach_.p);
      FB_LAUNCH_CHECK();
      if (n > 0) {
        halo_export_kernel<D><<<grid_for(n), kThreads, 0, s>>>(x, n, box_, uint32_t(lo_), need_.p, exp_.p,
                                                               counts_dev_.p);
        FB_LAUNCH_CHECK();
      }
      exported_ = read_count(0, s);
      gatherv_(exp_.p, exported_ * (D + 1), recv_.p, std::max<int64_t>(N_, 1) * (D + 1), counts_.data(), s, ctx_);
      int64_t total = 0, skip_lo = 0;
      for (int q = 0; q < nranks_; ++q) {
        const int64_t c = counts_[size_t(q)];
        if (c < 0 || c % (D + 1)) throw CudaError("halo exchange: a process sent a partial record");
        if (q < rank_) skip_lo += c;
        total += c;
      }
      if (counts_[size_t(rank_)] != exported_ * (D + 1) || total > std::max<int64_t>(N_, 1) * (D + 1))
        throw CudaError("halo exchange: the gathered sizes do not add up");
      // 4. the halo and the cell list over own + halo points
      const int64_t n_recv = total / (D + 1);
      if (n_recv > 0) {
        halo_keep_kernel<D><<<grid_for(n_recv), kThreads, 0, s>>>(
            recv_.p, n_recv, skip_lo / (D + 1), skip_lo / (D + 1) + exported_, box_, reach_.p, n, N_ - n, N_,
            comb_x_.p, comb_idx_.p, counts_dev_.p + 1, status_.p);
        FB_LAUNCH_CHECK();
      }
      halo_ = std::min<int64_t>(read_count(1, s), N_ - n);
    }
    const int64_t nc = n + halo_;
    if (nc > 0) {
      const int grid = grid_for(nc);
      FB_CUDA(cudaMemsetAsync(cell_count_.p, 0, sizeof(int) * (ncells_ + 1), s));
      cell_count_kernel<D><<<grid, kThreads, 0, s>>>(comb_x_.p, nc, box_, cell_count_.p, rank_buf_.p, status_.p);
      exclusive_scan(cell_count_.p, cell_start_.p, block_sums_.p, ncells_ + 1, s);
      cell_scatter_kernel<D><<<grid, kThreads, 0, s>>>(comb_x_.p, radii_.p, nc, box_, rank_buf_.p, cell_start_.p,
                                                       recs_.p, comb_idx_.p);
      FB_LAUNCH_CHECK();
      cell_pair_kernel<D><<<grid, kThreads, 0, s>>>(recs_.p, uniform_r_ ? nullptr : radii_.p, r0_, cell_start_.p, nc,
                                                    box_, a_, eps_, gout, e_part_.p, acc_g ? 1 : 0, status_.p,
                                                    uint32_t(lo_), uint32_t(n));
      FB_LAUNCH_CHECK();
    }
    // 5. the pattern's energy on every process
    if (nranks_ > 1) reduce_(e_part_.p, 1, s, ctx_);
    if (g && n > 0) {
      nan_if_nan_energy_kernel<<<grid_for(n * D), kThreads, 0, s>>>(e_part_.p, g, n * D);
      FB_LAUNCH_CHECK();
    }
    if (acc) add_scalar(e_part_.p, e, s);
    else FB_CUDA(cudaMemcpyAsync(e, e_part_.p, sizeof(double), cudaMemcpyDeviceToDevice, s));
  }

  int64_t N_, lo_, hi_;
  int rank_, nranks_;
  double a_, eps_;
  GatherVFn gatherv_;
  ReduceFn reduce_;
  void* ctx_;
  Box box_;
  int64_t ncells_ = 0;
  int ncol_ = 1, nwords_ = 1;
  bool uniform_r_ = false;
  double r0_ = 0.0;
  int64_t exported_ = 0, halo_ = 0;
  int* host_counts_ = nullptr;
  std::vector<int64_t> counts_;
  DevBuf<double> radii_, mask_d_, marks_, exp_, recv_, comb_x_, e_part_, scratch_g_;
  DevBuf<uint32_t> mask_, need_, reach_, comb_idx_, rank_buf_;
  DevBuf<int> counts_dev_, cell_count_, cell_start_, block_sums_;
  DevBuf<PairRec<D>> recs_;
};

}  // namespace

PotentialPtr make_inversepower_halo(double a, double eps, const std::vector<double>& radii_all,
                                    const std::vector<double>& boxv, int64_t lo, int64_t hi, int rank, int nranks,
                                    GatherVFn gatherv, ReduceFn reduce, void* ctx) {
  const int D = int(boxv.size());
  if (D == 1) return PotentialPtr(new InversePowerHalo<1>(a, eps, radii_all, boxv, lo, hi, rank, nranks, gatherv, reduce, ctx));
  if (D == 2) return PotentialPtr(new InversePowerHalo<2>(a, eps, radii_all, boxv, lo, hi, rank, nranks, gatherv, reduce, ctx));
  if (D == 3) return PotentialPtr(new InversePowerHalo<3>(a, eps, radii_all, boxv, lo, hi, rank, nranks, gatherv, reduce, ctx));
  throw InvalidArgument("InversePower: dimension " + std::to_string(D) + " is not supported");
}

PotentialPtr make_inversepower_shard(double a, double eps, const std::vector<double>& radii_all,
                                     const std::vector<double>& boxv, bool periodic, int64_t lo, int64_t hi,
                                     GatherFn gather, ReduceFn reduce, void* ctx) {
  const int D = int(boxv.size());
  if (D < 1 || D > 3) throw std::runtime_error("InversePower: dimension " + std::to_string(D) + " is not supported");
  return PotentialPtr(new InversePowerShard(a, eps, radii_all, boxv, periodic, lo, hi, gather, reduce, ctx));
}

PotentialPtr make_inversepower(double a, double eps, const std::vector<double>& radii, const std::vector<double>& boxv,
                               bool periodic, bool use_cell_lists, double ncellx_scale) {
  (void)use_cell_lists;
  (void)ncellx_scale;
  const int D = int(boxv.size());
  if (D == 1) return PotentialPtr(new InversePowerImpl<1>(a, eps, radii, boxv, periodic));
  if (D == 2) return PotentialPtr(new InversePowerImpl<2>(a, eps, radii, boxv, periodic));
  if (D == 3) return PotentialPtr(new InversePowerImpl<3>(a, eps, radii, boxv, periodic));
  throw std::runtime_error("InversePower: dimension " + std::to_string(D) + " is not supported on the device");
}

}  // namespace fb
