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
};

// A cell-sorted point: position, radius, original index and cell.
template <int D>
struct alignas(16) PairRec {
  double x[D];
  double r;
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

template <int D>
__global__ void __launch_bounds__(kThreads) cell_count_kernel(const double* __restrict__ x, int64_t N, Box b,
                                                              int* cell_count, uint32_t* rank, int* status) {
  bool bad = false;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    int cell;
    bad |= !cell_of<D>(x + j * D, b, cell);
    rank[j] = uint32_t(atomicAdd(&cell_count[cell], 1));
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
}

template <int D>
__global__ void __launch_bounds__(kThreads) cell_scatter_kernel(const double* __restrict__ x,
                                                                const double* __restrict__ radii, int64_t N, Box b,
                                                                const uint32_t* __restrict__ rank,
                                                                const int* __restrict__ cell_start, PairRec<D>* recs) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    PairRec<D> r;
#pragma unroll
    for (int a = 0; a < D; ++a) r.x[a] = x[j * D + a];
    cell_of<D>(r.x, b, r.cell);
    r.r = radii[j];
    r.idx = uint32_t(j);
    recs[int64_t(cell_start[r.cell]) + rank[j]] = r;
  }
}

// One thread per cell-sorted point; neighbours from the 3^D surrounding cells.
// cell_start has ncells + 1 entries (the last is N), so cells c..c+2 of a row
// are the records [cell_start[c], cell_start[c + 3]).
template <int D>
__global__ void __launch_bounds__(kThreads) cell_pair_kernel(const PairRec<D>* __restrict__ recs,
                                                             const int* __restrict__ cell_start, int64_t N, Box b,
                                                             double a_pow, double eps, double* grad, double* energy,
                                                             int accumulate, const int* __restrict__ status) {
  const bool bad = (*status) & STATUS_NONFINITE_INPUT;
  double e_loc = 0.0;
  const int nc0 = b.nc[0];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += int64_t(gridDim.x) * blockDim.x) {
    const PairRec<D> me = recs[i];
    double gi[D];
#pragma unroll
    for (int a = 0; a < D; ++a) gi[a] = 0.0;
    int ci[3] = {0, 0, 0};
    {
      int c = me.cell;
#pragma unroll
      for (int a = 0; a < D; ++a) {
        ci[a] = c % b.nc[a];
        c /= b.nc[a];
      }
    }
    auto visit = [&](int s0, int s1) {
      for (int j = s0; j < s1; ++j) {
        if (j == int(i)) continue;
        const PairRec<D> o = recs[j];
        double dr[D], r2 = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          dr[a] = min_image(me.x[a] - o.x[a], b.L[a], b.invL[a], true);
          r2 += dr[a] * dr[a];
        }
        double gij;
        const double e = pair_energy_gradient(r2, me.r + o.r, a_pow, eps, &gij);
        if (gij != 0.0) {
#pragma unroll
          for (int a = 0; a < D; ++a) gi[a] -= dr[a] * gij;
        }
        if (o.idx > me.idx) e_loc += e;
      }
    };
    const int n1 = D >= 2 ? 3 : 1, n2 = D >= 3 ? 3 : 1;
    for (int o2 = 0; o2 < n2; ++o2)
      for (int o1 = 0; o1 < n1; ++o1) {
        int row = 0;
        if (D >= 2) {
          int c1 = ci[1] + o1 - 1;
          c1 += c1 < 0 ? b.nc[1] : (c1 >= b.nc[1] ? -b.nc[1] : 0);
          row = c1 * nc0;
        }
        if (D >= 3) {
          int c2 = ci[2] + o2 - 1;
          c2 += c2 < 0 ? b.nc[2] : (c2 >= b.nc[2] ? -b.nc[2] : 0);
          row += c2 * nc0 * b.nc[1];
        }
        const int c0 = ci[0];
        if (c0 >= 1 && c0 <= nc0 - 2) {
          visit(cell_start[row + c0 - 1], cell_start[row + c0 + 2]);
        } else if (c0 == 0) {  // x wraps on the left
          visit(cell_start[row], cell_start[row + 2]);
          visit(cell_start[row + nc0 - 1], cell_start[row + nc0]);
        } else {  // c0 == nc0 - 1: x wraps on the right
          visit(cell_start[row + nc0 - 2], cell_start[row + nc0]);
          visit(cell_start[row], cell_start[row + 1]);
        }
      }
    const double nan = __longlong_as_double(0x7ff8000000000000ULL);
#pragma unroll
    for (int a = 0; a < D; ++a) {
      double* dst = grad + int64_t(me.idx) * D + a;
      const double v = bad ? nan : gi[a];
      *dst = accumulate ? *dst + v : v;
    }
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

template <int D>
class InversePowerImpl final : public Potential {
 public:
  InversePowerImpl(double a, double eps, const std::vector<double>& radii, const std::vector<double>& boxv,
                   bool periodic)
      : N_(int64_t(radii.size())), a_(a), eps_(eps), periodic_(periodic) {
    init_status();
    if (periodic && int(boxv.size()) != D) throw InvalidArgument("box.size() must be equal to ndim");
    double rmax = 0.0;
    for (double r : radii) rmax = std::max(rmax, r);
    const double rcut = 2.0 * rmax;  // inversepower_potential.hpp:115
    use_cells_ = periodic;
    int64_t ncells = 1;
    for (int a = 0; a < D; ++a) {
      box_.L[a] = periodic ? boxv[a] : 1.0;
      box_.invL[a] = 1.0 / box_.L[a];
    }
    if (periodic) {
      // cells of edge >= r_cut, at most about one cell per point (results do
      // not depend on the cell size; the reference picks its own via ncellx_scale)
      const double target = std::max(1.0, std::floor(std::pow(double(std::max<int64_t>(N_, 1)), 1.0 / D)));
      for (int a = 0; a < D; ++a) {
        // the margin keeps every cell at least r_cut wide after rounding
        int nc = rcut > 0 ? int(std::floor(box_.L[a] / (rcut * (1.0 + 1e-9)))) : 1;
        nc = std::max(1, std::min(nc, int(target)));
        if (nc < 3) use_cells_ = false;
        box_.nc[a] = nc;
        box_.cw[a] = box_.L[a] / nc;
        box_.inv_cw[a] = nc / box_.L[a];
        ncells *= nc;
      }
    }
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
      cell_scatter_kernel<D><<<grid, kThreads, 0, s>>>(x, radii_.p, N_, box_, rank_.p, cell_start_.p, recs_.p);
      FB_LAUNCH_CHECK();
      timer_mark("cell_sort", s);
      cell_pair_kernel<D><<<grid, kThreads, 0, s>>>(recs_.p, cell_start_.p, N_, box_, a_, eps_, g, e,
                                                    acc_grad ? 1 : 0, status_.p);
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
  DevBuf<double> radii_, scratch_grad_;
  DevBuf<int> cell_count_, cell_start_, block_sums_;
  DevBuf<uint32_t> rank_;
  DevBuf<PairRec<D>> recs_;
};

}  // namespace

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
