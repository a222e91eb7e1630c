// Device-side potential interface: the B200 counterpart of
// fresco::BasePotential (source/fresco/base_potential.hpp:15-156).  All
// pointers are device pointers; every call is asynchronous on the given
// stream and allocates nothing.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace fb {

using ReduceFn = void (*)(double* data, int64_t count, void* stream, void* ctx);
// Concatenation over the processes of their local arrays, in process order,
// into `full` (full_count values), ordered on `stream`.
using GatherFn = void (*)(const double* local, int64_t local_count, double* full, int64_t full_count, void* stream,
                          void* ctx);
// Concatenation over the processes of local arrays whose lengths differ, in
// process order, into `full` (at most full_capacity values); counts[q]
// (host memory) receives process q's length.  Ordered on `stream`.
using GatherVFn = void (*)(const double* local, int64_t local_count, double* full, int64_t full_capacity,
                           int64_t* counts, void* stream, void* ctx);

// *dst += *src on stream s (one device scalar)
void add_scalar(const double* src, double* dst, cudaStream_t s);

class Potential {
 public:
  virtual ~Potential();

  // Number of coordinates the potential expects (-1: any).
  virtual int64_t ndof() const = 0;

  // E(x) -> *energy (or += when accumulate).  base_potential.hpp:28-31.
  virtual void energy(const double* x, int64_t n, double* energy, bool accumulate, cudaStream_t s) = 0;

  // E(x), grad E(x).  With accumulate the gradient and energy are added to
  // what the buffers hold (base_potential.hpp:50-58 add_energy_gradient, here
  // without the temporary vector).
  virtual void energy_gradient(const double* x, int64_t n, double* grad, double* energy, bool accumulate,
                               cudaStream_t s) = 0;

  // energy_gradient (grad != nullptr) or energy, replayed as a CUDA graph
  // when the same call (buffers, accumulate flag, gradient mode) repeats: the
  // second call with a given set captures the launches on a private stream,
  // and that call and every later one launch the instantiated graph on s.
  // One-off buffer sets run directly.  Stage timing bypasses the graphs.
  void eval(const double* x, int64_t n, double* grad, double* energy, bool accumulate, cudaStream_t s);
  void set_graphs_enabled(bool on);

  // Sticky status bits (StatusBits) raised by kernels since the last read.
  virtual int read_and_clear_status(cudaStream_t s);

  virtual std::string kind() const = 0;

  // Gradient convention: 0 = the reference's own formula (default, drop-in
  // parity), 1 = the exact derivative of the energy with respect to the input
  // coordinates (what automatic differentiation needs).  They differ by the
  // reference's scalings: NUwU and NUwNU return d/dx of the 2 pi-scaled NUFFT
  // coordinate, UwNU divides by 2 pi, NUwNU drops conj(c_j), UwU halves the
  // rho term and drops the d(1/R) term.
  virtual void set_gradient_mode(int mode) { grad_mode_ = mode; }
  // The sum over the processes that share one pattern of a device array, in
  // place, ordered on `stream` (the caller's all-reduce).  Only a potential
  // with an exchange step (a NUwU shard) takes one; it then evaluates the
  // whole pattern's loss through it.
  // Whether an evaluation runs host code between its launches (an exchange
  // between processes): such a potential is never captured into a CUDA graph.
  virtual bool host_steps() const { return false; }
  virtual void set_reducer(ReduceFn fn, void* ctx) {
    (void)fn;
    (void)ctx;
    throw InvalidArgument(kind() + " has no exchange step between processes");
  }
  int gradient_mode() const { return grad_mode_; }
  // Human-readable set-up summary (kernel width, grids, ...).
  virtual std::string describe() const { return kind(); }
  // Points exported to and received from the other processes in the last
  // evaluation (repulsion with a halo exchange); false for other potentials.
  virtual bool halo_stats(int64_t* exported, int64_t* halo) const {
    (void)exported;
    (void)halo;
    return false;
  }

  int device = 0;

  // Per-stage CUDA-event timing (for the benchmark's roofline figures).  Each
  // evaluation records its own event set on the launch stream; collection
  // (a host sync) happens only when the totals are read.
  struct StageTimer {
    bool enabled = false;
    std::vector<std::vector<cudaEvent_t>> sets;
    std::vector<std::vector<std::string>> names;
    int used = 0;
    std::vector<std::string> total_names;
    std::vector<double> total_ms;
    std::vector<int> count;
  };
  StageTimer timer;
  void timer_begin(cudaStream_t s);
  void timer_mark(const char* name, cudaStream_t s);  // records the end of a stage
  void timer_collect();                              // host sync; accumulates elapsed times
  virtual bool timing_active() const { return timer.enabled; }

 protected:
  void invalidate_graphs();
  int grad_mode_ = 0;
  // True while eval() runs this potential's launches (directly or into its
  // own graph): only then may they fork onto side streams (a caller that
  // captures the launches into a graph of its own gets them in one stream).
  bool in_eval_ = false;
  DevBuf<int> status_;  // [0] current evaluation, [1] accumulated for the host
  void init_status();
  void begin_eval_status(cudaStream_t s) { FB_CUDA(cudaMemsetAsync(status_.p, 0, sizeof(int), s)); }

 private:
  struct GraphEntry {
    const double* x;
    double* g;
    double* e;
    int64_t n;
    bool acc;
    int mode;
    uint64_t last_use;
    cudaGraphExec_t exec;  // null until the second call with this key
  };
  static constexpr size_t kMaxGraphs = 8;
  std::vector<GraphEntry> graphs_;
  uint64_t graph_clock_ = 0;
  bool graphs_enabled_ = true;
  cudaStream_t capture_stream_ = nullptr;
};

using PotentialPtr = std::shared_ptr<Potential>;

// CombinedPotential (source/fresco/combine_potentials.hpp:16-59).
class CombinedPotential : public Potential {
 public:
  CombinedPotential();
  ~CombinedPotential() override;
  void add(PotentialPtr p);
  int64_t ndof() const override;
  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override;
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override;
  int read_and_clear_status(cudaStream_t s) override;
  void set_gradient_mode(int mode) override;
  bool timing_active() const override;
  bool host_steps() const override {
    for (auto& p : parts_)
      if (p->host_steps()) return true;
    return false;
  }
  std::string kind() const override { return "CombinedPotential"; }
  const std::vector<PotentialPtr>& parts() const { return parts_; }

 private:
  // Parts after the first run on side streams into their own gradient and
  // energy (gscr_, escr_), added to the first part's in part order at the join.
  void prepare_side(int64_t n);
  std::vector<PotentialPtr> parts_;
  std::vector<cudaStream_t> side_;
  std::vector<cudaEvent_t> done_;
  cudaEvent_t fork_ = nullptr;
  DevBuf<double> gscr_, escr_;
  int64_t scr_n_ = 0;
};

// One NUwU pattern whose points are split over several processes (GPUs).
// rho(k) is linear in the points, so each shard computes the undeconvolved
// rho of its own points at the active modes, the caller sums these over the
// shards (one all-reduce of 2 n_rho doubles), and each shard finishes the
// mode pass with the global rho and interpolates its own points.  Weights
// and 1/N use the totals of all shards.
class NUwUShard {
 public:
  virtual ~NUwUShard() = default;
  virtual int64_t n_rho() const = 0;  // active modes (complex values in rho)
  // rho[2 i], rho[2 i + 1] = rho of this shard's points at active mode i
  virtual void shard_rho(const double* x, double* rho, cudaStream_t s) = 0;
  // energy (every shard gets the same) and, if grad, this shard's gradient;
  // rho holds the sum over all shards
  virtual void shard_finish(const double* rho, double* grad, double* energy, cudaStream_t s) = 0;
};

// Sum over the points of NUwU's per-point weight factor (area^D with the
// reference's repeated area product, nuwu.hpp:125-149), in index order.
double nuwu_weight_factor_sum(const double* radii, int64_t n, int D);

// Factories (defined per potential family).
PotentialPtr make_nuwu_shard(const std::vector<double>& radii_local, int64_t n_total, double weight_sum_total,
                             double K, const std::vector<double>& sk, const std::vector<double>& v,
                             const std::vector<double>& L, double eps, int precision);
// InversePower over a pattern split into index slabs: this process owns points
// [lo, hi); each evaluation gathers every slab, evaluates the repulsion of the
// whole pattern and keeps this slab's gradient; the energy is counted once
// (by the process whose slab starts at point 0) and summed by `reduce`.
PotentialPtr make_inversepower_shard(double a, double eps, const std::vector<double>& radii_all,
                                     const std::vector<double>& boxv, bool periodic, int64_t lo, int64_t hi,
                                     GatherFn gather, ReduceFn reduce, void* ctx);
// InversePower (periodic, cell lists) over spatially compact index slabs:
// this process owns points [lo, hi) and is process `rank` of `nranks`; each
// evaluation exchanges only the points next to another process's points (a
// halo, gathered with `gatherv`), evaluates its own points' pairs and sums the
// energy with `reduce`.
PotentialPtr make_inversepower_halo(double a, double eps, const std::vector<double>& radii_all,
                                    const std::vector<double>& boxv, int64_t lo, int64_t hi, int rank, int nranks,
                                    GatherVFn gatherv, ReduceFn reduce, void* ctx);
PotentialPtr make_nuwu(const std::vector<double>& radii, double K, const std::vector<double>& sk,
                       const std::vector<double>& v, const std::vector<double>& L, double eps, int precision);
PotentialPtr make_uwu(const std::vector<int>& grid, double K, const std::vector<double>& sk,
                      const std::vector<double>& v, const std::vector<double>& L, double eps, int precision);
PotentialPtr make_uwnu(const std::vector<int>& grid, const std::vector<double>& kpts, const std::vector<double>& sk,
                       const std::vector<double>& v, const std::vector<double>& L, double eps, int precision);
PotentialPtr make_nuwnu(const std::vector<double>& radii, const std::vector<double>& kpts,
                        const std::vector<double>& sk, const std::vector<double>& v, const std::vector<double>& L,
                        double eps, int precision);
// fresco.utils.export_structure on the device (host arrays in and out):
// sk_out and gr_out hold Nk^ndim values in centred order, s_radial and g_radial
// Nk/2 + 1 radial averages.
void export_structure(const double* x, int64_t n_points, int ndim, const double* L, int Nk, const double* radii,
                      double tol, double* sk_out, double* gr_out, double* s_radial, double* g_radial);

// NUwNU loss and gradient from caller-owned device arrays with no device
// allocation; the per-k-point sums use a fixed static device array, so n_k is
// limited to nuwnu_noalloc_max_kpoints().
int64_t nuwnu_noalloc_max_kpoints();
void nuwnu_energy_gradient_noalloc(const double* d_x, int64_t n_points, int ndim, const double* d_weights,
                                   const double* d_kpts, const double* d_sk, const double* d_v, int64_t n_k,
                                   const double* L, int gradient_mode, double* d_grad, double* d_energy,
                                   bool accumulate, cudaStream_t stream);
PotentialPtr make_inversepower(double a, double eps, const std::vector<double>& radii,
                               const std::vector<double>& boxv, bool periodic, bool use_cell_lists,
                               double ncellx_scale);

}  // namespace fb
