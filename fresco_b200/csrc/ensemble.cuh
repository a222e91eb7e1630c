// Batched ensembles of independent 2D NUwU patterns and their device LBFGS.
//
// An ensemble holds P patterns, each with its own point count N_p, weights,
// mode grid (len(V_p) = (2K_p+1)^2) and targets S0_p, V_p, in one common box
// L.  It is the batched form of P pairs (fresco.potentials.NUwU,
// fresco.optimize.LBFGS_CPP) (fresco/potentials/nuwu.pyx:10-23,
// fresco/optimize/_lbfgs_cpp.pyx:43, opt.pyx:26-93): every pattern gets the
// loss, gradient and LBFGS trajectory it would get on its own, but all
// patterns are evaluated by one set of launches.
//
// Layout: the coordinates of all patterns are concatenated, pattern p at
// doubles [off_p, off_p + 2 N_p) of x (interleaved x0, y0, x1, ...).
// Patterns with the same mode grid form a group that shares its fine-grid
// geometry; per group and evaluation there is one launch per stage (sort
// count, sort scatter, spread, R2C, mode pass, C2C, interpolation), each
// covering every pattern of the group, and the groups run on forked streams.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace fb {

class Ensemble {
 public:
  virtual ~Ensemble();
  int n_patterns() const { return int(dof_off_.size()) - 1; }
  int64_t ndof() const { return dof_off_.back(); }
  const std::vector<int64_t>& dof_offsets() const { return dof_off_; }

  // Energies e[p] of every pattern and, when g is not null, the gradients
  // (device pointers, x layout).  Asynchronous on s: the groups run on
  // streams forked from s and joined back into it, so the call can be
  // captured into a CUDA graph on s.
  virtual void eval(const double* x, double* g, double* e, cudaStream_t s) = 0;

  // eval replayed as a CUDA graph for repeated (x, g, e) sets (captured on
  // the second call with a given set).
  void eval_graph(const double* x, double* g, double* e, cudaStream_t s);

  // Per-pattern status bits (StatusBits) raised since the last read (host
  // array of P ints); synchronises s.
  virtual void read_and_clear_status(int* out, cudaStream_t s) = 0;

  // Measures the spreading / interpolation variants of every group on x and
  // keeps the fastest (runs evaluations; synchronises s).
  virtual void tune(const double* x, double* g, double* e, cudaStream_t s) = 0;

  // Sets the split by hand: patterns whose tap work N w^2 is below ratio x
  // (the tile cells of all their bins) take the direct kernels (0: all
  // tiled, a huge ratio: all direct).
  virtual void set_split(double ratio) = 0;

  // Sets by hand the largest subproblem (points per tile block; bins are cut
  // into equal parts of at most that many): kMaxSub / 4 .. kMaxSub.  tune()
  // picks it per group together with the split.
  virtual void set_subproblem_cap(int cap) { (void)cap; }

  virtual std::string describe() const = 0;

  // Changes whenever the launch configuration changes (tune()), so that
  // graphs captured around eval know to recapture.
  int version() const { return version_; }

 protected:
  void invalidate_graphs();
  std::vector<int64_t> dof_off_{0};
  int version_ = 0;

 private:
  struct GraphEntry {
    const double* x;
    double* g;
    double* e;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs_;
  cudaStream_t capture_stream_ = nullptr;
};

using EnsemblePtr = std::shared_ptr<Ensemble>;

class Potential;
// Any single potential seen as a one-pattern ensemble, so that EnsembleLbfgs
// gives it a device-resident, graph-captured LBFGS.
EnsemblePtr make_potential_ensemble(std::shared_ptr<Potential> pot, int64_t n);

// radii: sum N_p values (pattern order); sk, v: sum n_modes[p] values.
EnsemblePtr make_nuwu_ensemble(int n_patterns, const int64_t* n_points, const double* radii, const int64_t* n_modes,
                               const double* sk, const double* v, const double* L, int ndim, double eps,
                               int precision);

struct EnsembleLbfgsParams {
  double tol = 1e-5;
  int M = 4;
  double maxstep = 0.1;
  double max_f_rise = 1e-4;
  double H0 = 0.1;
  bool rel_energy = false;
};

// LBFGS (source/lbfgs.cpp:9-258) for every pattern of an ensemble at once.
// Each pattern's iteration is a small state machine kept on the device: a
// new direction (two-loop recursion) when its last trial was accepted, a
// halved trial step after a rejected one, the accept test and memory update
// after each evaluation.  One ensemble step = one evaluation of every
// pattern; a step is one CUDA graph launch and needs no host round trip.
class EnsembleLbfgs {
 public:
  EnsembleLbfgs(EnsemblePtr ens, const double* x0, int64_t n, const EnsembleLbfgsParams& p);
  ~EnsembleLbfgs();
  EnsembleLbfgs(const EnsembleLbfgs&) = delete;
  EnsembleLbfgs& operator=(const EnsembleLbfgs&) = delete;

  // LBFGS_CPP.run(niter) for every pattern (optimizer.hpp:97-112): each
  // pattern iterates until rms <= tol or niter more iterations.  Returns the
  // number of ensemble steps taken.
  int run(int niter);
  // Exactly n ensemble steps (no host read in between).
  void steps(int n);
  // x, g (ndof doubles each) and per-pattern f, rms, iterations, evaluations
  // and whether the pattern still iterates.  Any pointer may be null.
  void get_state(double* x, double* g, double* f, double* rms, int* niter, int* nfev, int* active);
  int n_patterns() const { return P_; }

 private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
  int P_ = 0;
};

}  // namespace fb
