// Device-resident gradient optimisers: LBFGS (source/lbfgs.cpp:9-258) and
// modified FIRE (source/fresco/modified_fire.hpp:44-230, source/
// modified_fire.cpp:43-118), with the GradientOptimizer driver of
// source/fresco/optimizer.hpp:55-241.
//
// Vectors (x, g, LBFGS memory, FIRE velocities) stay in HBM; every dot
// product is an FP64 two-stage reduction with a fixed block count, so
// results are deterministic for a given device.  The host keeps only the
// control flow: it reads a few scalars once per potential evaluation (the
// line-search accept test and the stop criterion).
#pragma once

#include <memory>
#include <vector>

#include "potential.cuh"

namespace fb {

struct LbfgsParams {
  double tol = 1e-5;
  int M = 4;
  double maxstep = 0.1;
  double max_f_rise = 1e-4;
  double H0 = 0.1;
  bool rel_energy = false;
  int maxiter = 10000;
  int iprint = -1;
  int verbosity = 0;
};

struct FireParams {
  double dtstart = 0.1, dtmax = 1.0, maxstep = 0.5;
  int Nmin = 5;
  double finc = 1.1, fdec = 0.5, fa = 0.99, astart = 0.1, tol = 1e-3;
  bool stepback = true;
  int maxiter = 10000;
  int iprint = -1;
  int verbosity = 0;
};

class Optimizer {
 public:
  virtual ~Optimizer();
  virtual void one_iteration() = 0;
  virtual void run(int niter);  // optimizer.hpp:97-112
  void run();           // optimizer.hpp:118-121
  bool stop_criterion_satisfied();
  virtual void set_func_gradient(double f, const double* grad, int64_t n) = 0;
  virtual void reset(const double* x0, int64_t n) = 0;
  void get_state(double* x, double* g, double* f, double* rms, int* nfev, int* niter, int* maxiter, double* H0);
  // Exact-resume image of the optimiser's state (coordinates, gradient,
  // memory, step parameters, counters), host bytes.  An image loads into an
  // optimiser of the same family, size and memory length; the loaded one
  // continues the saved trajectory.
  int64_t state_bytes() const;
  void save_state(uint8_t* buf);
  void load_state(const uint8_t* buf, int64_t bytes);
  virtual double* device_x() = 0;
  virtual double* device_g() = 0;
  virtual double h0() const { return 0.0; }
  // LBFGS::set_H0 (source/fresco/lbfgs.hpp:70-76); other optimisers have no H0
  virtual void set_H0(double H0) {
    (void)H0;
    throw InvalidArgument("set_H0: only LBFGS has an initial inverse-Hessian scale");
  }
  // One pattern split over processes (each holds a slab of x): every dot
  // product's block partials are summed over the processes by fn before they
  // are used, and the rms is taken over global_ndof coordinates.
  virtual void set_reducer(ReduceFn fn, void* ctx, int64_t global_ndof) {
    (void)fn;
    (void)ctx;
    (void)global_ndof;
    throw InvalidArgument("this optimiser does not run over a sharded pattern (LBFGS does)");
  }

 protected:
  Optimizer(PotentialPtr pot, int64_t n, double tol, int maxiter, int iprint, int verbosity);
  // Image layout after the common header: the device blocks of `image_blocks`
  // in order.  family: 1 LBFGS, 2 FIRE (both FIRE forms share one layout).
  struct Block {
    void* dev;
    int64_t bytes;
  };
  virtual int family() const = 0;
  virtual int memory_length() const { return 0; }
  virtual std::vector<Block> image_blocks() = 0;
  // after a load: re-establish host mirrors and invariants from the device state
  virtual void after_load() {}
  virtual void initialize_func_gradient() = 0;
  void eval(const double* x, double* g, double* e);  // one potential call (nfev not touched)

  PotentialPtr pot_;
  cudaStream_t s_ = nullptr;
  int64_t n_;
  int P_;  // reduction blocks
  double tol_;
  int maxiter_, iprint_, verbosity_;
  int iter_ = 0, nfev_ = 0;
  double f_ = 0.0, rms_ = 1e10;
  bool func_initialized_ = false;
  DevBuf<double> part_;  // reduction partials [slots][P_]
  double* host_ = nullptr;  // pinned scalar mirror
};

std::unique_ptr<Optimizer> make_lbfgs(PotentialPtr pot, const double* x0, int64_t n, const LbfgsParams& p);
std::unique_ptr<Optimizer> make_fire(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p);
// Modified FIRE with each iteration one CUDA graph launch (same iterations and trajectory).
std::unique_ptr<Optimizer> make_fire_graph(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p);

}  // namespace fb
