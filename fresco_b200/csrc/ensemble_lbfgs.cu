// LBFGS for every pattern of an ensemble at once (ensemble.cuh).
//
// Per pattern the iteration is that of source/lbfgs.cpp:9-258 (the same
// steps as the single-pattern Lbfgs in optimizer.cu): two-loop recursion
// (lbfgs.cpp:107-170), uphill inversion and the maxstep cap (:176-197),
// backtracking by halving while E rises by more than max_f_rise, accepting
// after the tenth trial anyway (:200-236), memory update with ys/yy reset
// to 1 when zero (:66-105), rms = |g|/sqrt(n) (:243).
//
// Batched form: the coordinates of all patterns are one vector; blocks own
// chunks of ONE pattern (DofItem), so every dot product is a per-pattern
// sum of block partials (fixed order).  A pattern's progress lives in a
// device state word (BlState): after an accepted trial (nred = 0) the next
// step computes a new direction, after a rejected one (nred > 0) it only
// halves the trial step.  One ensemble step is
//   direction (1 + 2M launches, patterns that need none skip them)
//   -> trial point -> evaluation of every pattern -> accept test and memory
//   update (post) -> per-pattern state update (finalize)
// captured once as a CUDA graph.  steps(n) replays it n times; run(niter) is
// one graph launch: a conditional WHILE node repeats the step while a
// pattern is still iterating (checked on the device after every step), so
// the host waits once per run (the host-driven loop that reads the number of
// still-iterating patterns every few steps remains for a CUDA build that
// cannot capture the step into a conditional body).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ensemble.cuh"
#include "potential.cuh"

namespace fb {

namespace {

constexpr int kBlThreads = 512;
constexpr int kBlChunk = 4096;  // doubles per block

struct DofItem {
  int64_t i0, i1;  // dof range
  int p, pad_;     // pattern
};

struct PatRange {
  int lo, hi;  // item range of the pattern
};

struct BlState {
  double f, rms, H0, inv_sqrt_n, inv_n;
  int k, nred, iter, nfev, stop_iter, active;
};

struct BlParams {
  double tol, maxstep, max_f_rise;
  int M, rel;
};

enum BlSlot { B_IN = 0, B_OUT = 1, B_SG = 2, B_SS = 3, B_GG = 4, B_YS = 5, B_YY = 6, B_NSLOT = 7 };

// Sum of part[lo..hi), the same value on every thread of the block.
__device__ double pat_sum(const double* __restrict__ part, int lo, int hi) {
  __shared__ double sh[32];
  __shared__ double result;
  double v = 0.0;
  for (int i = lo + int(threadIdx.x); i < hi; i += blockDim.x) v += part[i];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) result = s;
  }
  __syncthreads();
  const double r = result;
  __syncthreads();
  return r;
}

// Block sums of v[0..K-1] into part[slot[k] * nitems + blockIdx.x].
template <int K>
__device__ void item_partials(double (&v)[K], double* part, int nitems, const int (&slot)[K]) {
  __shared__ double red[K][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) red[k][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = lane < nw ? red[k][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) part[int64_t(slot[k]) * nitems + blockIdx.x] = s;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ bool needs_direction(const BlState& s) { return s.active && s.nred == 0; }

// lbfgs.cpp:206-236: accept when E rose by less than max_f_rise (absolute,
// or relative to |f|), or after the tenth trial.
__device__ __forceinline__ bool bl_accept(const BlState& s, double fnew, const BlParams& prm) {
  double df = fnew - s.f;
  if (prm.rel) {
    double absf = 1e-100;
    if (s.f != 0) absf = fabs(s.f);
    df /= absf;
  }
  const bool ok = df < prm.max_f_rise;
  return ok || s.nred >= 9;
}

__global__ void __launch_bounds__(kBlThreads) bl_dot_gg(const double* __restrict__ g, const DofItem* __restrict__ items,
                                                        double* part, int nitems) {
  const DofItem it = items[blockIdx.x];
  double v[1] = {0.0};
  for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) v[0] += g[i] * g[i];
  const int sl[1] = {B_GG};
  item_partials<1>(v, part, nitems, sl);
}

// Block-wide sums of K per-item partial slots over the items [lo, hi) of one
// pattern (one block per pattern); the totals are valid in thread 0.
template <int K>
__device__ __forceinline__ void pattern_totals(const double* __restrict__ part, int nitems, int lo, int hi,
                                               const int (&slot)[K], double (&tot)[K]) {
  __shared__ double red[K][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double v = 0.0;
    for (int i = lo + int(threadIdx.x); i < hi; i += blockDim.x) v += part[int64_t(slot[k]) * nitems + i];
    v = warp_sum(v);
    if (lane == 0) red[k][wid] = v;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) tot[k] = warp_sum(lane < nw ? red[k][lane] : 0.0);
  }
}

constexpr int kFinThreads = 128;  // one block per pattern in the per-pattern state kernels

// Initial f and rms = sqrt(|g|^2 / n) (optimizer.hpp:203-210).
__global__ void __launch_bounds__(kFinThreads) bl_init_fin(BlState* st, const double* __restrict__ e,
                                                           const PatRange* __restrict__ pr,
                                                           const double* __restrict__ part, int nitems, int P,
                                                           BlParams prm) {
  const int p = blockIdx.x;
  const int sl[1] = {B_GG};
  double tot[1] = {0.0};
  pattern_totals<1>(part, nitems, pr[p].lo, pr[p].hi, sl, tot);
  if (threadIdx.x != 0) return;
  BlState s = st[p];
  const double gg = tot[0];
  s.f = e[p];
  s.rms = sqrt(gg * s.inv_n);
  s.nfev += 1;
  s.active = (s.rms > prm.tol) && (s.iter < s.stop_iter);
  st[p] = s;
}

// run(niter): every pattern may take niter more iterations while rms > tol.
__global__ void bl_set_stop(BlState* st, int P, int niter, BlParams prm) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  BlState s = st[p];
  s.stop_iter = s.iter + niter;
  s.active = (s.rms > prm.tol) && (s.iter < s.stop_iter);
  st[p] = s;
}

__global__ void bl_count_active(const BlState* __restrict__ st, int P, int* out) {
  int c = 0;
  for (int p = threadIdx.x; p < P; p += blockDim.x) c += st[p].active ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  __shared__ int sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += sh[w];
    *out = t;
  }
}

// The run loop's condition (run(niter) as one graph launch): continue while a
// pattern is still iterating and fewer than guard[1] steps have run; guard[0]
// counts the steps.  `first` marks the check before the first step.
__global__ void bl_loop(const BlState* __restrict__ st, int P, int* guard, cudaGraphConditionalHandle h, int first) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int p = threadIdx.x; p < P; p += blockDim.x)
    if (st[p].active) any = 1;  // every writer stores the same value
  __syncthreads();
  if (threadIdx.x == 0) {
    const int taken = first ? 0 : guard[0] + 1;
    guard[0] = taken;
    cudaGraphSetConditional(h, (any && taken < guard[1]) ? 1u : 0u);
  }
}

__global__ void bl_guard_init(int* guard, int limit) {
  guard[0] = 0;
  guard[1] = limit;
}

// step = g and the first dot: |g|^2 for k = 0, s_(k-1) . g otherwise.
__global__ void __launch_bounds__(kBlThreads) bl_dir_start(const double* __restrict__ g, double* __restrict__ step,
                                                           const double* __restrict__ S, int64_t nd,
                                                           const DofItem* __restrict__ items,
                                                           const BlState* __restrict__ st, int M, double* part,
                                                           int nitems) {
  const DofItem it = items[blockIdx.x];
  const BlState s = st[it.p];
  if (!needs_direction(s)) return;
  double v[1] = {0.0};
  if (s.k == 0) {
    for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) v[0] += g[i] * g[i];
  } else {
    const double* si = S + int64_t((s.k - 1) % M) * nd;
    #pragma unroll 4
    for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) {
      const double gi = g[i];
      step[i] = gi;
      v[0] += si[i] * gi;
    }
  }
  const int sl[1] = {B_IN};
  item_partials<1>(v, part, nitems, sl);
}

// Update u (0 <= u < 2M) of the two-loop recursion for every pattern that
// computes a direction: u < m backward, m <= u < 2m forward, m = min(k, M)
// (lbfgs.cpp:136-169); k = 0 takes the first step -H0 c g with c = 1/|g|
// when |g| > 1 and c = |g| otherwise (lbfgs.cpp:109-124).
__global__ void __launch_bounds__(kBlThreads) bl_update(int u, double* __restrict__ step, const double* __restrict__ g,
                                                        const double* __restrict__ S, const double* __restrict__ Y,
                                                        int64_t nd, const DofItem* __restrict__ items,
                                                        const BlState* __restrict__ st,
                                                        const PatRange* __restrict__ pr, const double* __restrict__ rho,
                                                        double* alpha, int M, double* part, int nitems) {
  const DofItem it = items[blockIdx.x];
  const BlState s = st[it.p];
  if (!needs_direction(s)) return;
  const PatRange r = pr[it.p];
  const int in_slot = (u & 1) ? B_OUT : B_IN, out_slot = (u & 1) ? B_IN : B_OUT;
  if (s.k == 0) {
    if (u != 0) return;
    double gnorm = sqrt(pat_sum(part + int64_t(B_IN) * nitems, r.lo, r.hi));
    if (gnorm > 1.0) gnorm = 1.0 / gnorm;
    const double pref = -gnorm * s.H0;
    double v[2] = {0.0, 0.0};
    for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) {
      const double x = pref * g[i];
      step[i] = x;
      v[0] += x * g[i];
      v[1] += x * x;
    }
    const int sl[2] = {B_SG, B_SS};
    item_partials<2>(v, part, nitems, sl);
    return;
  }
  const int m = min(s.k, M), jmin = s.k - m, jmax = s.k;
  if (u >= 2 * m) return;
  const double dotin = pat_sum(part + int64_t(in_slot) * nitems, r.lo, r.hi);
  const int64_t pm = int64_t(it.p) * M;
  double coef;
  const double* vec;
  const double* dnext;
  bool scale = false, ls = false;
  if (u < m) {
    const int t = u, j = jmax - 1 - t, i = j % M;
    const bool last = t == m - 1;
    const int inext = last ? (jmin % M) : ((j - 1) % M);
    coef = rho[pm + i] * dotin;
    if (int(blockIdx.x) == r.lo && threadIdx.x == 0) alpha[pm + i] = coef;
    vec = Y + int64_t(i) * nd;
    dnext = last ? Y + int64_t(inext) * nd : S + int64_t(inext) * nd;
    scale = last;
  } else {
    const int t = u - m, j = jmin + t, i = j % M;
    const bool last = t == m - 1;
    const double beta = -rho[pm + i] * dotin;
    coef = alpha[pm + i] - beta;
    vec = S + int64_t(i) * nd;
    dnext = last ? nullptr : Y + int64_t((j + 1) % M) * nd;
    ls = last;
  }
  const double h0 = -s.H0;
  double v[2] = {0.0, 0.0};
  #pragma unroll 4
  for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) {
    double x = step[i] - coef * vec[i];
    if (scale) x *= h0;
    step[i] = x;
    if (ls) {
      v[0] += x * g[i];
      v[1] += x * x;
    } else {
      v[0] += dnext[i] * x;
    }
  }
  if (ls) {
    const int sl[2] = {B_SG, B_SS};
    item_partials<2>(v, part, nitems, sl);
  } else {
    double w[1] = {v[0]};
    const int sl[1] = {out_slot};
    item_partials<1>(w, part, nitems, sl);
  }
}

// Trial point (lbfgs.cpp:176-204): uphill steps inverted, capped at maxstep,
// halved nred times.
__global__ void __launch_bounds__(kBlThreads) bl_trial(const double* __restrict__ X, const double* __restrict__ step,
                                                       double* __restrict__ XT, const DofItem* __restrict__ items,
                                                       const BlState* __restrict__ st, const PatRange* __restrict__ pr,
                                                       BlParams prm, const double* __restrict__ part, int nitems) {
  const DofItem it = items[blockIdx.x];
  const BlState s = st[it.p];
  if (!s.active) return;
  const PatRange r = pr[it.p];
  const double sg = pat_sum(part + int64_t(B_SG) * nitems, r.lo, r.hi);
  const double ss = pat_sum(part + int64_t(B_SS) * nitems, r.lo, r.hi);
  const double sgn = sg > 0.0 ? -1.0 : 1.0;
  const double stepnorm = sqrt(ss);
  double factor = 1.0;
  if (factor * stepnorm > prm.maxstep) factor = prm.maxstep / stepnorm;
  for (int q = 0; q < s.nred; ++q) factor *= 0.5;
  #pragma unroll 4
  for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) XT[i] = X[i] + factor * (sgn * step[i]);
}

// After the evaluation: on acceptance the memory pair (s, y) goes into slot
// k mod M and the trial becomes the current point (lbfgs.cpp:74-84).
__global__ void __launch_bounds__(kBlThreads) bl_post(double* __restrict__ X, double* __restrict__ G,
                                                      const double* __restrict__ XT, const double* __restrict__ GT,
                                                      double* __restrict__ S, double* __restrict__ Y, int64_t nd,
                                                      const DofItem* __restrict__ items,
                                                      const BlState* __restrict__ st, const double* __restrict__ e,
                                                      BlParams prm, double* part, int nitems) {
  const DofItem it = items[blockIdx.x];
  const BlState s = st[it.p];
  if (!s.active || !bl_accept(s, e[it.p], prm)) return;
  const int kl = s.k % prm.M;
  double* sk = S + int64_t(kl) * nd;
  double* yk = Y + int64_t(kl) * nd;
  double v[3] = {0.0, 0.0, 0.0};
  #pragma unroll 4
  for (int64_t i = it.i0 + threadIdx.x; i < it.i1; i += blockDim.x) {
    const double gi = GT[i];
    const double yi = gi - G[i];
    const double xi = XT[i];
    const double si = xi - X[i];
    yk[i] = yi;
    sk[i] = si;
    X[i] = xi;
    G[i] = gi;
    v[0] += gi * gi;
    v[1] += yi * si;
    v[2] += yi * yi;
  }
  const int sl[3] = {B_GG, B_YS, B_YY};
  item_partials<3>(v, part, nitems, sl);
}

// Per-pattern state update (lbfgs.cpp:86-104, 206-245); one block per
// pattern sums the pattern's item partials.
__global__ void __launch_bounds__(kFinThreads) bl_finalize(BlState* st, const double* __restrict__ e, double* rho,
                                                           const PatRange* __restrict__ pr, BlParams prm,
                                                           const double* __restrict__ part, int nitems, int P) {
  const int p = blockIdx.x;
  BlState s = st[p];
  if (!s.active) return;  // uniform over the block
  const double fnew = e[p];
  const bool accept = bl_accept(s, fnew, prm);
  double tot[3] = {0.0, 0.0, 0.0};
  if (accept) {
    const int sl[3] = {B_GG, B_YS, B_YY};
    pattern_totals<3>(part, nitems, pr[p].lo, pr[p].hi, sl, tot);
  }
  if (threadIdx.x != 0) return;
  s.nfev += 1;
  if (accept) {
    const double gg = tot[0];
    double ys = tot[1], yy = tot[2];
    s.f = fnew;
    s.rms = sqrt(gg) * s.inv_sqrt_n;
    if (ys == 0.0) ys = 1.0;
    rho[int64_t(p) * prm.M + s.k % prm.M] = 1.0 / ys;
    if (yy == 0.0) yy = 1.0;
    s.H0 = ys / yy;
    s.k += 1;
    s.nred = 0;
    s.iter += 1;
    s.active = (s.rms > prm.tol) && (s.iter < s.stop_iter);
  } else {
    s.nred += 1;
  }
  st[p] = s;
}

}  // namespace

// One potential as a one-pattern ensemble: eval calls the potential's own
// launches (not its graph cache), so they are captured into the LBFGS step.
class PotentialEnsemble final : public Ensemble {
 public:
  PotentialEnsemble(PotentialPtr pot, int64_t n) : pot_(std::move(pot)) {
    if (pot_ && pot_->host_steps())
      throw InvalidArgument("a graph-captured optimiser cannot capture a potential that exchanges between processes");
    if (!pot_) throw InvalidArgument("null potential");
    if (n <= 0) throw InvalidArgument("empty coordinate array");
    if (pot_->ndof() >= 0 && pot_->ndof() != n) throw InvalidArgument("x0 has the wrong size for the potential");
    dof_off_ = {0, n};
  }
  void eval(const double* x, double* g, double* e, cudaStream_t s) override {
    if (g) {
      pot_->energy_gradient(x, ndof(), g, e, false, s);
    } else {
      pot_->energy(x, ndof(), e, false, s);
    }
  }
  void read_and_clear_status(int* out, cudaStream_t s) override { out[0] = pot_->read_and_clear_status(s); }
  void tune(const double*, double*, double*, cudaStream_t) override {}
  void set_split(double) override {}
  std::string describe() const override { return pot_->describe(); }

 private:
  PotentialPtr pot_;
};

struct EnsembleLbfgs::Impl {
  EnsemblePtr ens;
  EnsembleLbfgsParams prm;
  BlParams bp{};
  int P = 0, nitems = 0;
  int64_t nd = 0;
  DevBuf<double> X, G, XT, GT, step, S, Y, rho, alpha, E, part;
  DevBuf<BlState> st;
  DevBuf<DofItem> items;
  DevBuf<PatRange> pr;
  DevBuf<int> count;
  int* host_count = nullptr;
  cudaStream_t s = nullptr, cap = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_version = -1;
  // run(niter) as one launch: a conditional WHILE node repeating the step
  cudaGraphExec_t run_graph = nullptr;
  int run_graph_version = -1;
  bool run_graph_unavailable = false;
  DevBuf<int> guard;
  int* host_guard = nullptr;
  bool initialized = false;

  void initialize() {
    ens->eval(X.p, G.p, E.p, s);
    bl_dot_gg<<<nitems, kBlThreads, 0, s>>>(G.p, items.p, part.p, nitems);
    bl_init_fin<<<P, kFinThreads, 0, s>>>(st.p, E.p, pr.p, part.p, nitems, P, bp);
    FB_LAUNCH_CHECK();
    initialized = true;
  }

  void issue_step(cudaStream_t q) {
    bl_dir_start<<<nitems, kBlThreads, 0, q>>>(G.p, step.p, S.p, nd, items.p, st.p, bp.M, part.p, nitems);
    for (int u = 0; u < 2 * bp.M; ++u)
      bl_update<<<nitems, kBlThreads, 0, q>>>(u, step.p, G.p, S.p, Y.p, nd, items.p, st.p, pr.p, rho.p, alpha.p, bp.M,
                                              part.p, nitems);
    bl_trial<<<nitems, kBlThreads, 0, q>>>(X.p, step.p, XT.p, items.p, st.p, pr.p, bp, part.p, nitems);
    FB_LAUNCH_CHECK();
    ens->eval(XT.p, GT.p, E.p, q);
    bl_post<<<nitems, kBlThreads, 0, q>>>(X.p, G.p, XT.p, GT.p, S.p, Y.p, nd, items.p, st.p, E.p, bp, part.p,
                                          nitems);
    bl_finalize<<<P, kFinThreads, 0, q>>>(st.p, E.p, rho.p, pr.p, bp, part.p, nitems, P);
    FB_LAUNCH_CHECK();
  }

  void ensure_graph() {
    if (graph && graph_version == ens->version()) return;
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    if (!cap) FB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t gr = nullptr;
    FB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed));
    try {
      issue_step(cap);
    } catch (...) {
      cudaStreamEndCapture(cap, &gr);
      if (gr) cudaGraphDestroy(gr);
      throw;
    }
    FB_CUDA(cudaStreamEndCapture(cap, &gr));
    const cudaError_t ie = cudaGraphInstantiate(&graph, gr, 0);
    cudaGraphDestroy(gr);
    FB_CUDA(ie);
    graph_version = ens->version();
  }

  // Top graph: a check kernel, then a WHILE node whose body is one step and
  // the check.  Returns false (and keeps the host-driven loop) when this CUDA
  // build cannot capture the step into a conditional body.
  bool ensure_run_graph() {
    if (run_graph_unavailable) return false;
    if (run_graph && run_graph_version == ens->version()) return true;
    if (run_graph) {
      cudaGraphExecDestroy(run_graph);
      run_graph = nullptr;
    }
    if (!cap) FB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t top = nullptr;
    FB_CUDA(cudaGraphCreate(&top, 0));
    bool ok = false;
    try {
      cudaGraphConditionalHandle hw;
      FB_CUDA(cudaGraphConditionalHandleCreate(&hw, top, 0, cudaGraphCondAssignDefault));
      BlState* stp = st.p;
      int* gp = guard.p;
      int Pv = P, first = 1;
      void* pre_args[] = {&stp, &Pv, &gp, &hw, &first};
      cudaKernelNodeParams kp{};
      kp.func = reinterpret_cast<void*>(bl_loop);
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(256);
      kp.kernelParams = pre_args;
      cudaGraphNode_t pre;
      FB_CUDA(cudaGraphAddKernelNode(&pre, top, nullptr, 0, &kp));
      cudaGraphNodeParams wp{};
      wp.type = cudaGraphNodeTypeConditional;
      wp.conditional.handle = hw;
      wp.conditional.type = cudaGraphCondTypeWhile;
      wp.conditional.size = 1;
      cudaGraphNode_t wn;
      FB_CUDA(cudaGraphAddNode(&wn, top, &pre, 1, &wp));
      cudaGraph_t body = wp.conditional.phGraph_out[0];
      FB_CUDA(cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
      cudaGraph_t captured = nullptr;
      cudaError_t ce = cudaSuccess;
      try {
        issue_step(cap);
        bl_loop<<<1, 256, 0, cap>>>(st.p, P, guard.p, hw, 0);
        ce = cudaPeekAtLastError();
      } catch (...) {
        cudaStreamEndCapture(cap, &captured);
        throw;
      }
      const cudaError_t ee = cudaStreamEndCapture(cap, &captured);
      if (ce == cudaSuccess && ee == cudaSuccess) ok = cudaGraphInstantiate(&run_graph, top, 0) == cudaSuccess;
    } catch (const CudaError&) {
      ok = false;
    } catch (...) {
      cudaGraphDestroy(top);
      throw;
    }
    cudaGraphDestroy(top);
    if (!ok) {
      cudaGetLastError();  // capture and instantiation errors are not sticky
      run_graph = nullptr;
      run_graph_unavailable = true;
      return false;
    }
    run_graph_version = ens->version();
    return true;
  }

  int active_count() {
    bl_count_active<<<1, 256, 0, s>>>(st.p, P, count.p);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaMemcpyAsync(host_count, count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaStreamSynchronize(s));
    return *host_count;
  }
};

EnsembleLbfgs::EnsembleLbfgs(EnsemblePtr ens, const double* x0, int64_t n, const EnsembleLbfgsParams& p)
    : impl_(new Impl) {
  Impl& I = *impl_;
  if (!ens) throw InvalidArgument("null ensemble");
  if (n != ens->ndof()) throw InvalidArgument("x0 has the wrong size for the ensemble");
  if (p.M < 1) throw InvalidArgument("LBFGS memory M must be >= 1");
  I.ens = std::move(ens);
  I.prm = p;
  I.bp = BlParams{p.tol, p.maxstep, p.max_f_rise, p.M, p.rel_energy ? 1 : 0};
  I.P = P_ = I.ens->n_patterns();
  I.nd = n;
  const std::vector<int64_t>& off = I.ens->dof_offsets();
  std::vector<DofItem> items;
  std::vector<PatRange> pr(I.P);
  for (int q = 0; q < I.P; ++q) {
    pr[q].lo = int(items.size());
    for (int64_t i = off[q]; i < off[q + 1]; i += kBlChunk)
      items.push_back(DofItem{i, std::min<int64_t>(off[q + 1], i + kBlChunk), q, 0});
    pr[q].hi = int(items.size());
  }
  I.nitems = int(items.size());
  I.items.alloc(items.size());
  FB_CUDA(cudaMemcpy(I.items.p, items.data(), sizeof(DofItem) * items.size(), cudaMemcpyHostToDevice));
  I.pr.alloc(I.P);
  FB_CUDA(cudaMemcpy(I.pr.p, pr.data(), sizeof(PatRange) * I.P, cudaMemcpyHostToDevice));
  for (DevBuf<double>* b : {&I.X, &I.G, &I.XT, &I.GT, &I.step}) b->alloc(n);
  I.S.alloc(size_t(n) * p.M);
  I.Y.alloc(size_t(n) * p.M);
  I.rho.alloc(size_t(I.P) * p.M);
  I.alpha.alloc(size_t(I.P) * p.M);
  I.E.alloc(I.P);
  I.part.alloc(size_t(B_NSLOT) * I.nitems);
  I.count.alloc(1);
  FB_CUDA(cudaMemset(I.rho.p, 0, I.rho.bytes()));
  FB_CUDA(cudaMemset(I.alpha.p, 0, I.alpha.bytes()));
  FB_CUDA(cudaMemset(I.part.p, 0, I.part.bytes()));
  FB_CUDA(cudaMemset(I.step.p, 0, I.step.bytes()));
  FB_CUDA(cudaMemcpy(I.X.p, x0, sizeof(double) * n, cudaMemcpyHostToDevice));
  FB_CUDA(cudaMemcpy(I.XT.p, x0, sizeof(double) * n, cudaMemcpyHostToDevice));
  std::vector<BlState> hs(I.P);
  for (int q = 0; q < I.P; ++q) {
    BlState b{};
    b.f = 0.0;
    b.rms = 1e10;
    b.H0 = p.H0;
    const double nq = double(off[q + 1] - off[q]);
    b.inv_sqrt_n = 1.0 / std::sqrt(nq);
    b.inv_n = 1.0 / nq;
    hs[q] = b;
  }
  I.st.alloc(I.P);
  FB_CUDA(cudaMemcpy(I.st.p, hs.data(), sizeof(BlState) * I.P, cudaMemcpyHostToDevice));
  FB_CUDA(cudaMallocHost(&I.host_count, sizeof(int)));
  FB_CUDA(cudaMallocHost(&I.host_guard, sizeof(int)));
  I.guard.alloc(2);
  FB_CUDA(cudaStreamCreateWithFlags(&I.s, cudaStreamNonBlocking));
  FB_CUDA(cudaDeviceSynchronize());
}

EnsembleLbfgs::~EnsembleLbfgs() {
  Impl& I = *impl_;
  if (I.s) cudaStreamSynchronize(I.s);
  if (I.graph) cudaGraphExecDestroy(I.graph);
  if (I.run_graph) cudaGraphExecDestroy(I.run_graph);
  if (I.host_guard) cudaFreeHost(I.host_guard);
  if (I.cap) cudaStreamDestroy(I.cap);
  if (I.s) cudaStreamDestroy(I.s);
  if (I.host_count) cudaFreeHost(I.host_count);
}

void EnsembleLbfgs::steps(int n) {
  Impl& I = *impl_;
  if (n < 0) throw InvalidArgument("the step count must be >= 0");
  if (!I.initialized) I.initialize();
  bl_set_stop<<<int(ceil_div(I.P, 128)), 128, 0, I.s>>>(I.st.p, I.P, n, I.bp);
  FB_LAUNCH_CHECK();
  I.ensure_graph();
  for (int i = 0; i < n; ++i) FB_CUDA(cudaGraphLaunch(I.graph, I.s));
  FB_CUDA(cudaStreamSynchronize(I.s));
}

int EnsembleLbfgs::run(int niter) {
  Impl& I = *impl_;
  if (niter < 0) throw InvalidArgument("niter must be >= 0");
  if (!I.initialized) I.initialize();
  bl_set_stop<<<int(ceil_div(I.P, 128)), 128, 0, I.s>>>(I.st.p, I.P, niter, I.bp);
  FB_LAUNCH_CHECK();
  // every iteration takes at most ten evaluations
  const int64_t max_steps = int64_t(niter) * 10;
  if (max_steps < (int64_t(1) << 30) && I.ensure_run_graph()) {  // one launch for the whole run
    bl_guard_init<<<1, 1, 0, I.s>>>(I.guard.p, int(max_steps));
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaGraphLaunch(I.run_graph, I.s));
    FB_CUDA(cudaMemcpyAsync(I.host_guard, I.guard.p, sizeof(int), cudaMemcpyDeviceToHost, I.s));
    FB_CUDA(cudaStreamSynchronize(I.s));
    return *I.host_guard;
  }
  I.ensure_graph();
  int64_t taken = 0;
  int chunk = 2;
  while (taken < max_steps && I.active_count() > 0) {
    const int64_t k = std::min<int64_t>(chunk, max_steps - taken);
    for (int64_t i = 0; i < k; ++i) FB_CUDA(cudaGraphLaunch(I.graph, I.s));
    taken += k;
    chunk = std::min(chunk * 2, 16);
  }
  FB_CUDA(cudaStreamSynchronize(I.s));
  return int(taken);
}

void EnsembleLbfgs::get_state(double* x, double* g, double* f, double* rms, int* niter, int* nfev, int* active) {
  Impl& I = *impl_;
  if (!I.initialized) I.initialize();
  if (x) FB_CUDA(cudaMemcpyAsync(x, I.X.p, sizeof(double) * I.nd, cudaMemcpyDeviceToHost, I.s));
  if (g) FB_CUDA(cudaMemcpyAsync(g, I.G.p, sizeof(double) * I.nd, cudaMemcpyDeviceToHost, I.s));
  std::vector<BlState> hs(I.P);
  FB_CUDA(cudaMemcpyAsync(hs.data(), I.st.p, sizeof(BlState) * I.P, cudaMemcpyDeviceToHost, I.s));
  FB_CUDA(cudaStreamSynchronize(I.s));
  for (int q = 0; q < I.P; ++q) {
    if (f) f[q] = hs[q].f;
    if (rms) rms[q] = hs[q].rms;
    if (niter) niter[q] = hs[q].iter;
    if (nfev) nfev[q] = hs[q].nfev;
    if (active) active[q] = hs[q].active;
  }
}

EnsemblePtr make_potential_ensemble(std::shared_ptr<Potential> pot, int64_t n) {
  return EnsemblePtr(new PotentialEnsemble(std::move(pot), n));
}

}  // namespace fb
