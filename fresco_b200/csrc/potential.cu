// Potential base-class services and CombinedPotential.
#include "potential.cuh"

namespace fb {

Potential::~Potential() {
  invalidate_graphs();
  if (capture_stream_) cudaStreamDestroy(capture_stream_);
}

void Potential::invalidate_graphs() {
  for (auto& ge : graphs_)
    if (ge.exec) cudaGraphExecDestroy(ge.exec);
  graphs_.clear();
}

void Potential::set_graphs_enabled(bool on) {
  graphs_enabled_ = on;
  if (!on) invalidate_graphs();
}

void Potential::eval(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) {
  auto direct = [&](cudaStream_t st) {
    struct Flag {
      bool& f;
      explicit Flag(bool& r) : f(r) { f = true; }
      ~Flag() { f = false; }
    } in_eval(in_eval_);
    if (g) energy_gradient(x, n, g, e, acc, st);
    else energy(x, n, e, acc, st);
  };
  if (!graphs_enabled_ || timing_active() || host_steps()) {
    direct(s);
    return;
  }
  ++graph_clock_;
  GraphEntry* hit = nullptr;
  for (auto& ge : graphs_)
    if (ge.x == x && ge.g == g && ge.e == e && ge.n == n && ge.acc == acc && ge.mode == grad_mode_) hit = &ge;
  if (hit && hit->exec) {
    hit->last_use = graph_clock_;
    FB_CUDA(cudaGraphLaunch(hit->exec, s));
    return;
  }
  if (!hit) {  // first sighting: remember the key, run directly
    if (graphs_.size() == kMaxGraphs) {
      size_t old = 0;
      for (size_t i = 1; i < graphs_.size(); ++i)
        if (graphs_[i].last_use < graphs_[old].last_use) old = i;
      if (graphs_[old].exec) cudaGraphExecDestroy(graphs_[old].exec);
      graphs_.erase(graphs_.begin() + old);
    }
    graphs_.push_back(GraphEntry{x, g, e, n, acc, grad_mode_, graph_clock_, nullptr});
    direct(s);
    return;
  }
  // second sighting: capture on the private stream, then launch on s
  if (!capture_stream_) FB_CUDA(cudaStreamCreateWithFlags(&capture_stream_, cudaStreamNonBlocking));
  FB_CUDA(cudaStreamBeginCapture(capture_stream_, cudaStreamCaptureModeRelaxed));
  cudaGraph_t graph = nullptr;
  try {
    direct(capture_stream_);
  } catch (...) {
    cudaStreamEndCapture(capture_stream_, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  FB_CUDA(cudaStreamEndCapture(capture_stream_, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t rc = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  FB_CUDA(rc);
  hit->exec = exec;
  hit->last_use = graph_clock_;
  FB_CUDA(cudaGraphLaunch(exec, s));
}

void Potential::init_status() {
  FB_CUDA(cudaGetDevice(&device));
  status_.alloc(2);
  FB_CUDA(cudaMemset(status_.p, 0, 2 * sizeof(int)));
}

int Potential::read_and_clear_status(cudaStream_t s) {
  if (!status_.p) return 0;
  int h = 0;
  FB_CUDA(cudaMemcpyAsync(&h, status_.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaMemsetAsync(status_.p + 1, 0, sizeof(int), s));
  FB_CUDA(cudaStreamSynchronize(s));
  return h;
}

void Potential::timer_begin(cudaStream_t s) {
  if (!timer.enabled) return;
  if (timer.used == int(timer.sets.size())) {
    timer.sets.emplace_back();
    timer.names.emplace_back();
  }
  timer.names[timer.used].clear();
  ++timer.used;
  timer_mark("__begin", s);
}

void Potential::timer_mark(const char* name, cudaStream_t s) {
  if (!timer.enabled || timer.used == 0) return;
  auto& set = timer.sets[timer.used - 1];
  auto& nm = timer.names[timer.used - 1];
  const size_t i = nm.size();
  if (i >= set.size()) {
    cudaEvent_t e;
    FB_CUDA(cudaEventCreate(&e));
    set.push_back(e);
  }
  nm.push_back(name);
  FB_CUDA(cudaEventRecord(set[i], s));
}

void Potential::timer_collect() {
  for (int u = 0; u < timer.used; ++u) {
    auto& set = timer.sets[u];
    auto& nm = timer.names[u];
    if (nm.size() < 2) continue;
    FB_CUDA(cudaEventSynchronize(set[nm.size() - 1]));
    for (size_t i = 1; i < nm.size(); ++i) {
      float ms = 0.f;
      FB_CUDA(cudaEventElapsedTime(&ms, set[i - 1], set[i]));
      size_t k = 0;
      while (k < timer.total_names.size() && timer.total_names[k] != nm[i]) ++k;
      if (k == timer.total_names.size()) {
        timer.total_names.push_back(nm[i]);
        timer.total_ms.push_back(0.0);
        timer.count.push_back(0);
      }
      timer.total_ms[k] += ms;
      timer.count[k] += 1;
    }
  }
  timer.used = 0;
}

namespace {
__global__ void add_scalar_kernel(const double* __restrict__ src, double* dst) { *dst += *src; }
}  // namespace

void add_scalar(const double* src, double* dst, cudaStream_t s) {
  add_scalar_kernel<<<1, 1, 0, s>>>(src, dst);
  FB_LAUNCH_CHECK();
}

namespace {
// g[i] += side[0][i] + side[1][i] + ... (in part order), e += the side energies.
__global__ void combine_sides_kernel(double* g, int64_t n, const double* __restrict__ side, int nside, double* e,
                                     const double* __restrict__ se) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double v = g[i];
    for (int k = 0; k < nside; ++k) v += side[int64_t(k) * n + i];
    g[i] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double v = *e;
    for (int k = 0; k < nside; ++k) v += se[k];
    *e = v;
  }
}
}  // namespace

CombinedPotential::CombinedPotential() { init_status(); }

CombinedPotential::~CombinedPotential() {
  for (cudaStream_t st : side_) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t ev : done_) cudaEventDestroy(ev);
  if (fork_) cudaEventDestroy(fork_);
}

void CombinedPotential::add(PotentialPtr p) {
  if (!p) throw InvalidArgument("cannot add a null potential");
  parts_.push_back(std::move(p));
  invalidate_graphs();
  const int64_t n = ndof();
  if (parts_.size() >= 2 && n > 0) prepare_side(n);
}

// Side streams, events and scratch for the parts after the first, made when
// a part is added (never on the evaluation path).
void CombinedPotential::prepare_side(int64_t n) {
  const size_t nside = parts_.size() - 1;
  if (!fork_) FB_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  while (side_.size() < nside) {
    cudaStream_t st;
    cudaEvent_t ev;
    FB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    FB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    side_.push_back(st);
    done_.push_back(ev);
  }
  if (scr_n_ != n || gscr_.n < size_t(n) * nside) {
    FB_CUDA(cudaDeviceSynchronize());  // no launch may still use the old scratch
    gscr_.alloc(size_t(n) * nside);
    escr_.alloc(nside);
    scr_n_ = n;
  }
}

bool CombinedPotential::timing_active() const {
  if (timer.enabled) return true;
  for (auto& p : parts_)
    if (p->timing_active()) return true;
  return false;
}

int64_t CombinedPotential::ndof() const {
  int64_t n = -1;
  for (auto& p : parts_) n = std::max(n, p->ndof());
  return n;
}

void CombinedPotential::energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) {
  if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
  for (auto& p : parts_) p->energy(x, n, e, true, s);
}

void CombinedPotential::energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc,
                                        cudaStream_t s) {
  // combine_potentials.hpp:43-57: zero, then add every part.
  if (!acc) {
    FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    if (parts_.empty()) FB_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * n, s));
  }
  const size_t nside = parts_.empty() ? 0 : parts_.size() - 1;
  if (!in_eval_ || nside == 0 || n != scr_n_ || side_.size() < nside || host_steps() || timing_active()) {
    bool first = true;
    for (auto& p : parts_) {
      p->energy_gradient(x, n, g, e, acc || !first, s);
      first = false;
    }
    return;
  }
  // The parts are independent until their results are summed: the first runs
  // on s into g and e, the others at the same time on side streams into their
  // own scratch, then the scratch is added in part order, which gives the
  // same sums as adding the parts one after another.
  FB_CUDA(cudaEventRecord(fork_, s));
  for (size_t k = 0; k < nside; ++k) {
    FB_CUDA(cudaStreamWaitEvent(side_[k], fork_, 0));
    parts_[k + 1]->energy_gradient(x, n, gscr_.p + int64_t(k) * n, escr_.p + k, false, side_[k]);
    FB_CUDA(cudaEventRecord(done_[k], side_[k]));
  }
  parts_[0]->energy_gradient(x, n, g, e, acc, s);
  for (size_t k = 0; k < nside; ++k) FB_CUDA(cudaStreamWaitEvent(s, done_[k], 0));
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), int64_t(sm_count()) * 4)));
  combine_sides_kernel<<<grid, 256, 0, s>>>(g, n, gscr_.p, int(nside), e, escr_.p);
  FB_LAUNCH_CHECK();
}

void CombinedPotential::set_gradient_mode(int mode) {
  grad_mode_ = mode;
  for (auto& p : parts_) p->set_gradient_mode(mode);
}

int CombinedPotential::read_and_clear_status(cudaStream_t s) {
  int st = 0;
  for (auto& p : parts_) st |= p->read_and_clear_status(s);
  return st;
}

}  // namespace fb
