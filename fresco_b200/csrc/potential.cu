// Potential base-class services and CombinedPotential.
#include "potential.cuh"

namespace fb {

void Potential::init_status() {
  FB_CUDA(cudaGetDevice(&device));
  status_.alloc(1);
  FB_CUDA(cudaMemset(status_.p, 0, sizeof(int)));
}

int Potential::read_and_clear_status(cudaStream_t s) {
  if (!status_.p) return 0;
  int h = 0;
  FB_CUDA(cudaMemcpyAsync(&h, status_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FB_CUDA(cudaMemsetAsync(status_.p, 0, sizeof(int), s));
  FB_CUDA(cudaStreamSynchronize(s));
  return h;
}

void Potential::timer_begin(cudaStream_t s) {
  if (!timer.enabled) return;
  timer.next = 0;
  timer_mark("__begin", s);
}

void Potential::timer_mark(const char* name, cudaStream_t s) {
  if (!timer.enabled) return;
  const int i = timer.next++;
  if (i >= int(timer.ev.size())) {
    cudaEvent_t e;
    FB_CUDA(cudaEventCreate(&e));
    timer.ev.push_back(e);
    timer.names.push_back(name);
    timer.total_ms.push_back(0.0);
    timer.count.push_back(0);
  }
  timer.names[i] = name;
  FB_CUDA(cudaEventRecord(timer.ev[i], s));
}

void Potential::timer_collect() {
  if (!timer.enabled || timer.next < 2) return;
  FB_CUDA(cudaEventSynchronize(timer.ev[timer.next - 1]));
  for (int i = 1; i < timer.next; ++i) {
    float ms = 0.f;
    FB_CUDA(cudaEventElapsedTime(&ms, timer.ev[i - 1], timer.ev[i]));
    timer.total_ms[i] += ms;
    timer.count[i] += 1;
  }
  timer.next = 0;
}

CombinedPotential::CombinedPotential() { init_status(); }

void CombinedPotential::add(PotentialPtr p) {
  if (!p) throw InvalidArgument("cannot add a null potential");
  parts_.push_back(std::move(p));
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
  bool first = true;
  for (auto& p : parts_) {
    p->energy_gradient(x, n, g, e, acc || !first, s);
    first = false;
  }
}

int CombinedPotential::read_and_clear_status(cudaStream_t s) {
  int st = 0;
  for (auto& p : parts_) st |= p->read_and_clear_status(s);
  return st;
}

}  // namespace fb
