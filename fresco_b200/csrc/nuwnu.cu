// NUwNU: structure-factor loss of a point pattern at non-uniform k-points
// (source/fresco/nuwnu.hpp:17-291).
//
// Reference semantics: x_j = (p_j - round(p_j/L) + L) 2 pi / L in both the
// energy and the gradient (nuwnu.hpp:134, 193), frequencies s_k = K_k used
// as given (no 2 pi / L, nuwnu.hpp:47-76), rho_k = sum_j c_j exp(+i s_k.x_j)
// (type 3, iflag +1), S = |rho|^2/N, d = (S - S0)/S0', phi = sum V d^2,
// factor_k = (-4i/N) V d rho / S0' and grad[D j + a] =
// Re(sum_k s_k[a] factor_k exp(-i s_k.x_j)) (type 3, iflag -1; the reference
// omits conj(c_j) here, nuwnu.hpp:269, and so does this implementation).
//
// B200 form: both transforms are evaluated as exact FP64 direct sums, O(N M),
// which is the fastest form for the few-peak targets this loss is used with
// (examples/NUwNU.ipynb: 5 k-points) and more accurate than a type-3 NUFFT.
// The forward sum runs over (point chunks) x (frequency chunks) with block
// reductions; the adjoint is one thread per point with the frequencies
// staged in shared memory.  The `precision` argument is accepted; the
// arithmetic is FP64 either way.
#include <cuda.h>

#include <cmath>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "potential.cuh"
#include "type3.cuh"

namespace fb {

namespace {

constexpr int kThreads = 256;
constexpr int kFreqChunk = 8;    // frequencies per block in the forward sum
constexpr int kAdjTile = 512;    // frequencies staged per shared-memory tile in the adjoint
constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ double nuwnu_coord(const double* __restrict__ p, int64_t j, int a, int D, double L) {
  const double v = p[j * D + a];
  return (v - round(v / L) + L) * 2 * kPi / L;  // nuwnu.hpp:134 / 193, same operation order
}

template <int D>
__global__ void __launch_bounds__(kThreads) nuwnu_forward_kernel(const double* __restrict__ pts, int64_t N,
                                                                  const double* __restrict__ s, int64_t M,
                                                                  const double* __restrict__ c, double cu,
                                                                  double L0, double L1, double L2, double2* rho,
                                                                  int* status, const int* __restrict__ only_if) {
  if (only_if != nullptr && *only_if == 0) return;  // runs only when the type-3 path declined this evaluation
  // frequency chunks k0 = blockIdx.y * kFreqChunk + gridDim.y * kFreqChunk * t
  // (gridDim.y is capped at the launch limit, 65535)
  __shared__ double red[2 * kFreqChunk][kThreads / 32];
  bool bad = false;
  for (int64_t k0 = int64_t(blockIdx.y) * kFreqChunk; k0 < M; k0 += int64_t(gridDim.y) * kFreqChunk) {
    double sk[kFreqChunk][D];
#pragma unroll
    for (int q = 0; q < kFreqChunk; ++q)
#pragma unroll
      for (int a = 0; a < D; ++a) sk[q][a] = (k0 + q < M) ? s[(k0 + q) * D + a] : 0.0;
    double re[kFreqChunk], im[kFreqChunk];
#pragma unroll
    for (int q = 0; q < kFreqChunk; ++q) re[q] = im[q] = 0.0;
    const double Ls[3] = {L0, L1, L2};
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
      double x[D];
#pragma unroll
      for (int a = 0; a < D; ++a) {
        x[a] = nuwnu_coord(pts, j, a, D, Ls[a]);
        bad |= !isfinite(x[a]);
      }
      const double cj = c ? c[j] : cu;
#pragma unroll
      for (int q = 0; q < kFreqChunk; ++q) {
        double ph = 0.0;
#pragma unroll
        for (int a = 0; a < D; ++a) ph += sk[q][a] * x[a];
        double sn, cs;
        sincos(ph, &sn, &cs);
        re[q] += cj * cs;
        im[q] += cj * sn;
      }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();  // the previous chunk's partial sums have been read
#pragma unroll
    for (int q = 0; q < kFreqChunk; ++q) {
      const double a = warp_sum(re[q]), b = warp_sum(im[q]);
      if (lane == 0) {
        red[2 * q][wid] = a;
        red[2 * q + 1][wid] = b;
      }
    }
    __syncthreads();
    if (threadIdx.x < 2 * kFreqChunk) {
      double t = 0.0;
      for (int w = 0; w < int(blockDim.x) / 32; ++w) t += red[threadIdx.x][w];
      const int q = threadIdx.x / 2;
      if (k0 + q < M) atomicAdd((threadIdx.x & 1) ? &rho[k0 + q].y : &rho[k0 + q].x, t);
    }
  }
  if (bad && blockIdx.y == 0) raise_status(status, STATUS_NONFINITE_INPUT);
}

__global__ void __launch_bounds__(kThreads) nuwnu_loss_kernel(const double2* __restrict__ rho, int64_t M, double invN,
                                                              const double* __restrict__ sk,
                                                              const double* __restrict__ v, double* energy,
                                                              double2* factor, const int* __restrict__ status) {
  double phi = 0.0;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < M; k += int64_t(gridDim.x) * blockDim.x) {
    const double2 r = rho[k];
    const double s0 = sk[k];
    const double dn = s0 != 0.0 ? s0 : 1.0;
    const double d = ((r.x * r.x + r.y * r.y) * invN - s0) / dn;
    phi += v[k] * d * d;
    // factor = (-4i/N) V d rho / S0'
    const double a = 4.0 * invN * v[k] * d / dn;
    factor[k] = make_double2(a * r.y, -a * r.x);
  }
  block_sum_atomic(phi, energy);
  if (blockIdx.x == 0 && threadIdx.x == 0 && ((*status) & STATUS_NONFINITE_INPUT))
    atomicAdd(energy, __longlong_as_double(0x7ff8000000000000ULL));
}

template <int D>
__global__ void __launch_bounds__(kThreads) nuwnu_adjoint_kernel(const double* __restrict__ pts, int64_t N,
                                                                  const double* __restrict__ s, int64_t M,
                                                                  const double2* __restrict__ factor, double L0,
                                                                  double L1, double L2, double* grad, int accumulate,
                                                                  const int* __restrict__ status,
                                                                  const double* __restrict__ c, double cu, int exact,
                                                                  const int* __restrict__ only_if) {
  if (only_if != nullptr && *only_if == 0) return;  // runs only when the type-3 path declined this evaluation
  __shared__ double ss[kAdjTile * D];
  __shared__ double2 sf[kAdjTile];
  const double Ls[3] = {L0, L1, L2};
  const bool bad = (*status) & STATUS_NONFINITE_INPUT;
  for (int64_t base = int64_t(blockIdx.x) * blockDim.x; base < N; base += int64_t(gridDim.x) * blockDim.x) {
    const int64_t j = base + threadIdx.x;
    const bool active = j < N;
    double x[D], g[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      x[a] = active ? nuwnu_coord(pts, j, a, D, Ls[a]) : 0.0;
      g[a] = 0.0;
    }
    for (int64_t t0 = 0; t0 < M; t0 += kAdjTile) {
      __syncthreads();
      const int cnt = int((M - t0) < kAdjTile ? (M - t0) : kAdjTile);
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
#pragma unroll
        for (int a = 0; a < D; ++a) ss[q * D + a] = s[(t0 + q) * D + a];
        sf[q] = factor[t0 + q];
      }
      __syncthreads();
      if (active) {
        for (int q = 0; q < cnt; ++q) {
          double ph = 0.0;
#pragma unroll
          for (int a = 0; a < D; ++a) ph += ss[q * D + a] * x[a];
          double sn, cs;
          sincos(-ph, &sn, &cs);
          const double2 fq = sf[q];
          const double re = fq.x * cs - fq.y * sn;  // Re(factor * exp(-i ph))
#pragma unroll
          for (int a = 0; a < D; ++a) g[a] += ss[q * D + a] * re;
        }
      }
    }
    if (active) {
      const double nan = __longlong_as_double(0x7ff8000000000000ULL);
      // exact derivative: c_j * (2 pi / L) times the reference's value
      const double cj = exact ? (c ? c[j] : cu) : 1.0;
#pragma unroll
      for (int a = 0; a < D; ++a) {
        double* dst = grad + j * D + a;
        const double v = bad ? nan : (exact ? g[a] * cj * 2 * kPi / Ls[a] : g[a]);
        *dst = accumulate ? *dst + v : v;
      }
    }
  }
}

// Type-3 path helpers.  rho is zeroed for the direct fallback when the
// window flag says the type-3 result is not to be used.
__global__ void nuwnu_zero_if_kernel(double2* rho, int64_t M, const int* __restrict__ flag, int* status) {
  if (*flag == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(status, STATUS_EXACT_FALLBACK);
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < M; k += int64_t(gridDim.x) * blockDim.x)
    rho[k] = make_double2(0.0, 0.0);
}

// Adjoint strengths: vector a holds s_k[a] factor_k (nuwnu.hpp:231-282).
__global__ void __launch_bounds__(kThreads) nuwnu_t3_strength_kernel(const double* __restrict__ s, int64_t M, int D,
                                                                     const double2* __restrict__ factor,
                                                                     double2* str) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < M * D; i += int64_t(gridDim.x) * blockDim.x) {
    const int a = int(i / M);
    const int64_t k = i - int64_t(a) * M;
    const double2 f = factor[k];
    const double sa = s[k * D + a];
    str[i] = make_double2(sa * f.x, sa * f.y);
  }
}

// grad[D j + a] (+)= Re(out_a(x_j)) (nuwnu.hpp:269, no conj(c_j)); the exact
// derivative multiplies by c_j 2 pi / L.  Skipped when the window flag sent
// the evaluation to the direct sums.
__global__ void __launch_bounds__(kThreads) nuwnu_t3_grad_kernel(const double2* __restrict__ out, int64_t N, int D,
                                                                 const int* __restrict__ flag,
                                                                 const int* __restrict__ status,
                                                                 const double* __restrict__ c, double cu, int exact,
                                                                 double L0, double L1, double L2, double* grad,
                                                                 int accumulate) {
  if (*flag != 0) return;
  const bool bad = (*status) & STATUS_NONFINITE_INPUT;
  const double Ls[3] = {L0, L1, L2};
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N * D; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t j = i / D;
    const int a = int(i - j * D);
    double v = out[int64_t(a) * N + j].x;
    if (exact) v *= (c ? c[j] : cu) * 2 * kPi / Ls[a];
    if (bad) v = __longlong_as_double(0x7ff8000000000000ULL);
    grad[i] = accumulate ? grad[i] + v : v;
  }
}

// Evaluations with at least this many (point, k-point) pairs use the type-3
// NUFFT; fewer are cheaper as direct sums.
constexpr double kType3MinPairs = double(1 << 22);

// Range of the reference's coordinate map x = (p - round(p/L) + L) 2 pi / L
// (nuwnu.hpp:134) over p in [-L, 2L): the window the type-3 plans cover.
// Points beyond it send that evaluation to the direct sums.
void nuwnu_map_window(double L, double& lo, double& hi) {
  lo = INFINITY;
  hi = -INFINITY;
  for (int k = -1; k <= 2; ++k) {
    const double pl = std::max(-L, (k - 0.5) * L), ph = std::min(2.0 * L, (k + 0.5) * L);
    if (!(ph > pl)) continue;
    for (double p : {pl, ph}) {
      const double x = (p - k + L) * 2 * kPi / L;
      lo = std::min(lo, x);
      hi = std::max(hi, x);
    }
  }
  const double m = 1e-9 * (hi - lo) + 1e-12;
  lo -= m;
  hi += m;
}

template <int D, typename T>
class NUwNUImpl final : public Potential {
 public:
  NUwNUImpl(const std::vector<double>& radii, const std::vector<double>& kpts, const std::vector<double>& sk,
            const std::vector<double>& v, const std::vector<double>& L, double eps)
      : N_(int64_t(radii.size())) {
    init_status();
    if (sk.size() != v.size()) throw InvalidArgument("len(Sk) must equal len(V)");
    M_ = int64_t(kpts.size()) / D;  // nuwnu.hpp:40
    if (int64_t(sk.size()) < M_) throw InvalidArgument("Sk/V need one value per k-point");
    for (int a = 0; a < D; ++a) L_[a] = L[a];
    // weights, nuwnu.hpp:81-105 (area factor applied once per dimension)
    std::vector<double> c(radii.size(), 1.0);
    double sum = 0.0;
    for (size_t i = 0; i < c.size(); ++i) {
      for (int j = 0; j < D; ++j) {
        if (D == 2) c[i] = c[i] * M_PI * radii[i] * radii[i];
        else if (D == 3) c[i] = c[i] * M_PI * radii[i] * radii[i] * radii[i] * 4.0 / 3.0;
      }
      sum += c[i];
    }
    bool uniform = true;
    for (size_t i = 0; i < c.size(); ++i) {
      c[i] *= double(c.size()) / sum;
      if (c[i] != c[0]) uniform = false;
    }
    if (uniform && !c.empty()) {
      cu_ = c[0];
    } else if (!c.empty()) {
      c_.alloc(c.size());
      FB_CUDA(cudaMemcpy(c_.p, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
    }
    s_.alloc(std::max<int64_t>(M_ * D, 1));
    sk_.alloc(std::max<int64_t>(M_, 1));
    v_.alloc(std::max<int64_t>(M_, 1));
    rho_.alloc(std::max<int64_t>(M_, 1));
    factor_.alloc(std::max<int64_t>(M_, 1));
    if (M_) {
      FB_CUDA(cudaMemcpy(s_.p, kpts.data(), sizeof(double) * M_ * D, cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(sk_.p, sk.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(v_.p, v.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
    }
    // type-3 NUFFT plans: forward (points -> k-points, iflag +1, nuwnu.hpp:77,
    // 165) and adjoint (k-points -> points, iflag -1, nuwnu.hpp:78, 231-282);
    // the k-points are sorted and their factors computed once here
    if (N_ > 0 && M_ > 0 && double(N_) * double(M_) >= kType3MinPairs) {
      double xlo[3], xhi[3], klo[3], khi[3];
      for (int a = 0; a < D; ++a) {
        nuwnu_map_window(L_[a], xlo[a], xhi[a]);
        klo[a] = INFINITY;
        khi[a] = -INFINITY;
        for (int64_t k = 0; k < M_; ++k) {
          klo[a] = std::min(klo[a], kpts[size_t(k * D + a)]);
          khi[a] = std::max(khi[a], kpts[size_t(k * D + a)]);
        }
        if (!std::isfinite(klo[a]) || !std::isfinite(khi[a])) throw InvalidArgument("non-finite k-point");
      }
      fwd_.reset(new Type3<T>(D, N_, M_, xlo, xhi, klo, khi, +1, eps, 1));
      adj_.reset(new Type3<T>(D, M_, N_, klo, khi, xlo, xhi, -1, eps, D));
      fwd_->set_targets(s_.p, TYPE3_IDENTITY, nullptr, nullptr);
      adj_->set_sources(s_.p, TYPE3_IDENTITY, nullptr, nullptr);
      t3str_.alloc(M_ * D);
      t3out_.alloc(N_ * D);
      FB_CUDA(cudaDeviceSynchronize());
    }
  }

  int64_t ndof() const override { return N_ * D; }
  std::string kind() const override { return "NUwNU"; }
  std::string describe() const override {
    std::string s = "NUwNU D=" + std::to_string(D) + " N=" + std::to_string(N_) + " kpoints=" + std::to_string(M_);
    if (fwd_)
      s += std::string(" precision=") + (sizeof(T) == 4 ? "fp32" : "fp64") + " forward " + fwd_->describe() +
           " adjoint " + adj_->describe() + " (exact sums for points outside the planned window)";
    else
      s += " exact FP64 direct sums";
    return s;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override { run(x, nullptr, e, acc, s); }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    timer_begin(s);
    begin_eval_status(s);
    if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    if (M_ == 0 || N_ == 0) {
      if (g && !acc) FB_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * N_ * D, s));
      return;
    }
    const int pblocks = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(N_, kThreads), 2 * int64_t(sm_count()))));
    dim3 fg(pblocks, unsigned(std::min<int64_t>(ceil_div(M_, kFreqChunk), 65535)));
    const int mg = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(M_, kThreads), int64_t(sm_count()) * 4)));
    const int* flag = nullptr;
    if (fwd_) {
      // type 3; the direct sums run instead when a point is outside the plans' window
      fwd_->set_sources(x, TYPE3_NUWNU_MAP, L_, s);
      fwd_->execute_real(c_.p, cu_, rho_.p, s);
      flag = fwd_->window_flag();
      nuwnu_zero_if_kernel<<<mg, kThreads, 0, s>>>(rho_.p, M_, flag, status_.p);
      FB_LAUNCH_CHECK();
      // the direct sums below only run when the flag is set; a modest grid
      // (the kernel strides over the frequency chunks) keeps the launch that
      // exits at once cheap
      fg.y = std::min(fg.y, 64u);
    } else {
      FB_CUDA(cudaMemsetAsync(rho_.p, 0, sizeof(double2) * M_, s));
    }
    nuwnu_forward_kernel<D><<<fg, kThreads, 0, s>>>(x, N_, s_.p, M_, c_.p, cu_, L_[0], L_[1], L_[2], rho_.p,
                                                    status_.p, flag);
    FB_LAUNCH_CHECK();
    nuwnu_loss_kernel<<<mg, kThreads, 0, s>>>(rho_.p, M_, 1.0 / double(N_), sk_.p, v_.p, e, factor_.p, status_.p);
    FB_LAUNCH_CHECK();
    timer_mark("forward", s);
    if (!g) return;
    const int ag = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(N_, kThreads), int64_t(sm_count()) * 8)));
    if (adj_) {
      const int sg = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(M_ * D, kThreads), int64_t(sm_count()) * 8)));
      nuwnu_t3_strength_kernel<<<sg, kThreads, 0, s>>>(s_.p, M_, D, factor_.p, t3str_.p);
      FB_LAUNCH_CHECK();
      adj_->set_targets(x, TYPE3_NUWNU_MAP, L_, s);
      adj_->execute_cplx(t3str_.p, t3out_.p, s);
      nuwnu_t3_grad_kernel<<<ag, kThreads, 0, s>>>(t3out_.p, N_, D, flag, status_.p, c_.p, cu_,
                                                   grad_mode_ == 1 ? 1 : 0, L_[0], L_[1], L_[2], g, acc ? 1 : 0);
      FB_LAUNCH_CHECK();
    }
    nuwnu_adjoint_kernel<D><<<ag, kThreads, 0, s>>>(x, N_, s_.p, M_, factor_.p, L_[0], L_[1], L_[2], g,
                                                    acc ? 1 : 0, status_.p, c_.p, cu_, grad_mode_ == 1 ? 1 : 0, flag);
    FB_LAUNCH_CHECK();
    timer_mark("adjoint", s);
  }

  int64_t N_, M_ = 0;
  double L_[3] = {1, 1, 1};
  double cu_ = 1.0;
  DevBuf<double> c_, s_, sk_, v_;
  DevBuf<double2> rho_, factor_;
  std::unique_ptr<Type3<T>> fwd_, adj_;  // null: direct sums only
  DevBuf<double2> t3str_, t3out_;        // adjoint strengths (D x M), outputs (D x N)
};

}  // namespace

// ---- allocation-free form --------------------------------------------------
//
// fresco_nuwnu_energy_gradient_noalloc evaluates the same loss and gradient as
// a NUwNU handle without any device allocation: no handle is created, the
// caller's device arrays are read directly, and the per-k-point sums (rho and
// the loss factor) plus the status word live in the file-scope array below.
// The array is part of the library's device image, so every GPU that loads
// the library holds its 128 KiB until the process exits.  All calls share it:
// two calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on it and both results are undefined.
constexpr int64_t kNoAllocMaxK = 4096;
static __device__ __align__(256) double2 g_nuwnu_noalloc_scratch[2 * kNoAllocMaxK + 1];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
struct NoAllocSlot {
  unsigned long long ctx_id = 0;  // CUDA context the address belongs to (0: none yet)
  double2* ptr = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

// Unique id of the calling thread's current CUDA context (cuCtxGetCurrent,
// cuCtxGetId from the driver), or 0 when the driver offers no id.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static const std::pair<GetCurrent, GetId> fns = [] {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    const bool ok = cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
                    qa == cudaDriverEntryPointSuccess &&
                    cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
                    qb == cudaDriverEntryPointSuccess;
    if (!ok) {
      cudaGetLastError();
      return std::pair<GetCurrent, GetId>(nullptr, nullptr);
    }
    return std::pair<GetCurrent, GetId>(reinterpret_cast<GetCurrent>(a), reinterpret_cast<GetId>(b));
  }();
  if (!fns.first) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (fns.first(&ctx) != CUDA_SUCCESS || !ctx || fns.second(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the current device's context.  The
// first call in a context looks it up (cudaGetSymbolAddress, which may load
// the library's device code into that context); later calls in the same
// context reuse the cached address.  A new context on the device (after
// cudaDeviceReset, or a caller that makes another context current) gets its
// own lookup, so a cached address is never used outside the context it
// belongs to.
double2* noalloc_scratch_on_current_device() {
  int dev = -1;
  FB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    throw std::runtime_error("device index " + std::to_string(dev) + " is beyond the " +
                             std::to_string(kNoAllocMaxDevices) + " devices the allocation-free entry point supports");
  const unsigned long long ctx = current_context_id();  // 0 before the runtime has made a context current
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocSlot& slot = g_noalloc_slot[dev];
  if (!slot.ptr || ctx == 0 || slot.ctx_id != ctx) {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_nuwnu_noalloc_scratch);
    if (rc != cudaSuccess || !ptr)
      throw std::runtime_error(std::string("cudaGetSymbolAddress of the NUwNU scratch array failed: ") +
                               cudaGetErrorString(rc));
    slot.ptr = static_cast<double2*>(ptr);
    slot.ctx_id = current_context_id();  // the lookup made the device's context current
  }
  return slot.ptr;
}

template <int D>
void noalloc_launch(const double* x, int64_t N, const double* c, const double* s, const double* sk, const double* v,
                    int64_t M, const double* L, int mode, double* g, double* e, bool acc, double2* scratch,
                    cudaStream_t st) {
  double2* rho = scratch;
  double2* factor = scratch + kNoAllocMaxK;
  int* status = reinterpret_cast<int*>(scratch + 2 * kNoAllocMaxK);
  // the array keeps the previous call's sums and status: clear what must start at zero
  FB_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(int), st));
  if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), st));
  if (M == 0 || N == 0) {
    if (g && !acc) FB_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * N * D, st));
    return;
  }
  FB_CUDA(cudaMemsetAsync(rho, 0, sizeof(double2) * M, st));
  const double L0 = L[0], L1 = D > 1 ? L[1] : 1.0, L2 = D > 2 ? L[2] : 1.0;
  const int pblocks = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(N, kThreads), 2 * int64_t(sm_count()))));
  dim3 fg(pblocks, unsigned(ceil_div(M, kFreqChunk)));
  nuwnu_forward_kernel<D><<<fg, kThreads, 0, st>>>(x, N, s, M, c, 1.0, L0, L1, L2, rho, status, nullptr);
  FB_LAUNCH_CHECK();
  const int mg = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(M, kThreads), int64_t(sm_count()) * 4)));
  nuwnu_loss_kernel<<<mg, kThreads, 0, st>>>(rho, M, 1.0 / double(N), sk, v, e, factor, status);
  FB_LAUNCH_CHECK();
  if (!g) return;
  const int ag = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(N, kThreads), int64_t(sm_count()) * 8)));
  nuwnu_adjoint_kernel<D><<<ag, kThreads, 0, st>>>(x, N, s, M, factor, L0, L1, L2, g, acc ? 1 : 0, status, c, 1.0,
                                                   mode == 1 ? 1 : 0, nullptr);
  FB_LAUNCH_CHECK();
}

}  // namespace

int64_t nuwnu_noalloc_max_kpoints() { return kNoAllocMaxK; }

void nuwnu_energy_gradient_noalloc(const double* d_x, int64_t n_points, int ndim, const double* d_weights,
                                   const double* d_kpts, const double* d_sk, const double* d_v, int64_t n_k,
                                   const double* L, int gradient_mode, double* d_grad, double* d_energy,
                                   bool accumulate, cudaStream_t stream) {
  if (ndim < 1 || ndim > 3) throw InvalidArgument("Invalid dimension: " + std::to_string(ndim));
  if (n_points < 0 || n_k < 0) throw InvalidArgument("negative size");
  if (n_k > kNoAllocMaxK)
    throw InvalidArgument("n_k = " + std::to_string(n_k) + " exceeds the allocation-free NUwNU maximum of " +
                          std::to_string(kNoAllocMaxK) + " k-points; use a NUwNU handle for more");
  if (gradient_mode != 0 && gradient_mode != 1) throw InvalidArgument("gradient mode must be 0 or 1");
  if (!L) throw InvalidArgument("null box lengths");
  if (!d_energy) throw InvalidArgument("null energy pointer");
  if (n_points > 0 && !d_x) throw InvalidArgument("null coordinate array");
  if (n_k > 0 && (!d_kpts || !d_sk || !d_v)) throw InvalidArgument("null k-point, Sk or V array");
  double2* scratch = noalloc_scratch_on_current_device();
  switch (ndim) {
    case 1:
      noalloc_launch<1>(d_x, n_points, d_weights, d_kpts, d_sk, d_v, n_k, L, gradient_mode, d_grad, d_energy,
                        accumulate, scratch, stream);
      break;
    case 2:
      noalloc_launch<2>(d_x, n_points, d_weights, d_kpts, d_sk, d_v, n_k, L, gradient_mode, d_grad, d_energy,
                        accumulate, scratch, stream);
      break;
    default:
      noalloc_launch<3>(d_x, n_points, d_weights, d_kpts, d_sk, d_v, n_k, L, gradient_mode, d_grad, d_energy,
                        accumulate, scratch, stream);
      break;
  }
}

PotentialPtr make_nuwnu(const std::vector<double>& radii, const std::vector<double>& kpts,
                        const std::vector<double>& sk, const std::vector<double>& v, const std::vector<double>& L,
                        double eps, int precision) {
  const int D = int(L.size());
  const bool f32 = precision == 1;
#define FB_NUWNU(DD)                                                             \
  return f32 ? PotentialPtr(new NUwNUImpl<DD, float>(radii, kpts, sk, v, L, eps)) \
             : PotentialPtr(new NUwNUImpl<DD, double>(radii, kpts, sk, v, L, eps))
  if (D == 1) FB_NUWNU(1);
  if (D == 2) FB_NUWNU(2);
  if (D == 3) FB_NUWNU(3);
#undef FB_NUWNU
  throw std::runtime_error("Invalid dimension: " + std::to_string(D));
}

}  // namespace fb
