// UwU: structure-factor loss of an intensity grid on its own k-grid
// (source/fresco/uwu.hpp:17-195).
//
// The reference (uwu.hpp:152-194) computes R = sum(x), rho = FFT_+(x)
// (unnormalised, row-major, sign +1), S = |rho|^2 / R, d = (S - S0)/S0',
// phi = sum V d^2, f = (2/R) V d rho / S0' and grad = Re FFT_-(f); Sk and V
// arrive ifftshifted (fresco/potentials/uwu.pyx:14-15).  That gradient is the
// reference's own formula (it is not the exact derivative of phi: the
// exact one is 2 grad - sum_k 2 V d S/(R S0')), kept here for drop-in parity.
//
// B200 form: x is real, so one R2C transform gives X(k) = FFT_-(x)(k) on the
// half spectrum and rho = conj X.  Re FFT_-(f) = FFT_-(f^H) with the Hermitian
// part f^H(k) = (f(k) + conj f(-k))/2 = rho(k) a(k)/R, a = A q - B (A, B fold
// V and S0 at k and -k, q = |rho|^2/R), and FFT_-(f^H) is the C2R transform of
// conj(f^H) = X a / R: one R2C and one C2R per evaluation, and only the modes
// with V(k) != 0 or V(-k) != 0 are touched in between.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "potential.cuh"

namespace fb {

namespace {

constexpr int kThreads = 256;

struct UwuCoef {
  double A, B;    // gradient fold
  double w2, s0;  // phi term of this entry: w2 (q - s0)^2
  double w2m, s0m;  // phi term of the mirror -k when the mirror is not stored itself (else w2m = 0)
};

__device__ double sum_partials(const double* __restrict__ part, int P) {
  __shared__ double sh[32];
  __shared__ double result;
  double v = 0.0;
  for (int i = threadIdx.x; i < P; i += blockDim.x) v += part[i];
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

// grid = T(x), block partial sums of x (rhotot, uwu.hpp:157-163; summed
// deterministically instead of the reference's racy OpenMP accumulation).
template <typename T>
__global__ void __launch_bounds__(kThreads) uwu_load_kernel(const double* __restrict__ x, int64_t G, T* grid,
                                                            double* part, int* status) {
  double s = 0.0;
  bool bad = false;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < G; i += int64_t(gridDim.x) * blockDim.x) {
    const double v = x[i];
    grid[i] = T(v);
    s += v;
    bad |= !isfinite(v);
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
  __shared__ double red[32];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) uwu_modes_kernel(int64_t n_active, const int64_t* __restrict__ hidx,
                                                             const UwuCoef* __restrict__ coef,
                                                             const cplx_t<T>* __restrict__ X, cplx_t<T>* H,
                                                             const double* __restrict__ part, int P, double* energy,
                                                             int want_grad, int exact, double* csum) {
  const double R = sum_partials(part, P);
  const double invR = 1.0 / R;
  double phi = 0.0, cterm = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_active;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = hidx[i];
    const cplx_t<T> xv = X[h];
    const double xr = double(xv.x), xi = double(xv.y);
    const double q = (xr * xr + xi * xi) * invR;
    const UwuCoef c = coef[i];
    const double d1 = q - c.s0, d2 = q - c.s0m;
    phi += c.w2 * d1 * d1 + c.w2m * d2 * d2;
    // exact derivative: C = sum_k 2 V d S / (R S0') over all k (the d(1/R) term)
    cterm += 2.0 * invR * q * (c.w2 * d1 + c.w2m * d2);
    if (want_grad) {
      const double a = (c.A * q - c.B) * invR * (exact ? 2.0 : 1.0);
      cplx_t<T> out;
      out.x = T(xr * a);
      out.y = T(xi * a);
      H[h] = out;
    }
  }
  block_sum_atomic(phi, energy);
  if (exact) block_sum_atomic(cterm, csum);
}

// Exact derivative: subtract C from every output by lowering the k = 0 term
// of the C2R input (its real part reaches every grid point once).
template <typename T>
__global__ void uwu_offset_kernel(cplx_t<T>* H, const double* __restrict__ csum) {
  H[0].x = T(double(H[0].x) - *csum);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) uwu_store_kernel(const T* __restrict__ g, int64_t G, double* grad,
                                                             int accumulate) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < G; i += int64_t(gridDim.x) * blockDim.x) {
    const double v = double(g[i]);
    grad[i] = accumulate ? grad[i] + v : v;
  }
}

template <typename T>
class UwUImpl final : public Potential {
 public:
  UwUImpl(const std::vector<int>& grid, double K, const std::vector<double>& sk, const std::vector<double>& v,
          const std::vector<double>& L, double eps)
      : dims_(grid) {
    init_status();
    const int D = int(grid.size());
    if (D < 1 || D > 3) throw std::runtime_error("Invalid dimension: " + std::to_string(D));
    if (sk.size() != v.size()) throw InvalidArgument("len(Sk) must equal len(V)");
    G_ = 1;
    for (int n : grid) {
      if (n < 1) throw InvalidArgument("grid sizes must be positive");
      G_ *= n;
    }
    if (int64_t(v.size()) < G_) throw InvalidArgument("Sk/V must hold one value per grid point");
    const int nl = grid[D - 1];
    nh_ = nl / 2 + 1;
    GH_ = (G_ / nl) * nh_;
    // active half-spectrum entries
    std::vector<int64_t> hidx;
    std::vector<UwuCoef> coef;
    std::vector<int> idx(D), mir(D);
    for (int64_t outer = 0; outer < G_ / nl; ++outer) {
      int64_t r = outer;
      for (int a = D - 2; a >= 0; --a) {
        idx[a] = int(r % grid[a]);
        r /= grid[a];
      }
      for (int j = 0; j < nh_; ++j) {
        idx[D - 1] = j;
        int64_t fi = 0, mi = 0;
        for (int a = 0; a < D; ++a) {
          mir[a] = (grid[a] - idx[a]) % grid[a];
          fi = fi * grid[a] + idx[a];
          mi = mi * grid[a] + mir[a];
        }
        const double vk = v[fi], vm = v[mi];
        if (vk == 0.0 && vm == 0.0) continue;
        const double s0k = sk[fi], s0m = sk[mi];
        const double dk = s0k != 0.0 ? s0k : 1.0, dm = s0m != 0.0 ? s0m : 1.0;
        UwuCoef c;
        c.A = vk / (dk * dk) + vm / (dm * dm);
        c.B = vk * s0k / (dk * dk) + vm * s0m / (dm * dm);
        c.w2 = vk / (dk * dk);
        c.s0 = s0k;
        const bool mirror_stored = (j == 0) || (nl % 2 == 0 && j == nl / 2);
        c.w2m = mirror_stored ? 0.0 : vm / (dm * dm);
        c.s0m = s0m;
        hidx.push_back(outer * nh_ + j);
        coef.push_back(c);
      }
    }
    n_active_ = int64_t(hidx.size());
    if (n_active_) {
      hidx_.alloc(n_active_);
      coef_.alloc(n_active_);
      FB_CUDA(cudaMemcpy(hidx_.p, hidx.data(), sizeof(int64_t) * n_active_, cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(coef_.p, coef.data(), sizeof(UwuCoef) * n_active_, cudaMemcpyHostToDevice));
    }
    P_ = std::max(1, std::min(1024, 2 * sm_count()));
    part_.alloc(P_);
    csum_.alloc(1);
    grid_.alloc(G_);
    X_.alloc(GH_);
    H_.alloc(GH_);
    const bool f32 = sizeof(T) == 4;
    std::vector<int> dims(grid);
    FB_CUFFT(cufftPlanMany(&r2c_, D, dims.data(), nullptr, 1, 0, nullptr, 1, 0, f32 ? CUFFT_R2C : CUFFT_D2Z, 1));
    FB_CUFFT(cufftPlanMany(&c2r_, D, dims.data(), nullptr, 1, 0, nullptr, 1, 0, f32 ? CUFFT_C2R : CUFFT_Z2D, 1));
    FB_CUDA(cudaDeviceSynchronize());
  }

  ~UwUImpl() override {
    if (r2c_) cufftDestroy(r2c_);
    if (c2r_) cufftDestroy(c2r_);
  }

  int64_t ndof() const override { return G_; }
  std::string kind() const override { return "UwU"; }
  std::string describe() const override {
    std::string s = std::string("UwU precision=") + (sizeof(T) == 4 ? "fp32" : "fp64") + " grid=";
    for (size_t a = 0; a < dims_.size(); ++a) s += (a ? "x" : "") + std::to_string(dims_[a]);
    s += " active_modes=" + std::to_string(n_active_);
    return s;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override {
    run(x, nullptr, e, acc, s);
  }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    timer_begin(s);
    begin_eval_status(s);
    if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    uwu_load_kernel<T><<<P_, kThreads, 0, s>>>(x, G_, grid_.p, part_.p, status_.p);
    FB_LAUNCH_CHECK();
    FB_CUFFT(cufftSetStream(r2c_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecR2C(r2c_, reinterpret_cast<cufftReal*>(grid_.p), reinterpret_cast<cufftComplex*>(X_.p)));
    } else {
      FB_CUFFT(cufftExecD2Z(r2c_, reinterpret_cast<cufftDoubleReal*>(grid_.p),
                            reinterpret_cast<cufftDoubleComplex*>(X_.p)));
    }
    timer_mark("fft_forward", s);
    // cuFFT's C2R may overwrite its input, so the field is rebuilt every call:
    // zeros everywhere, then the active modes.
    if (g) FB_CUDA(cudaMemsetAsync(H_.p, 0, H_.bytes(), s));
    const int mgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n_active_, kThreads), 4 * sm_count())));
    const int exact = (g != nullptr && grad_mode_ == 1) ? 1 : 0;
    if (exact) FB_CUDA(cudaMemsetAsync(csum_.p, 0, sizeof(double), s));
    uwu_modes_kernel<T><<<mgrid, kThreads, 0, s>>>(n_active_, hidx_.p, coef_.p, X_.p, H_.p, part_.p, P_, e,
                                                   g != nullptr, exact, csum_.p);
    FB_LAUNCH_CHECK();
    if (exact) {
      uwu_offset_kernel<T><<<1, 1, 0, s>>>(H_.p, csum_.p);
      FB_LAUNCH_CHECK();
    }
    timer_mark("modes", s);
    if (!g) return;
    FB_CUFFT(cufftSetStream(c2r_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecC2R(c2r_, reinterpret_cast<cufftComplex*>(H_.p), reinterpret_cast<cufftReal*>(grid_.p)));
    } else {
      FB_CUFFT(cufftExecZ2D(c2r_, reinterpret_cast<cufftDoubleComplex*>(H_.p),
                            reinterpret_cast<cufftDoubleReal*>(grid_.p)));
    }
    timer_mark("fft_inverse", s);
    uwu_store_kernel<T><<<P_, kThreads, 0, s>>>(grid_.p, G_, g, acc ? 1 : 0);
    FB_LAUNCH_CHECK();
    timer_mark("store", s);
  }

  std::vector<int> dims_;
  int64_t G_ = 1, GH_ = 1;
  int nh_ = 1;
  int P_ = 1;
  int64_t n_active_ = 0;
  DevBuf<int64_t> hidx_;
  DevBuf<UwuCoef> coef_;
  DevBuf<double> part_, csum_;
  DevBuf<T> grid_;
  DevBuf<cplx_t<T>> X_, H_;
  cufftHandle r2c_ = 0, c2r_ = 0;
};

}  // namespace

PotentialPtr make_uwu(const std::vector<int>& grid, double K, const std::vector<double>& sk,
                      const std::vector<double>& v, const std::vector<double>& L, double eps, int precision) {
  if (precision == 1) return PotentialPtr(new UwUImpl<float>(grid, K, sk, v, L, eps));
  return PotentialPtr(new UwUImpl<double>(grid, K, sk, v, L, eps));
}

}  // namespace fb
