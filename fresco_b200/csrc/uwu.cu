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

#include "fft_block.cuh"
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

// ---------------------------------------------------------------------------
// Band transforms for 2D grids N x N (N a power of two in 512..8192) whose
// active modes lie in |k0| <= KB0 and 0 <= k1 <= KB1 of the half spectrum
// (k1 along the fast axis), both small: register FFTs (RegFft<T, N>) that
// read the caller's FP64 grid once and write the FP64 gradient once.
//   rows_fwd:  two grid rows per transform (z = a + i b), sums the rows for R,
//              keeps k1 = 0..KB1 of each row               -> band1[KB1+1][N]
//   modes:     one k1 per block: column FFT of band1, the mode pass of
//              uwu_modes_kernel on |k0| <= KB0, and the inverse column FFT
//              of the field                                  -> band2[KB1+1][N]
//   rows_c2r:  two gradient rows per transform from the Hermitian row
//              spectra k1 = -KB1..KB1 (the C2R of cuFFT: the imaginary part
//              of k1 = 0 is ignored, no normalisation).
// ---------------------------------------------------------------------------

template <typename T, int N>
__global__ void __launch_bounds__(N / 8) uwu_band_rows_fwd(const double* __restrict__ x, cplx_t<T>* __restrict__ band1,
                                                           int KB1, const cplx_t<T>* __restrict__ tw, double* part,
                                                           int* status) {
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* buf = reinterpret_cast<cplx_t<T>*>(smem_raw) + threadIdx.y * fft_padded(N);
  __shared__ double red[N / 8 / 32];
  const int t = threadIdx.x;
  const int64_t y = 2 * (2 * int64_t(blockIdx.x) + threadIdx.y);
  const double* ra = x + y * N;
  const double* rb = ra + N;
  cplx_t<T> v[F::E];
  double sum = 0.0;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < F::E; ++j) {
    const double a = ra[t + j * (N / F::E)], b = rb[t + j * (N / F::E)];
    sum += a + b;
    bad |= !isfinite(a) || !isfinite(b);
    v[j].x = T(a);
    v[j].y = T(b);
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
  const int tid = threadIdx.y * F::TPB + t;
  sum = warp_sum(sum);
  if ((tid & 31) == 0) red[tid >> 5] = sum;
  F::run(v, buf, tw, t, 1 + threadIdx.y);
  // A(k) = (Z(k) + conj Z(-k)) / 2, B(k) = (Z(k) - conj Z(-k)) / (2i)
  for (int k = t; k <= KB1; k += F::TPB) {
    const cplx_t<T> zk = buf[fpad(k)], zm = buf[fpad(k == 0 ? 0 : N - k)];
    cplx_t<T> A, B;
    A.x = T(0.5) * (zk.x + zm.x);
    A.y = T(0.5) * (zk.y - zm.y);
    B.x = T(0.5) * (zk.y + zm.y);
    B.y = T(0.5) * (zm.x - zk.x);
    band1[int64_t(k) * N + y] = A;
    band1[int64_t(k) * N + y + 1] = B;
  }
  __syncthreads();
  if (tid < 32) {
    double s = tid < N / 8 / 32 ? red[tid] : 0.0;
    s = warp_sum(s);
    if (tid == 0) part[blockIdx.x] = s;
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(N / 16) uwu_band_modes(const cplx_t<T>* __restrict__ band1,
                                                         cplx_t<T>* __restrict__ band2,
                                                         const UwuCoef* __restrict__ box, int KB0,
                                                         const cplx_t<T>* __restrict__ tw,
                                                         const double* __restrict__ part, int P, double* energy,
                                                         int want_grad, int exact, double* csum) {
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* col = reinterpret_cast<cplx_t<T>*>(smem_raw);
  cplx_t<T>* h = col + fft_padded(N);
  const int t = threadIdx.x;
  const int j = blockIdx.x;  // k1
  const int NY = 2 * KB0 + 1;
  const double R = sum_partials(part, P);  // ends with __syncthreads
  const double invR = 1.0 / R;
  if (want_grad)
    for (int i = t; i < N; i += F::TPB) h[fpad(i)] = cplx_t<T>{T(0), T(0)};
  {
    cplx_t<T> v[F::E];
#pragma unroll
    for (int jj = 0; jj < F::E; ++jj) v[jj] = band1[int64_t(j) * N + t + jj * (N / F::E)];
    F::run(v, col, tw, t, 1);  // X(k0, k1) for every k0, natural order
  }
  double phi = 0.0, cterm = 0.0;
  const UwuCoef* crow = box + int64_t(j) * NY;
  for (int i = t; i < NY; i += F::TPB) {
    const UwuCoef c = crow[i];
    if (c.w2 == 0.0 && c.w2m == 0.0 && c.A == 0.0 && c.B == 0.0) continue;  // not an active entry
    const int k0 = i - KB0;
    const int r = k0 < 0 ? k0 + N : k0;
    const cplx_t<T> xv = col[fpad(r)];
    const double xr = double(xv.x), xi = double(xv.y);
    const double q = (xr * xr + xi * xi) * invR;
    const double d1 = q - c.s0, d2 = q - c.s0m;
    phi += c.w2 * d1 * d1 + c.w2m * d2 * d2;
    cterm += 2.0 * invR * q * (c.w2 * d1 + c.w2m * d2);
    if (want_grad) {
      const double a = (c.A * q - c.B) * invR * (exact ? 2.0 : 1.0);
      cplx_t<T> o;
      o.x = T(xr * a);
      o.y = T(xi * a);
      h[fpad(r)] = o;
    }
  }
  block_sum_atomic(phi, energy);  // ends with __syncthreads
  if (exact) block_sum_atomic(cterm, csum);
  if (!want_grad) return;
  // inverse (sign +1) column transform: conj(FFT(conj(h)))
  cplx_t<T> v[F::E];
#pragma unroll
  for (int jj = 0; jj < F::E; ++jj) {
    const cplx_t<T> w = h[fpad(t + jj * (N / F::E))];
    v[jj].x = w.x;
    v[jj].y = -w.y;
  }
  group_sync(1, F::TPB);  // every input is in registers before h is reused
  F::run(v, h, tw, t, 1);
  for (int y = t; y < N; y += F::TPB) {
    const cplx_t<T> w = h[fpad(y)];
    band2[int64_t(j) * N + y] = cplx_t<T>{w.x, -w.y};
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(N / 8) uwu_band_rows_c2r(const cplx_t<T>* __restrict__ band2, int KB1,
                                                           const cplx_t<T>* __restrict__ tw, double* grad,
                                                           int accumulate, int exact, const double* __restrict__ csum) {
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* buf = reinterpret_cast<cplx_t<T>*>(smem_raw) + threadIdx.y * fft_padded(N);
  const int t = threadIdx.x;
  const int64_t y = 2 * (2 * int64_t(blockIdx.x) + threadIdx.y);
  // conj of Z(k) = A(k) + i B(k) over the Hermitian extension of rows y, y+1
  cplx_t<T> v[F::E];
#pragma unroll
  for (int jj = 0; jj < F::E; ++jj) {
    const int k = t + jj * (N / F::E);
    T zr = T(0), zi = T(0);
    if (k == 0) {
      zr = band2[y].x;
      zi = band2[y + 1].x;
    } else if (k <= KB1) {
      const cplx_t<T> A = band2[int64_t(k) * N + y], B = band2[int64_t(k) * N + y + 1];
      zr = A.x - B.y;
      zi = A.y + B.x;
    } else if (k >= N - KB1) {
      const int m = N - k;
      const cplx_t<T> A = band2[int64_t(m) * N + y], B = band2[int64_t(m) * N + y + 1];
      zr = A.x + B.y;  // conj(A) + i conj(B)
      zi = -A.y + B.x;
    }
    v[jj].x = zr;
    v[jj].y = -zi;
  }
  F::run(v, buf, tw, t, 1 + threadIdx.y);
  const double off = exact ? *csum : 0.0;
  double* ga = grad + y * N;
  double* gb = ga + N;
  for (int i = t; i < N; i += F::TPB) {
    const cplx_t<T> w = buf[fpad(i)];  // z = conj(w): a = w.x, b = -w.y
    const double a = double(w.x) - off, b = -double(w.y) - off;
    ga[i] = accumulate ? ga[i] + a : a;
    gb[i] = accumulate ? gb[i] + b : b;
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
    csum_.alloc(1);
    setup_band(hidx, coef);
    if (band_) {
      part_.alloc(dims_[0] / 4);
      FB_CUDA(cudaDeviceSynchronize());
      return;  // no cuFFT plans or full-size spectra: the band kernels do all transforms
    }
    part_.alloc(P_);
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
    if (band_) s += " fft=band|k0|<=" + std::to_string(KB0_) + ",k1<=" + std::to_string(KB1_);
    return s;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override {
    run(x, nullptr, e, acc, s);
  }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  // 2D N x N grids with N a power of two in 512..8192 and the active entries
  // in a narrow band of the half spectrum use the band kernels.
  void setup_band(const std::vector<int64_t>& hidx, const std::vector<UwuCoef>& coef) {
    band_ = false;
    if (dims_.size() != 2 || n_active_ == 0) return;
    const int N = dims_[0];
    if (dims_[1] != N || N < 512 || N > 8192 || (N & (N - 1)) != 0) return;
    if (2 * size_t(fft_padded(N)) * sizeof(cplx_t<T>) > 200 * 1024) return;
    int kb0 = 0, kb1 = 0;
    for (int64_t h : hidx) {
      const int i0 = int(h / nh_), j = int(h % nh_);
      kb0 = std::max(kb0, i0 <= N / 2 ? i0 : N - i0);
      kb1 = std::max(kb1, j);
    }
    if (kb1 + 1 > N / 4 || 2 * kb0 + 1 > N / 2) return;
    KB0_ = kb0;
    KB1_ = kb1;
    const int NY = 2 * KB0_ + 1;
    std::vector<UwuCoef> box(size_t(KB1_ + 1) * NY, UwuCoef{0, 0, 0, 0, 0, 0});
    for (size_t i = 0; i < hidx.size(); ++i) {
      const int i0 = int(hidx[i] / nh_), j = int(hidx[i] % nh_);
      const int k0 = i0 <= N / 2 ? i0 : i0 - N;
      box[size_t(j) * NY + (k0 + KB0_)] = coef[i];
    }
    box_.alloc(box.size());
    FB_CUDA(cudaMemcpy(box_.p, box.data(), sizeof(UwuCoef) * box.size(), cudaMemcpyHostToDevice));
    const std::vector<double> tw = fft_twiddles(N);
    std::vector<cplx_t<T>> th(N);
    for (int k = 0; k < N; ++k) {
      th[k].x = T(tw[2 * size_t(k)]);
      th[k].y = T(tw[2 * size_t(k) + 1]);
    }
    tw_.alloc(N);
    FB_CUDA(cudaMemcpy(tw_.p, th.data(), sizeof(cplx_t<T>) * N, cudaMemcpyHostToDevice));
    band1_.alloc(int64_t(KB1_ + 1) * N);
    band2_.alloc(int64_t(KB1_ + 1) * N);
    smem_ = 2 * size_t(fft_padded(N)) * sizeof(cplx_t<T>);
    switch (N) {
      case 512: band_attrs<512>(); break;
      case 1024: band_attrs<1024>(); break;
      case 2048: band_attrs<2048>(); break;
      case 4096: band_attrs<4096>(); break;
      default: band_attrs<8192>(); break;
    }
    band_ = true;
  }

  template <int N>
  void band_attrs() {
    ensure_dynamic_smem(uwu_band_rows_fwd<T, N>, smem_);
    ensure_dynamic_smem(uwu_band_modes<T, N>, smem_);
    ensure_dynamic_smem(uwu_band_rows_c2r<T, N>, smem_);
  }

  template <int N>
  void run_band_n(const double* x, double* g, double* e, bool acc, int exact, cudaStream_t s) {
    const dim3 rows(N / 16, 2);
    uwu_band_rows_fwd<T, N><<<N / 4, rows, smem_, s>>>(x, band1_.p, KB1_, tw_.p, part_.p, status_.p);
    FB_LAUNCH_CHECK();
    timer_mark("fft_forward", s);
    uwu_band_modes<T, N><<<KB1_ + 1, N / 16, smem_, s>>>(band1_.p, band2_.p, box_.p, KB0_, tw_.p, part_.p, N / 4, e,
                                                         g != nullptr, exact, csum_.p);
    FB_LAUNCH_CHECK();
    timer_mark("modes", s);
    if (!g) return;
    uwu_band_rows_c2r<T, N><<<N / 4, rows, smem_, s>>>(band2_.p, KB1_, tw_.p, g, acc ? 1 : 0, exact, csum_.p);
    FB_LAUNCH_CHECK();
    timer_mark("fft_inverse", s);
  }

  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    timer_begin(s);
    begin_eval_status(s);
    if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    if (band_) {
      const int exact = (g != nullptr && grad_mode_ == 1) ? 1 : 0;
      if (exact) FB_CUDA(cudaMemsetAsync(csum_.p, 0, sizeof(double), s));
      switch (dims_[0]) {
        case 512: run_band_n<512>(x, g, e, acc, exact, s); break;
        case 1024: run_band_n<1024>(x, g, e, acc, exact, s); break;
        case 2048: run_band_n<2048>(x, g, e, acc, exact, s); break;
        case 4096: run_band_n<4096>(x, g, e, acc, exact, s); break;
        default: run_band_n<8192>(x, g, e, acc, exact, s); break;
      }
      return;
    }
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
  bool band_ = false;
  int KB0_ = 0, KB1_ = 0;
  size_t smem_ = 0;
  DevBuf<UwuCoef> box_;
  DevBuf<cplx_t<T>> tw_, band1_, band2_;
};

}  // namespace

PotentialPtr make_uwu(const std::vector<int>& grid, double K, const std::vector<double>& sk,
                      const std::vector<double>& v, const std::vector<double>& L, double eps, int precision) {
  if (precision == 1) return PotentialPtr(new UwUImpl<float>(grid, K, sk, v, L, eps));
  return PotentialPtr(new UwUImpl<double>(grid, K, sk, v, L, eps));
}

}  // namespace fb
