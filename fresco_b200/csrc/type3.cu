// Type-3 NUFFT (type3.cuh): coordinate maps and window checks, centring
// phases, output factors, inner pre-correction; spreading, sorting, the inner
// FFT and interpolation are the NUFFT building blocks of nufft.cuh.
#include "type3.cuh"

#include <cmath>
#include <stdexcept>
#include <string>

namespace fb {

namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.14159265358979323846;

struct T3Params {
  int D = 1, map = TYPE3_IDENTITY, sign = 1;
  double L[3] = {1, 1, 1};
  double C[3] = {0, 0, 0};   // centre of the coordinates being set
  double R[3] = {1, 1, 1};   // their half-width (window)
  double Dc[3] = {0, 0, 0};  // centre of the other side (phases)
  double P[3] = {1, 1, 1};   // sources: spreading-grid period; targets: unused
  double h[3] = {1, 1, 1};   // spreading-grid spacing
  double alpha[3] = {1, 1, 1};
  double zmax[3] = {1, 1, 1};
  double C_src[3] = {0, 0, 0};  // targets: the source centre (output phase)
  const double* cheb[3] = {nullptr, nullptr, nullptr};
  int ncheb[3] = {0, 0, 0};
};

__device__ __forceinline__ double t3_map(double v, int map, double L) {
  // nuwnu.hpp:134 / 193, the reference's operation order
  return map == TYPE3_NUWNU_MAP ? (v - round(v / L) + L) * 2.0 * kPi / L : v;
}

// Clenshaw evaluation of sum_k c_k T_k(z / zmax) (|z| <= zmax).
__device__ __forceinline__ double chebyshev(const double* __restrict__ c, int n, double z, double zmax) {
  const double y = z / zmax, y2 = 2.0 * y;
  double b1 = 0.0, b2 = 0.0;
  for (int k = n - 1; k >= 1; --k) {
    const double b0 = fma(y2, b1, c[k] - b2);
    b2 = b1;
    b1 = b0;
  }
  return fma(y, b1, c[0] - b2);
}

// Sources: sort coordinate x' + P/2 (x' = x - C), phase exp(i sign Dc . x'),
// window flag.
__global__ void __launch_bounds__(kThreads) t3_source_kernel(const double* __restrict__ coords, int64_t n,
                                                             T3Params p, double* xs, double2* phase, int* flag) {
  bool out = false;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += int64_t(gridDim.x) * blockDim.x) {
    double ph = 0.0;
    for (int a = 0; a < p.D; ++a) {
      const double xp = t3_map(coords[j * p.D + a], p.map, p.L[a]) - p.C[a];
      out |= !(fabs(xp) <= p.R[a]);
      xs[j * p.D + a] = xp + 0.5 * p.P[a];
      ph += p.Dc[a] * xp;
    }
    double sn, cs;
    sincos(p.sign * ph, &sn, &cs);
    phase[j] = make_double2(cs, sn);
  }
  if (out) atomicOr(flag, 1);
}

// Targets: inner-grid coordinate theta = (t - Dc) h, output factor
// h^d exp(i sign t . C_src) / prod psi^(t - Dc), window flag.
__global__ void __launch_bounds__(kThreads) t3_target_kernel(const double* __restrict__ coords, int64_t n,
                                                             T3Params p, double* xt, double2* post, int* flag) {
  bool out = false;
  for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += int64_t(gridDim.x) * blockDim.x) {
    double ph = 0.0, den = 1.0;
    for (int a = 0; a < p.D; ++a) {
      const double t = t3_map(coords[k * p.D + a], p.map, p.L[a]);
      const double tp = t - p.C[a];
      out |= !(fabs(tp) <= p.R[a]);
      xt[k * p.D + a] = tp * p.h[a];
      ph += t * p.C_src[a];
      // psi^(xi) = alpha F(xi alpha), F fitted on [-zmax, zmax]
      const double z = fmin(fmax(tp * p.alpha[a], -p.zmax[a]), p.zmax[a]);
      den *= p.alpha[a] * chebyshev(p.cheb[a], p.ncheb[a], z, p.zmax[a]) / p.h[a];
    }
    double sn, cs;
    sincos(p.sign * ph, &sn, &cs);
    post[k] = make_double2(cs / den, sn / den);
  }
  if (out) atomicOr(flag + 1, 1);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) t3_strength_real_kernel(const double* __restrict__ a, double uniform,
                                                                    const double2* __restrict__ phase, int64_t n,
                                                                    int nvec, cplx_t<T>* str) {
  const int64_t tot = n * nvec;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot; i += int64_t(gridDim.x) * blockDim.x) {
    const double w = a ? a[i] : uniform;
    const double2 ph = phase[i % n];
    cplx_t<T> v;
    v.x = T(w * ph.x);
    v.y = T(w * ph.y);
    str[i] = v;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) t3_strength_cplx_kernel(const double2* __restrict__ a,
                                                                    const double2* __restrict__ phase, int64_t n,
                                                                    int nvec, cplx_t<T>* str) {
  const int64_t tot = n * nvec;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < tot; i += int64_t(gridDim.x) * blockDim.x) {
    const double2 w = a[i], ph = phase[i % n];
    cplx_t<T> v;
    v.x = T(w.x * ph.x - w.y * ph.y);
    v.y = T(w.x * ph.y + w.y * ph.x);
    str[i] = v;
  }
}

// Inner type 2: the spreading grid's cell l is Fourier mode m = l - nf/2;
// H[m mod nf2] = grid[l] / corr(m) (the other cells of H stay zero).
template <typename T>
__global__ void __launch_bounds__(kThreads) t3_precorrect_kernel(const cplx_t<T>* __restrict__ grid, Geom gout,
                                                                 Geom gin, int nvec, const double* __restrict__ c0,
                                                                 const double* __restrict__ c1,
                                                                 const double* __restrict__ c2, cplx_t<T>* H) {
  const int64_t Go = gout.G(), Gi = gin.G();
  const int n0 = gout.nf[0], n1 = gout.nf[1];
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < Go * nvec;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int v = int(i / Go);
    const int64_t l = i - int64_t(v) * Go;
    const int l0 = int(l % n0);
    const int64_t r = l / n0;
    const int l1 = int(r % n1), l2 = int(r / n1);
    const int m0 = l0 - n0 / 2, m1 = l1 - n1 / 2, m2 = l2 - gout.nf[2] / 2;
    double p = c0[l0];
    if (gout.D >= 2) p *= c1[l1];
    if (gout.D >= 3) p *= c2[l2];
    const int d0 = m0 < 0 ? m0 + gin.nf[0] : m0;
    const int d1 = gout.D >= 2 ? (m1 < 0 ? m1 + gin.nf[1] : m1) : 0;
    const int d2 = gout.D >= 3 ? (m2 < 0 ? m2 + gin.nf[2] : m2) : 0;
    const cplx_t<T> g = grid[i];
    cplx_t<T> o;
    o.x = T(double(g.x) / p);
    o.y = T(double(g.y) / p);
    H[int64_t(v) * Gi + (int64_t(d2) * gin.nf[1] + d1) * gin.nf[0] + d0] = o;
  }
}

__global__ void __launch_bounds__(kThreads) t3_post_kernel(const double2* __restrict__ post, int64_t n, int nvec,
                                                           double2* out) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n * nvec;
       i += int64_t(gridDim.x) * blockDim.x) {
    const double2 f = post[i % n], v = out[i];
    out[i] = make_double2(v.x * f.x - v.y * f.y, v.x * f.y + v.y * f.x);
  }
}

int grid_for(int64_t n) {
  return int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(std::max<int64_t>(n, 1), kThreads),
                                                    int64_t(sm_count()) * 8)));
}

Geom t3_geom(int D, const int64_t* nf, int w, bool f32) {
  int tile[3];
  if (D == 1) {
    tile[0] = 1024;
    tile[1] = tile[2] = 1;
  } else if (D == 2) {
    tile[0] = tile[1] = kTile2D;
    tile[2] = 1;
  } else if (f32) {
    tile[0] = 16;
    tile[1] = 16;
    tile[2] = 8;
  } else {
    tile[0] = tile[1] = tile[2] = 8;
  }
  return make_geom(D, nf, w, tile);
}

}  // namespace

template <typename T>
Type3<T>::Type3(int D, int64_t n_src, int64_t n_tgt, const double* src_lo, const double* src_hi,
                const double* tgt_lo, const double* tgt_hi, int sign, double eps, int nvec)
    : D_(D), sign_(sign >= 0 ? 1 : -1), nvec_(nvec), Ns_(n_src), Nt_(n_tgt) {
  if (D < 1 || D > 3) throw InvalidArgument("type 3: dimension must be 1, 2 or 3");
  if (nvec < 1) throw InvalidArgument("type 3: at least one strength vector");
  es_ = es_params(eps, sizeof(T) == 4 ? 10 : 16);
  poly_ = es_poly_coefficients(es_, es_.w);
  const int w = es_.w;
  int64_t nf[3] = {1, 1, 1}, nf2[3] = {1, 1, 1};
  for (int a = 0; a < D; ++a) {
    if (!(src_hi[a] >= src_lo[a]) || !(tgt_hi[a] >= tgt_lo[a]) || !std::isfinite(src_hi[a] - src_lo[a]) ||
        !std::isfinite(tgt_hi[a] - tgt_lo[a]))
      throw InvalidArgument("type 3: coordinate windows must be finite and ordered");
    C_[a] = 0.5 * (src_lo[a] + src_hi[a]);
    X_[a] = 0.5 * (src_hi[a] - src_lo[a]) * (1.0 + 1e-12) + 1e-300;
    Dc_[a] = 0.5 * (tgt_lo[a] + tgt_hi[a]);
    S_[a] = 0.5 * (tgt_hi[a] - tgt_lo[a]) * (1.0 + 1e-12) + 1e-300;
    // spacing from the frequency extent (upsampling 2), size from the source
    // extent plus the kernel's reach; a degenerate extent gets the smallest grid
    const double hmax = 2.0 * X_[a] / w + 1.0;
    h_[a] = std::min(kPi / (2.0 * S_[a]), hmax);
    const double need = std::ceil(2.0 * X_[a] / h_[a]) + w + 2;
    if (need > double(int64_t(1) << 24)) throw InvalidArgument("type 3: the product of the extents is too large");
    nf[a] = next_smooth_even(std::max<int64_t>(2 * w, int64_t(need)));
    nf_[a] = int(nf[a]);
    P_[a] = double(nf[a]) * h_[a];
    alpha_[a] = 0.5 * w * h_[a];
    nf2[a] = fine_grid_size(nf[a], w);
  }
  gout_ = t3_geom(D, nf, w, sizeof(T) == 4);
  gin_ = t3_geom(D, nf2, w, sizeof(T) == 4);
  for (int a = 0; a < 3; ++a) {
    std::vector<double> pc =
        a < D ? es_correction(es_, gin_.nf[a], -(nf_[a] / 2), nf_[a]) : std::vector<double>(1, 1.0);
    corr_[a].alloc(pc.size());
    FB_CUDA(cudaMemcpy(corr_[a].p, pc.data(), sizeof(double) * pc.size(), cudaMemcpyHostToDevice));
    if (a < D) {
      const std::vector<double> ch = es_fourier_chebyshev(es_, S_[a] * alpha_[a] * (1.0 + 1e-9));
      ncheb_[a] = int(ch.size());
      cheb_[a].alloc(ch.size());
      FB_CUDA(cudaMemcpy(cheb_[a].p, ch.data(), sizeof(double) * ch.size(), cudaMemcpyHostToDevice));
    }
  }
  alloc_sort(sort_src_, Ns_, gout_);
  alloc_sort(sort_tgt_, Nt_, gin_);
  const bool f32 = sizeof(T) == 4;
  rec_src_.alloc(std::max<int64_t>(Ns_, 1) * rec_bytes(D, f32));
  rec_tgt_.alloc(std::max<int64_t>(Nt_, 1) * rec_bytes(D, f32));
  xs_.alloc(std::max<int64_t>(Ns_ * D, 1));
  xt_.alloc(std::max<int64_t>(Nt_ * D, 1));
  phase_src_.alloc(std::max<int64_t>(Ns_, 1));
  post_.alloc(std::max<int64_t>(Nt_, 1));
  str_.alloc(std::max<int64_t>(Ns_ * nvec_, 1));
  grid_.alloc(gout_.G() * nvec_);
  H_.alloc(gin_.G() * nvec_);
  F_.alloc(gin_.G() * nvec_);
  FB_CUDA(cudaMemset(H_.p, 0, H_.bytes()));
  flag_.alloc(2);
  status_.alloc(2);
  FB_CUDA(cudaMemset(flag_.p, 0, 2 * sizeof(int)));
  FB_CUDA(cudaMemset(status_.p, 0, 2 * sizeof(int)));
  int dims[3];
  for (int a = 0; a < D; ++a) dims[a] = gin_.nf[D - 1 - a];
  const int Gi = int(gin_.G());
  FB_CUFFT(cufftPlanMany(&plan_, D, dims, nullptr, 1, Gi, nullptr, 1, Gi, f32 ? CUFFT_C2C : CUFFT_Z2Z, nvec_));
  FB_CUDA(cudaDeviceSynchronize());
}

template <typename T>
Type3<T>::~Type3() {
  if (plan_) cufftDestroy(plan_);
}

template <typename T>
std::string Type3<T>::describe() const {
  std::string s = "type3 w=" + std::to_string(es_.w) + " grid=";
  for (int a = 0; a < D_; ++a) s += (a ? "x" : "") + std::to_string(nf_[a]);
  s += " fine=";
  for (int a = 0; a < D_; ++a) s += (a ? "x" : "") + std::to_string(gin_.nf[a]);
  return s;
}

template <typename T>
void Type3<T>::set_sources(const double* d_coords, int map, const double* L, cudaStream_t s) {
  FB_CUDA(cudaMemsetAsync(flag_.p, 0, sizeof(int), s));
  if (Ns_ == 0) return;
  T3Params p;
  p.D = D_;
  p.map = map;
  p.sign = sign_;
  for (int a = 0; a < D_; ++a) {
    p.L[a] = L ? L[a] : 1.0;
    p.C[a] = C_[a];
    p.R[a] = X_[a];
    p.Dc[a] = Dc_[a];
    p.P[a] = P_[a];
  }
  t3_source_kernel<<<grid_for(Ns_), kThreads, 0, s>>>(d_coords, Ns_, p, xs_.p, phase_src_.p, flag_.p);
  FB_LAUNCH_CHECK();
  MapParams mp;
  mp.kind = 1;
  mp.stride = D_;
  for (int a = 0; a < D_; ++a) mp.L[a] = P_[a];
  bin_sort<T>(xs_.p, Ns_, mp, gout_, sort_src_, rec_src_.p, status_.p, s);
}

template <typename T>
void Type3<T>::set_targets(const double* d_coords, int map, const double* L, cudaStream_t s) {
  FB_CUDA(cudaMemsetAsync(flag_.p + 1, 0, sizeof(int), s));
  if (Nt_ == 0) return;
  T3Params p;
  p.D = D_;
  p.map = map;
  p.sign = sign_;
  for (int a = 0; a < D_; ++a) {
    p.L[a] = L ? L[a] : 1.0;
    p.C[a] = Dc_[a];
    p.R[a] = S_[a];
    p.h[a] = h_[a];
    p.alpha[a] = alpha_[a];
    p.zmax[a] = S_[a] * alpha_[a] * (1.0 + 1e-9);
    p.C_src[a] = C_[a];
    p.cheb[a] = cheb_[a].p;
    p.ncheb[a] = ncheb_[a];
  }
  t3_target_kernel<<<grid_for(Nt_), kThreads, 0, s>>>(d_coords, Nt_, p, xt_.p, post_.p, flag_.p);
  FB_LAUNCH_CHECK();
  MapParams mp;
  mp.kind = 1;
  mp.stride = D_;
  for (int a = 0; a < D_; ++a) mp.L[a] = 2.0 * kPi;
  bin_sort<T>(xt_.p, Nt_, mp, gin_, sort_tgt_, rec_tgt_.p, status_.p + 1, s);
}

template <typename T>
void Type3<T>::execute_real(const double* a, double uniform, double2* out, cudaStream_t s) {
  if (Ns_ > 0) {
    t3_strength_real_kernel<T><<<grid_for(Ns_ * nvec_), kThreads, 0, s>>>(a, uniform, phase_src_.p, Ns_, nvec_,
                                                                           str_.p);
    FB_LAUNCH_CHECK();
  }
  run(str_.p, out, s);
}

template <typename T>
void Type3<T>::execute_cplx(const double2* a, double2* out, cudaStream_t s) {
  if (Ns_ > 0) {
    t3_strength_cplx_kernel<T><<<grid_for(Ns_ * nvec_), kThreads, 0, s>>>(a, phase_src_.p, Ns_, nvec_, str_.p);
    FB_LAUNCH_CHECK();
  }
  run(str_.p, out, s);
}

template <typename T>
void Type3<T>::exec_fft(cplx_t<T>* in, cplx_t<T>* out, cudaStream_t s) {
  FB_CUFFT(cufftSetStream(plan_, s));
  const int dir = sign_ > 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
  if (sizeof(T) == 4) {
    FB_CUFFT(cufftExecC2C(plan_, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftComplex*>(out), dir));
  } else {
    FB_CUFFT(cufftExecZ2Z(plan_, reinterpret_cast<cufftDoubleComplex*>(in), reinterpret_cast<cufftDoubleComplex*>(out),
                          dir));
  }
}

template <typename T>
void Type3<T>::run(const cplx_t<T>* strengths, double2* out, cudaStream_t s) {
  if (Nt_ == 0) return;
  const int64_t Go = gout_.G(), Gi = gin_.G();
  FB_CUDA(cudaMemsetAsync(grid_.p, 0, grid_.bytes(), s));
  if (Ns_ > 0)
    for (int v = 0; v < nvec_; ++v)
      spread_cplx<T>(rec_src_.p, strengths + int64_t(v) * Ns_, sort_src_, gout_, poly_, grid_.p + int64_t(v) * Go, s);
  t3_precorrect_kernel<T><<<grid_for(Go * nvec_), kThreads, 0, s>>>(grid_.p, gout_, gin_, nvec_, corr_[0].p,
                                                                     corr_[1].p, corr_[2].p, H_.p);
  FB_LAUNCH_CHECK();
  exec_fft(H_.p, F_.p, s);
  for (int v = 0; v < nvec_; ++v)
    interp<T>(rec_tgt_.p, Nt_, nullptr, T(1), sort_tgt_, gin_, poly_, F_.p + int64_t(v) * Gi, 1, INTERP_CPLX, nullptr,
              out + int64_t(v) * Nt_, 0, nullptr, s);
  t3_post_kernel<<<grid_for(Nt_ * nvec_), kThreads, 0, s>>>(post_.p, Nt_, nvec_, out);
  FB_LAUNCH_CHECK();
}

template class Type3<float>;
template class Type3<double>;

}  // namespace fb
