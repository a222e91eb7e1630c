// NUwU: structure-factor loss of a point pattern on a uniform k-grid and its
// gradient with respect to the points (source/fresco/nuwu.hpp:17-318).
//
// Per evaluation (get_energy_gradient, nuwu.hpp:210-317):
//   1. bin-sort the points by fine-grid tile (replaces finufft_setpts x2,
//      nuwu.hpp:256-257: one sort serves both transforms);
//   2. spread the real weights c_j with the ES kernel (type 1, iflag +1,
//      nuwu.hpp:50,258) and R2C-transform the real fine grid (cuFFT);
//   3. one pass over the active modes (V(k) != 0 or V(-k) != 0): deconvolve,
//      S = |rho|^2/N, d = (S - S0)/S0', phi += V d^2 (FP64), and the packed
//      type-2 field (nuwu.hpp:260-287);
//   4. C2C-transform the packed field (iflag -1, nuwu.hpp:51,291-309);
//   5. interpolate at the points and write grad = c_j * Re(...) (nuwu.hpp:294-315).
//
// Packing.  The reference computes grad[d*j+a] = Re(conj(c_j) T2(f_a)(x_j))
// with f_a(k) = -i k_a F(k), F = (4/N) V d rho / S0'.  For real c (always the
// case, nuwu.hpp:125-149) Re T2(f) = T2(f^H) with the Hermitian part
// f^H(k) = (f(k) + conj f(-k))/2, so T2 of h = f_x^H + i f_y^H returns the x
// and y components as its real and imaginary parts: one FFT and one
// interpolation pass serve two dimensions.  f_a^H = -i k_a F^H with
// F^H(k) = (2/N) rho(k) [A(k) q - B(k)], q = |rho|^2/N, where A and B fold
// V and S0 at k and -k (precomputed per mode at set-up).
#include <cmath>
#include <string>
#include <vector>

#include "band_fft.cuh"
#include "fft_block.cuh"
#include "nufft.cuh"
#include "nuwu_modes.cuh"
#include "potential.cuh"

namespace fb {

namespace {

template <int D, typename T>
__global__ void __launch_bounds__(256) nuwu_modes_kernel(
    int n, int K, double invN, const int* __restrict__ mode_idx, const ModeCoef* __restrict__ coef, int n_active,
    const cplx_t<T>* __restrict__ bhat, int nh0, Geom g, const double* __restrict__ corr0, const double* __restrict__ corr1,
    const double* __restrict__ corr2, cplx_t<T>* hgrid, int64_t G, double* energy, const int* __restrict__ status,
    int want_grad) {
  double phi = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_active; i += gridDim.x * blockDim.x)
    phi += nuwu_mode_term<D, T>(mode_idx[i], n, K, coef[i], bhat, nh0, g.nf[0], g.nf[1], g.nf[2], corr0, corr1, corr2,
                                invN, hgrid, G, want_grad != 0);
  block_sum_atomic(phi, energy);
  if (blockIdx.x == 0 && threadIdx.x == 0 && status != nullptr && ((*status) & STATUS_NONFINITE_INPUT)) {
    atomicAdd(energy, __longlong_as_double(0x7ff8000000000000ULL));
  }
}

// Undeconvolved rho of this point set at every active mode (shard step 1);
// a non-finite coordinate makes rho[0] NaN so that the sum over shards, and
// every shard's energy, carries it.
template <int D, typename T>
__global__ void __launch_bounds__(256) nuwu_gather_rho_kernel(int n, int K, const int* __restrict__ mode_idx,
                                                              int n_active, const cplx_t<T>* __restrict__ bhat, int nh0,
                                                              Geom g, double2* rho, const int* __restrict__ status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_active; i += gridDim.x * blockDim.x) {
    double2 r = nuwu_mode_rho<D, T>(mode_idx[i], n, K, bhat, nh0, g.nf[1], g.nf[2]);
    if (i == 0 && status != nullptr && ((*status) & STATUS_NONFINITE_INPUT))
      r.x = __longlong_as_double(0x7ff8000000000000ULL);
    rho[i] = r;
  }
}

// Mode pass from the summed rho of all shards (shard step 2).
template <int D, typename T>
__global__ void __launch_bounds__(256) nuwu_modes_from_rho_kernel(
    int n, int K, double invN, const int* __restrict__ mode_idx, const ModeCoef* __restrict__ coef, int n_active,
    const double2* __restrict__ rho, Geom g, const double* __restrict__ corr0, const double* __restrict__ corr1,
    const double* __restrict__ corr2, cplx_t<T>* hgrid, int64_t G, double* energy, int want_grad) {
  double phi = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_active; i += gridDim.x * blockDim.x)
    phi += nuwu_mode_apply<D, T>(mode_idx[i], n, K, coef[i], rho[i], g.nf[0], g.nf[1], g.nf[2], corr0, corr1, corr2,
                                 invN, hgrid, G, want_grad != 0);
  block_sum_atomic(phi, energy);
}

template <int D, typename T>
class NUwUImpl final : public Potential, public NUwUShard {
 public:
  // n_total >= 0 makes a shard of a pattern of n_total points whose weight
  // factors (area^D per point) sum to weight_sum_total over all shards.
  NUwUImpl(const std::vector<double>& radii, double K, const std::vector<double>& sk, const std::vector<double>& v,
           const std::vector<double>& L, double eps, int64_t n_total = -1, double weight_sum_total = 0.0)
      : N_(int64_t(radii.size())), Karg_(K) {
    sharded_ = n_total >= 0;
    n_total_ = sharded_ ? n_total : N_;
    if (sharded_ && (n_total_ < N_ || !(weight_sum_total > 0.0)))
      throw InvalidArgument("sharded NUwU: n_total must cover this shard's points and the weight sum be positive");
    invN_ = 1.0 / double(n_total_);
    init_status();
    if (sk.size() != v.size()) throw InvalidArgument("len(Sk) must equal len(V)");
    if (int(L.size()) != D) throw InvalidArgument("len(L) must equal the dimension");
    for (int a = 0; a < D; ++a) L_[a] = L[a];
    // nuwu.hpp:54-79: K_ = int((sqrt(len V) - 1) / 2) (cbrt in 3D)
    const double vs = double(v.size());
    size_t kk;
    if (D == 1) kk = size_t((v.size() - 1) / 2);
    else if (D == 2) kk = size_t((std::sqrt(vs) - 1) / 2);
    else kk = size_t((std::cbrt(vs) - 1) / 2);
    K_ = int(kk);
    n_ = 2 * K_ + 1;
    int64_t nm = 1;
    for (int a = 0; a < D; ++a) nm *= n_;
    if (nm > int64_t(v.size())) throw InvalidArgument("V too short for its mode grid");
    nmodes_ = nm;

    // weights, nuwu.hpp:125-149 (area factor applied once per dimension)
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
    const double scale = sharded_ ? double(n_total_) / weight_sum_total : double(c.size()) / sum;
    for (size_t i = 0; i < c.size(); ++i) {
      c[i] *= scale;
      if (c[i] != c[0]) uniform = false;
    }
    if (uniform && !c.empty()) {
      uniform_c_ = T(c[0]);
    } else if (!c.empty()) {
      std::vector<T> ct(c.begin(), c.end());
      cw_.alloc(c.size());
      FB_CUDA(cudaMemcpy(cw_.p, ct.data(), sizeof(T) * c.size(), cudaMemcpyHostToDevice));
    }

    // ES kernel and fine grid
    es_ = es_params(eps, sizeof(T) == 4 ? 10 : 16);
    poly_ = es_poly_coefficients(es_, es_.w);
    int64_t nf[3] = {1, 1, 1};
    for (int a = 0; a < D; ++a) nf[a] = fine_grid_size(n_, es_.w);
    int tile[3];
    if (D == 1) { tile[0] = 1024; tile[1] = tile[2] = 1; }
    else if (D == 2) { tile[0] = kTile2D; tile[1] = kTile2D; tile[2] = 1; }
    else if (sizeof(T) == 4) { tile[0] = 16; tile[1] = 16; tile[2] = 8; }
    else { tile[0] = 8; tile[1] = 8; tile[2] = 8; }
    geom_ = make_geom(D, nf, es_.w, tile);
    alloc_sort(sort_, N_, geom_);
    recs_.alloc(std::max<int64_t>(N_, 1) * rec_bytes(D, sizeof(T) == 4));

    const int64_t G = geom_.G();
    nh0_ = geom_.nf[0] / 2 + 1;
    const int64_t GH = int64_t(nh0_) * geom_.nf[1] * geom_.nf[2];
    spread_grid_.alloc(G);
    bhat_.alloc(GH);
    nfields_ = (D == 3) ? 2 : 1;
    // 3D: the x/y field (G cells), then the z field's half spectrum (GH cells);
    // the type-2 output holds the complex x/y grid, then the real z grid
    hgrid_.alloc(D == 3 ? G + GH : G);
    ggrid_.alloc(D == 3 ? G + (G + 1) / 2 : G);
    FB_CUDA(cudaMemset(hgrid_.p, 0, hgrid_.bytes()));

    // correction factors per dimension, k = -K..K
    for (int a = 0; a < D; ++a) {
      std::vector<double> pc = es_correction(es_, geom_.nf[a], -K_, n_);
      corr_[a].alloc(n_);
      FB_CUDA(cudaMemcpy(corr_[a].p, pc.data(), sizeof(double) * n_, cudaMemcpyHostToDevice));
    }

    // active modes and their coefficients
    std::vector<int> idx;
    std::vector<ModeCoef> coef;
    nuwu_mode_table(D, n_, v.data(), sk.data(), idx, coef);
    n_active_ = int(idx.size());
    if (n_active_) {
      mode_idx_.alloc(n_active_);
      coef_.alloc(n_active_);
      FB_CUDA(cudaMemcpy(mode_idx_.p, idx.data(), sizeof(int) * n_active_, cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(coef_.p, coef.data(), sizeof(ModeCoef) * n_active_, cudaMemcpyHostToDevice));
    }

    // cuFFT plans (dims slowest first)
    int dims[3];
    for (int a = 0; a < D; ++a) dims[a] = geom_.nf[D - 1 - a];
    const bool f32 = sizeof(T) == 4;
    const cufftType r2c = f32 ? CUFFT_R2C : CUFFT_D2Z, c2c = f32 ? CUFFT_C2C : CUFFT_Z2Z;
    // 2D: row/column passes pruned to the columns |k_x| <= kx_max that hold
    // active modes (the type-1 column pass needs only k_x in [0, kx_max]; the
    // type-2 input is zero outside k_x in [-kx_max, kx_max])
    int kx_max = 0;
    for (int i = 0; i < n_active_; ++i) kx_max = std::max(kx_max, std::abs(idx[i] % n_ - K_));
    if (!sharded_) setup_band(idx, coef);  // a shard needs rho from the full R2C output
    pruned_ = !band_ && (D == 2) && n_active_ > 0 && 2 * kx_max + 1 < geom_.nf[0];
    if (band_) {
      // no cuFFT plans: the band kernels do all transforms
    } else if (pruned_) {
      const int nf0 = geom_.nf[0], nf1 = geom_.nf[1];
      kx_max_ = kx_max;
      int n0 = nf0, n1 = nf1, emb0 = nf0, embh = nh0_, emb1 = nf1;
      FB_CUFFT(cufftPlanMany(&plan_r2c_, 1, &n0, &emb0, 1, nf0, &embh, 1, nh0_, r2c, nf1));
      FB_CUFFT(cufftPlanMany(&plan_col1_, 1, &n1, &emb1, nh0_, 1, &emb1, nh0_, 1, c2c, kx_max + 1));
      FB_CUFFT(cufftPlanMany(&plan_col2a_, 1, &n1, &emb1, nf0, 1, &emb1, nf0, 1, c2c, kx_max + 1));
      if (kx_max > 0) FB_CUFFT(cufftPlanMany(&plan_col2b_, 1, &n1, &emb1, nf0, 1, &emb1, nf0, 1, c2c, kx_max));
      FB_CUFFT(cufftPlanMany(&plan_c2c_, 1, &n0, &emb0, 1, nf0, &emb0, 1, nf0, c2c, nf1));
      // column-pass output: the columns outside the active band stay zero for good
      tgrid_.alloc(G);
      FB_CUDA(cudaMemset(tgrid_.p, 0, tgrid_.bytes()));
    } else {
      FB_CUFFT(cufftPlanMany(&plan_r2c_, D, dims, nullptr, 1, 0, nullptr, 1, 0, r2c, 1));
      FB_CUFFT(cufftPlanMany(&plan_c2c_, D, dims, nullptr, 1, int(G), nullptr, 1, int(G), c2c, 1));
      if (D == 3) FB_CUFFT(cufftPlanMany(&plan_c2r_, D, dims, nullptr, 1, 0, nullptr, 1, 0, f32 ? CUFFT_C2R : CUFFT_Z2D, 1));
    }
    FB_CUDA(cudaDeviceSynchronize());
  }

  ~NUwUImpl() override {
    for (cufftHandle h : {plan_r2c_, plan_c2c_, plan_c2r_, plan_col1_, plan_col2a_, plan_col2b_})
      if (h) cufftDestroy(h);
  }

  int64_t ndof() const override { return N_ * D; }
  std::string kind() const override { return "NUwU"; }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override {
    run(x, nullptr, e, acc, s);
  }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

  int64_t n_rho() const override { return n_active_; }

  void shard_rho(const double* x, double* rho, cudaStream_t s) override {
    begin_eval_status(s);
    spread_and_transform(x, s);
    if (n_active_ > 0) {
      const int grid = int(std::min<int64_t>(ceil_div(n_active_, 256), int64_t(sm_count()) * 8));
      nuwu_gather_rho_kernel<D, T><<<grid, 256, 0, s>>>(n_, K_, mode_idx_.p, n_active_, bhat_.p, nh0_, geom_,
                                                         reinterpret_cast<double2*>(rho), status_.p);
      FB_LAUNCH_CHECK();
    }
  }

  void shard_finish(const double* rho, double* g, double* e, cudaStream_t s) override {
    shard_finish(rho, g, e, s, false);
  }

  // acc: the gradient is added to g (e always receives this term's energy alone)
  void shard_finish(const double* rho, double* g, double* e, cudaStream_t s, bool acc) {
    FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    if (g) clear_z_half(s);
    if (n_active_ > 0) {
      const int grid = int(std::min<int64_t>(ceil_div(n_active_, 256), int64_t(sm_count()) * 8));
      nuwu_modes_from_rho_kernel<D, T><<<grid, 256, 0, s>>>(
          n_, K_, invN_, mode_idx_.p, coef_.p, n_active_, reinterpret_cast<const double2*>(rho), geom_, corr_[0].p,
          D >= 2 ? corr_[1].p : corr_[0].p, D >= 3 ? corr_[2].p : corr_[0].p, hgrid_.p, geom_.G(), e,
          g != nullptr);
      FB_LAUNCH_CHECK();
    }
    if (g) type2_and_interp(g, e, acc, s);
  }

  std::string describe() const override {
    std::string s = "NUwU D=" + std::to_string(D) + " precision=" + (sizeof(T) == 4 ? "fp32" : "fp64") +
                    " N=" + std::to_string(N_) + " modes/dim=" + std::to_string(n_) + " w=" + std::to_string(es_.w) +
                    " beta=" + std::to_string(es_.beta) + " nf=";
    for (int a = 0; a < D; ++a) s += (a ? "x" : "") + std::to_string(geom_.nf[a]);
    s += " tile=";
    for (int a = 0; a < D; ++a) s += (a ? "x" : "") + std::to_string(geom_.tile[a]);
    s += " bins=" + std::to_string(geom_.nbins()) + " active_modes=" + std::to_string(n_active_);
    if (band_) s += " fft=band|kx|<=" + std::to_string(Kx_) + ",|ky|<=" + std::to_string(Ky_);
    if (pruned_) s += " fft=columns|kx|<=" + std::to_string(kx_max_);
    return s;
  }

  const Geom& geom() const { return geom_; }
  const ESParams& es() const { return es_; }
  int n_active() const { return n_active_; }

 private:
  // sort, spread and type-1 transform of the full R2C path (bhat holds the
  // half spectrum afterwards; pruned 2D grids transform only the columns
  // k_x <= kx_max)
  void spread_and_transform(const double* x, cudaStream_t s) {
    MapParams mp;
    mp.kind = 0;
    mp.stride = D;
    for (int a = 0; a < D; ++a) mp.L[a] = L_[a];
    bin_sort<T>(x, N_, mp, geom_, sort_, recs_.p, status_.p, s);
    FB_CUDA(cudaMemsetAsync(spread_grid_.p, 0, spread_grid_.bytes(), s));
    spread_real<T>(recs_.p, cw_.p, uniform_c_, sort_, geom_, poly_, spread_grid_.p, s);
    FB_CUFFT(cufftSetStream(plan_r2c_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecR2C(plan_r2c_, reinterpret_cast<cufftReal*>(spread_grid_.p),
                            reinterpret_cast<cufftComplex*>(bhat_.p)));
    } else {
      FB_CUFFT(cufftExecD2Z(plan_r2c_, reinterpret_cast<cufftDoubleReal*>(spread_grid_.p),
                            reinterpret_cast<cufftDoubleComplex*>(bhat_.p)));
    }
    if (pruned_) exec_c2c(plan_col1_, bhat_.p, bhat_.p, s);
  }

  // type-2 transform of the packed field and interpolation at the points
  void type2_and_interp(double* g, double* e, bool acc, cudaStream_t s) {
    if (pruned_) {
      const int off = geom_.nf[0] - kx_max_;
      exec_c2c(plan_col2a_, hgrid_.p, tgrid_.p, s);
      if (kx_max_ > 0) exec_c2c(plan_col2b_, hgrid_.p + off, tgrid_.p + off, s);
      exec_c2c(plan_c2c_, tgrid_.p, ggrid_.p, s);
    } else {
      exec_type2_fields(s);
    }
    GradScale gs;  // exact mode: x = (p - round(p/L)) 2 pi / L, so d/dp = (2 pi / L) d/dx
    if (grad_mode_ == 1)
      for (int a = 0; a < D; ++a) gs.s[a] = 2.0 * M_PI / L_[a];
    interp<T>(recs_.p, N_, cw_.p, uniform_c_, sort_, geom_, poly_, ggrid_.p, nfields_, INTERP_GRAD, g, nullptr,
              acc ? 1 : 0, status_.p, s, gs, e);
  }

  bool host_steps() const override { return sharded_ && reducer_ != nullptr; }

  void set_reducer(ReduceFn fn, void* ctx) override {
    if (!sharded_) throw InvalidArgument("NUwU: only a shard of a pattern takes a reducer");
    reducer_ = fn;
    reducer_ctx_ = ctx;
    if (!rho_sum_.p) rho_sum_.alloc(2 * std::max<int64_t>(n_active_, 1));
    if (!e_part_.p) e_part_.alloc(1);
  }

  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    if (sharded_ && reducer_) {  // this shard's rho, the sum over the shards, the shared mode pass
      shard_rho(x, rho_sum_.p, s);
      reducer_(rho_sum_.p, 2 * n_active_, s, reducer_ctx_);
      shard_finish(rho_sum_.p, g, acc ? e_part_.p : e, s, acc);
      if (acc) add_scalar(e_part_.p, e, s);
      return;
    }
    if (sharded_ && n_total_ != N_)
      throw InvalidArgument("sharded NUwU: evaluate through the shard calls (rho, sum over shards, finish)");
    timer_begin(s);
    begin_eval_status(s);
    if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    MapParams mp;
    mp.kind = 0;
    mp.stride = D;
    for (int a = 0; a < D; ++a) mp.L[a] = L_[a];
    bin_sort<T>(x, N_, mp, geom_, sort_, recs_.p, status_.p, s);
    timer_mark("sort", s);
    if (!band_) {  // the band row transform leaves the grid zeroed for the next evaluation
      FB_CUDA(cudaMemsetAsync(spread_grid_.p, 0, spread_grid_.bytes(), s));
      timer_mark("zero_grid", s);
    }
    spread_real<T>(recs_.p, cw_.p, uniform_c_, sort_, geom_, poly_, spread_grid_.p, s);
    timer_mark("spread", s);
    if (band_) {
      run_band(e, g, acc, s);
      return;
    }
    FB_CUFFT(cufftSetStream(plan_r2c_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecR2C(plan_r2c_, reinterpret_cast<cufftReal*>(spread_grid_.p),
                            reinterpret_cast<cufftComplex*>(bhat_.p)));
    } else {
      FB_CUFFT(cufftExecD2Z(plan_r2c_, reinterpret_cast<cufftDoubleReal*>(spread_grid_.p),
                            reinterpret_cast<cufftDoubleComplex*>(bhat_.p)));
    }
    if (pruned_) exec_c2c(plan_col1_, bhat_.p, bhat_.p, s);  // columns k_x = 0..kx_max, in place
    timer_mark("fft_type1", s);
    if (g) clear_z_half(s);
    if (n_active_ > 0) {
      const int grid = int(std::min<int64_t>(ceil_div(n_active_, 256), int64_t(sm_count()) * 8));
      nuwu_modes_kernel<D, T><<<grid, 256, 0, s>>>(
          n_, K_, invN_, mode_idx_.p, coef_.p, n_active_, bhat_.p, nh0_, geom_, corr_[0].p,
          D >= 2 ? corr_[1].p : corr_[0].p, D >= 3 ? corr_[2].p : corr_[0].p, hgrid_.p, geom_.G(), e, status_.p,
          g != nullptr);
      FB_LAUNCH_CHECK();
    } else {
      nuwu_modes_kernel<D, T><<<1, 32, 0, s>>>(n_, K_, 1.0, mode_idx_.p, coef_.p, 0, bhat_.p, nh0_, geom_,
                                               corr_[0].p, corr_[0].p, corr_[0].p, hgrid_.p, geom_.G(), e,
                                               status_.p, 0);
      FB_LAUNCH_CHECK();
    }
    timer_mark("modes", s);
    if (!g) return;
    if (pruned_) {
      // columns k_x in [0, kx_max] and [nf0 - kx_max, nf0), then every row
      const int off = geom_.nf[0] - kx_max_;
      exec_c2c(plan_col2a_, hgrid_.p, tgrid_.p, s);
      if (kx_max_ > 0) exec_c2c(plan_col2b_, hgrid_.p + off, tgrid_.p + off, s);
      exec_c2c(plan_c2c_, tgrid_.p, ggrid_.p, s);
    } else {
      exec_type2_fields(s);
    }
    timer_mark("fft_type2", s);
    GradScale gs;  // exact mode: x = (p - round(p/L)) 2 pi / L, so d/dp = (2 pi / L) d/dx
    if (grad_mode_ == 1)
      for (int a = 0; a < D; ++a) gs.s[a] = 2.0 * M_PI / L_[a];
    interp<T>(recs_.p, N_, cw_.p, uniform_c_, sort_, geom_, poly_, ggrid_.p, nfields_, INTERP_GRAD, g, nullptr,
              acc ? 1 : 0, status_.p, s, gs, e);
    timer_mark("interp", s);
  }

  // 2D band transforms (see band_rows_r2c_kernel): used when the fine grid is
  // N x N with N a power of two in 512..8192.
  template <int N>
  void band_attrs() {
    const size_t cb = sizeof(cplx_t<T>);
    smem_rows_ = 2 * size_t(fft_padded(N)) * cb;
    smem_modes_ = 3 * size_t(fft_padded(N)) * cb;
    ensure_dynamic_smem(band_rows_r2c_kernel<T, N>, smem_rows_);
    ensure_dynamic_smem(band_rows_c2c_kernel<T, N>, smem_rows_);
    ensure_dynamic_smem(band_modes_kernel<T, N>, smem_modes_);
  }

  void setup_band(const std::vector<int>& idx, const std::vector<ModeCoef>& coef) {
    band_ = false;
    if (D != 2 || n_active_ == 0) return;
    const int nf0 = geom_.nf[0], nf1 = geom_.nf[1];
    if (nf0 != nf1 || nf0 < 512 || nf0 > 8192 || (nf0 & (nf0 - 1)) != 0) return;
    if (3 * size_t(fft_padded(nf0)) * sizeof(cplx_t<T>) > 200 * 1024) return;
    int kxm = 0, kym = 0;
    for (int m : idx) {
      kxm = std::max(kxm, std::abs(m % n_ - K_));
      kym = std::max(kym, std::abs(m / n_ - K_));
    }
    if (2 * kxm + 1 > nf0 / 2) return;
    Kx_ = kxm;
    Ky_ = kym;
    const std::vector<double> t = fft_twiddles(nf0);
    std::vector<cplx_t<T>> h(nf0);
    for (int j = 0; j < nf0; ++j) {
      h[j].x = T(t[2 * size_t(j)]);
      h[j].y = T(t[2 * size_t(j) + 1]);
    }
    tw_.alloc(nf0);
    FB_CUDA(cudaMemcpy(tw_.p, h.data(), sizeof(cplx_t<T>) * nf0, cudaMemcpyHostToDevice));
    const int NY = 2 * Ky_ + 1, NX = 2 * Kx_ + 1;
    std::vector<ModeCoef> box(size_t(NX) * NY, ModeCoef{0.0, 0.0, 0.0, 0.0});
    for (size_t i = 0; i < idx.size(); ++i) {
      const int kx = idx[i] % n_ - K_, ky = idx[i] / n_ - K_;
      box[size_t(kx + Kx_) * NY + (ky + Ky_)] = coef[i];
    }
    coef_box_.alloc(box.size());
    FB_CUDA(cudaMemcpy(coef_box_.p, box.data(), sizeof(ModeCoef) * box.size(), cudaMemcpyHostToDevice));
    band1_.alloc(int64_t(nf1) * (Kx_ + 1));
    band2_.alloc(int64_t(nf1) * NX);
    switch (nf0) {
      case 512: band_attrs<512>(); break;
      case 1024: band_attrs<1024>(); break;
      case 2048: band_attrs<2048>(); break;
      case 4096: band_attrs<4096>(); break;
      default: band_attrs<8192>(); break;
    }
    FB_CUDA(cudaMemset(spread_grid_.p, 0, spread_grid_.bytes()));
    band_ = true;
  }

  template <int N>
  void run_band_n(double* e, double* g, cudaStream_t s) {
    const dim3 blk(N / 16, 2);
    const BandBatch<T> bb{spread_grid_.p, 0,       band1_.p, 0, band2_.p, 0,       ggrid_.p,
                          0,              coef_box_.p, 0,   nullptr,  invN_, e, status_.p, nullptr};
    band_rows_r2c_kernel<T, N><<<N / 4, blk, smem_rows_, s>>>(spread_grid_.p, 0, tw_.p, Kx_ + 1, band1_.p, 0);
    FB_LAUNCH_CHECK();
    timer_mark("fft_type1", s);
    band_modes_kernel<T, N><<<Kx_ + 1, blk, smem_modes_, s>>>(bb, tw_.p, Kx_, Ky_, K_, corr_[0].p, corr_[1].p,
                                                               g != nullptr);
    FB_LAUNCH_CHECK();
    timer_mark("modes", s);
    if (!g) return;
    band_rows_c2c_kernel<T, N><<<N / 2, blk, smem_rows_, s>>>(bb, Kx_, tw_.p);
    FB_LAUNCH_CHECK();
    timer_mark("fft_type2", s);
  }

  void run_band(double* e, double* g, bool acc, cudaStream_t s) {
    switch (geom_.nf[0]) {
      case 512: run_band_n<512>(e, g, s); break;
      case 1024: run_band_n<1024>(e, g, s); break;
      case 2048: run_band_n<2048>(e, g, s); break;
      case 4096: run_band_n<4096>(e, g, s); break;
      default: run_band_n<8192>(e, g, s); break;
    }
    if (!g) return;
    GradScale gs;
    if (grad_mode_ == 1)
      for (int a = 0; a < D; ++a) gs.s[a] = 2.0 * M_PI / L_[a];
    interp<T>(recs_.p, N_, cw_.p, uniform_c_, sort_, geom_, poly_, ggrid_.p, nfields_, INTERP_GRAD, g, nullptr,
              acc ? 1 : 0, status_.p, s, gs, e);
    timer_mark("interp", s);
  }

  // forward (sign -1) complex transform on stream s
  // Type-2 transforms of the packed fields (not the pruned 2D passes): the x/y
  // field C2C; in 3D the z field's half spectrum C2R into the real grid after
  // the complex one.  A C2R transform overwrites its input, so the mode pass
  // works on a half spectrum cleared by clear_z_half().
  void exec_type2_fields(cudaStream_t s) {
    exec_c2c(plan_c2c_, hgrid_.p, ggrid_.p, s);
    if (D != 3) return;
    const int64_t G = geom_.G();
    FB_CUFFT(cufftSetStream(plan_c2r_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecC2R(plan_c2r_, reinterpret_cast<cufftComplex*>(hgrid_.p + G),
                            reinterpret_cast<cufftReal*>(ggrid_.p + G)));
    } else {
      FB_CUFFT(cufftExecZ2D(plan_c2r_, reinterpret_cast<cufftDoubleComplex*>(hgrid_.p + G),
                            reinterpret_cast<cufftDoubleReal*>(ggrid_.p + G)));
    }
  }
  void clear_z_half(cudaStream_t s) {
    if (D == 3)
      FB_CUDA(cudaMemsetAsync(hgrid_.p + geom_.G(), 0,
                              sizeof(cplx_t<T>) * size_t(nh0_) * geom_.nf[1] * geom_.nf[2], s));
  }

  static void exec_c2c(cufftHandle plan, cplx_t<T>* in, cplx_t<T>* out, cudaStream_t s) {
    FB_CUFFT(cufftSetStream(plan, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftComplex*>(out),
                            CUFFT_FORWARD));
    } else {
      FB_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(in),
                            reinterpret_cast<cufftDoubleComplex*>(out), CUFFT_FORWARD));
    }
  }

  int64_t N_;
  bool sharded_ = false;
  ReduceFn reducer_ = nullptr;
  void* reducer_ctx_ = nullptr;
  DevBuf<double> rho_sum_, e_part_;
  int64_t n_total_ = 0;
  double invN_ = 1.0;
  double Karg_;
  double L_[3] = {1, 1, 1};
  int K_ = 0, n_ = 1;
  int64_t nmodes_ = 1;
  T uniform_c_ = T(1);
  DevBuf<T> cw_;
  ESParams es_;
  std::vector<double> poly_;
  Geom geom_;
  SortBufs sort_;
  DevBuf<unsigned char> recs_;
  int nh0_ = 1;
  int nfields_ = 1;
  DevBuf<T> spread_grid_;
  DevBuf<cplx_t<T>> bhat_, hgrid_, ggrid_, tgrid_;
  DevBuf<double> corr_[3];
  DevBuf<int> mode_idx_;
  DevBuf<ModeCoef> coef_;
  int n_active_ = 0;
  cufftHandle plan_r2c_ = 0, plan_c2c_ = 0, plan_c2r_ = 0, plan_col1_ = 0, plan_col2a_ = 0, plan_col2b_ = 0;
  bool pruned_ = false;
  int kx_max_ = 0;
  bool band_ = false;
  int Kx_ = 0, Ky_ = 0;
  DevBuf<cplx_t<T>> tw_, band1_, band2_;
  DevBuf<ModeCoef> coef_box_;
  size_t smem_rows_ = 0, smem_modes_ = 0;
};

}  // namespace

double nuwu_weight_factor_sum(const double* radii, int64_t n, int D) {
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double c = 1.0;
    for (int j = 0; j < D; ++j) {
      if (D == 2) c = c * M_PI * radii[i] * radii[i];
      else if (D == 3) c = c * M_PI * radii[i] * radii[i] * radii[i] * 4.0 / 3.0;
    }
    sum += c;
  }
  return sum;
}

PotentialPtr make_nuwu_shard(const std::vector<double>& radii_local, int64_t n_total, double weight_sum_total,
                             double K, const std::vector<double>& sk, const std::vector<double>& v,
                             const std::vector<double>& L, double eps, int precision) {
  const int D = int(L.size());
  const bool f32 = precision == 1;
#define FB_SHARD(DD)                                                                                               \
  return f32 ? PotentialPtr(new NUwUImpl<DD, float>(radii_local, K, sk, v, L, eps, n_total, weight_sum_total))    \
             : PotentialPtr(new NUwUImpl<DD, double>(radii_local, K, sk, v, L, eps, n_total, weight_sum_total))
  if (D == 1) FB_SHARD(1);
  if (D == 2) FB_SHARD(2);
  if (D == 3) FB_SHARD(3);
#undef FB_SHARD
  throw std::runtime_error("Invalid dimension: " + std::to_string(D));
}

PotentialPtr make_nuwu(const std::vector<double>& radii, double K, const std::vector<double>& sk,
                       const std::vector<double>& v, const std::vector<double>& L, double eps, int precision) {
  const int D = int(L.size());
  const bool f32 = precision == 1;
  if (D == 1) return f32 ? PotentialPtr(new NUwUImpl<1, float>(radii, K, sk, v, L, eps))
                         : PotentialPtr(new NUwUImpl<1, double>(radii, K, sk, v, L, eps));
  if (D == 2) return f32 ? PotentialPtr(new NUwUImpl<2, float>(radii, K, sk, v, L, eps))
                         : PotentialPtr(new NUwUImpl<2, double>(radii, K, sk, v, L, eps));
  if (D == 3) return f32 ? PotentialPtr(new NUwUImpl<3, float>(radii, K, sk, v, L, eps))
                         : PotentialPtr(new NUwUImpl<3, double>(radii, K, sk, v, L, eps));
  throw std::runtime_error("Invalid dimension: " + std::to_string(D));
}

}  // namespace fb
