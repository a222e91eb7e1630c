// UwNU: structure-factor loss of an intensity grid at non-uniform k-points
// (source/fresco/uwnu.hpp:214-356).
//
// Reference semantics: k~_j = K_j * 2 pi / L per dimension (uwnu.hpp:243-276,
// fixed at construction), rho_j = sum_n x_n exp(+i n.k~_j) over the centred
// grid modes n (FINUFFT type 2, iflag +1, dimension 0 fastest, modeord 0;
// uwnu.hpp:279, 326), S = |rho|^2 (rhotot = 1), d = (S - S0)/S0',
// phi = sum V d^2, f_j = 4 V_j d_j rho_j / S0'_j and
// grad_n = Re(sum_j f_j exp(-i n.k~_j)) / (2 pi) (type 1, iflag -1,
// uwnu.hpp:340-353).  The reference's get_energy also prints every |rho_j|
// (uwnu.hpp:301); this implementation does not print.
//
// B200 form: the k-points are bin-sorted once at set-up.  Each evaluation:
// pre-correct x into the zero-padded fine grid, one C2C transform (sign +1),
// interpolate at the k-points, a loss pass that also forms f, spread f
// (complex strengths), one C2C transform (sign -1), and a pass that
// deconvolves and writes the gradient.
#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "nufft.cuh"
#include "potential.cuh"

namespace fb {

namespace {

constexpr int kThreads = 256;
constexpr double kTwoPi = 6.28318530717958647692;

// H[n mod nf] = x_n / p(n) for every grid mode n (dimension 0 fastest).
template <typename T>
__global__ void __launch_bounds__(kThreads) uwnu_precorrect_kernel(const double* __restrict__ x, int64_t G, int D,
                                                                   int n0, int n1, int n2, Geom g,
                                                                   const double* __restrict__ p0,
                                                                   const double* __restrict__ p1,
                                                                   const double* __restrict__ p2, cplx_t<T>* H,
                                                                   int* status) {
  bool bad = false;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < G; i += int64_t(gridDim.x) * blockDim.x) {
    const int i0 = int(i % n0);
    const int64_t r = i / n0;
    const int i1 = int(r % n1);
    const int i2 = int(r / n1);
    int k0 = i0 - n0 / 2, k1 = i1 - n1 / 2, k2 = i2 - n2 / 2;
    double p = p0[i0];
    if (D >= 2) p *= p1[i1];
    if (D >= 3) p *= p2[i2];
    const double v = x[i];
    bad |= !isfinite(v);
    const int l0 = k0 < 0 ? k0 + g.nf[0] : k0;
    const int l1 = D >= 2 ? (k1 < 0 ? k1 + g.nf[1] : k1) : 0;
    const int l2 = D >= 3 ? (k2 < 0 ? k2 + g.nf[2] : k2) : 0;
    cplx_t<T> h;
    h.x = T(v / p);
    h.y = T(0);
    H[(int64_t(l2) * g.nf[1] + l1) * g.nf[0] + l0] = h;
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
}

// Loss over the k-points and the type-1 strengths f_j = 4 V d rho / S0'.
template <typename T>
__global__ void __launch_bounds__(kThreads) uwnu_loss_kernel(const double2* __restrict__ rho, int64_t M,
                                                             const double* __restrict__ sk,
                                                             const double* __restrict__ v, double* energy,
                                                             cplx_t<T>* f, int want_grad) {
  double phi = 0.0;
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < M; j += int64_t(gridDim.x) * blockDim.x) {
    const double2 r = rho[j];
    const double s0 = sk[j];
    const double dn = s0 != 0.0 ? s0 : 1.0;
    const double d = (r.x * r.x + r.y * r.y - s0) / dn;  // uwnu.hpp:330-336 (rhotot = 1)
    phi += v[j] * d * d;
    if (want_grad) {
      const double a = 4.0 * v[j] * d / dn;
      cplx_t<T> o;
      o.x = T(a * r.x);
      o.y = T(a * r.y);
      f[j] = o;
    }
  }
  block_sum_atomic(phi, energy);
}

// grad_n = Re(B[n mod nf] / p(n)) * out_scale (1/(2 pi) in the reference's convention,
// uwnu.hpp:352; 1 for the exact derivative), B the sign -1 transform of the spread strengths.
template <typename T>
__global__ void __launch_bounds__(kThreads) uwnu_extract_kernel(const cplx_t<T>* __restrict__ B, int64_t G, int D,
                                                                int n0, int n1, int n2, Geom g,
                                                                const double* __restrict__ p0,
                                                                const double* __restrict__ p1,
                                                                const double* __restrict__ p2, double* grad,
                                                                int accumulate, double out_scale) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < G; i += int64_t(gridDim.x) * blockDim.x) {
    const int i0 = int(i % n0);
    const int64_t r = i / n0;
    const int i1 = int(r % n1);
    const int i2 = int(r / n1);
    const int k0 = i0 - n0 / 2, k1 = i1 - n1 / 2, k2 = i2 - n2 / 2;
    double p = p0[i0];
    if (D >= 2) p *= p1[i1];
    if (D >= 3) p *= p2[i2];
    const int l0 = k0 < 0 ? k0 + g.nf[0] : k0;
    const int l1 = D >= 2 ? (k1 < 0 ? k1 + g.nf[1] : k1) : 0;
    const int l2 = D >= 3 ? (k2 < 0 ? k2 + g.nf[2] : k2) : 0;
    const double val = double(B[(int64_t(l2) * g.nf[1] + l1) * g.nf[0] + l0].x) / p * out_scale;
    grad[i] = accumulate ? grad[i] + val : val;
  }
}

template <typename T>
class UwNUImpl final : public Potential {
 public:
  UwNUImpl(const std::vector<int>& grid, const std::vector<double>& kpts, const std::vector<double>& sk,
           const std::vector<double>& v, const std::vector<double>& L, double eps)
      : D_(int(L.size())) {
    init_status();
    if (D_ < 1 || D_ > 3) throw std::runtime_error("Invalid dimension: " + std::to_string(D_));
    if (int(grid.size()) < D_) throw InvalidArgument("grid needs one size per dimension");
    if (sk.size() != v.size()) throw InvalidArgument("len(Sk) must equal len(V)");
    M_ = int64_t(sk.size());
    if (int64_t(kpts.size()) < M_ * D_) throw InvalidArgument("K needs ndim values per k-point");
    G_ = 1;
    for (int a = 0; a < 3; ++a) {
      n_[a] = a < D_ ? grid[a] : 1;
      if (n_[a] < 1) throw InvalidArgument("grid sizes must be positive");
      G_ *= n_[a];
    }
    es_ = es_params(eps, sizeof(T) == 4 ? 10 : 16);
    poly_ = es_poly_coefficients(es_, es_.w);
    int64_t nf[3] = {1, 1, 1};
    for (int a = 0; a < D_; ++a) nf[a] = fine_grid_size(n_[a], es_.w);
    int tile[3];
    if (D_ == 1) { tile[0] = 1024; tile[1] = tile[2] = 1; }
    else if (D_ == 2) { tile[0] = kTile2D; tile[1] = kTile2D; tile[2] = 1; }
    else if (sizeof(T) == 4) { tile[0] = 16; tile[1] = 16; tile[2] = 8; }
    else { tile[0] = 8; tile[1] = 8; tile[2] = 8; }
    geom_ = make_geom(D_, nf, es_.w, tile);
    const int64_t FG = geom_.G();
    H_.alloc(FG);
    Gf_.alloc(FG);
    FB_CUDA(cudaMemset(H_.p, 0, H_.bytes()));
    for (int a = 0; a < 3; ++a) {
      std::vector<double> pc = a < D_ ? es_correction(es_, geom_.nf[a], -(n_[a] / 2), n_[a]) : std::vector<double>(1, 1.0);
      corr_[a].alloc(pc.size());
      FB_CUDA(cudaMemcpy(corr_[a].p, pc.data(), sizeof(double) * pc.size(), cudaMemcpyHostToDevice));
    }
    sk_.alloc(std::max<int64_t>(M_, 1));
    v_.alloc(std::max<int64_t>(M_, 1));
    rho_.alloc(std::max<int64_t>(M_, 1));
    f_.alloc(std::max<int64_t>(M_, 1));
    if (M_) {
      FB_CUDA(cudaMemcpy(sk_.p, sk.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(v_.p, v.data(), sizeof(double) * M_, cudaMemcpyHostToDevice));
    }
    // the k-points never move: sort them once (uwnu.hpp:280-281 sets the points in the constructor)
    DevBuf<double> kd(std::max<int64_t>(M_ * D_, 1));
    std::vector<double> kk(kpts.begin(), kpts.begin() + M_ * D_);
    if (M_) FB_CUDA(cudaMemcpy(kd.p, kk.data(), sizeof(double) * M_ * D_, cudaMemcpyHostToDevice));
    alloc_sort(sort_, M_, geom_);
    recs_.alloc(std::max<int64_t>(M_, 1) * rec_bytes(D_, sizeof(T) == 4));
    MapParams mp;
    mp.kind = 1;
    mp.stride = D_;
    for (int a = 0; a < D_; ++a) mp.L[a] = L[a];
    DevBuf<int> st(2);
    FB_CUDA(cudaMemset(st.p, 0, 2 * sizeof(int)));
    bin_sort<T>(kd.p, M_, mp, geom_, sort_, recs_.p, st.p, nullptr);
    int hst[2] = {0, 0};
    FB_CUDA(cudaMemcpy(hst, st.p, sizeof(hst), cudaMemcpyDeviceToHost));
    if (hst[0]) throw InvalidArgument("non-finite k-point");
    int dims[3];
    for (int a = 0; a < D_; ++a) dims[a] = geom_.nf[D_ - 1 - a];
    FB_CUFFT(cufftPlanMany(&plan_, D_, dims, nullptr, 1, 0, nullptr, 1, 0, sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z, 1));
    if (D_ == 2) setup_pruned();
    FB_CUDA(cudaDeviceSynchronize());
  }

  ~UwNUImpl() override {
    if (plan_) cufftDestroy(plan_);
    for (auto& kv : plans_) cufftDestroy(kv.second);
  }

  int64_t ndof() const override { return G_; }
  std::string kind() const override { return "UwNU"; }
  std::string describe() const override {
    std::string s = std::string("UwNU precision=") + (sizeof(T) == 4 ? "fp32" : "fp64") + " grid=";
    for (int a = 0; a < D_; ++a) s += (a ? "x" : "") + std::to_string(n_[a]);
    s += " kpoints=" + std::to_string(M_) + " w=" + std::to_string(es_.w) + " nf=";
    for (int a = 0; a < D_; ++a) s += (a ? "x" : "") + std::to_string(geom_.nf[a]);
    if (pruned_) {
      int nc = 0;
      for (auto& r : col_ranges_) nc += r.second;
      s += " fft=pruned rows=" + std::to_string(n_[1]) + " cols=" + std::to_string(nc);
    }
    return s;
  }

  void energy(const double* x, int64_t n, double* e, bool acc, cudaStream_t s) override { run(x, nullptr, e, acc, s); }
  void energy_gradient(const double* x, int64_t n, double* g, double* e, bool acc, cudaStream_t s) override {
    run(x, g, e, acc, s);
  }

 private:
  void exec(cplx_t<T>* in, cplx_t<T>* out, int dir, cudaStream_t s) {
    FB_CUFFT(cufftSetStream(plan_, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecC2C(plan_, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftComplex*>(out), dir));
    } else {
      FB_CUFFT(cufftExecZ2Z(plan_, reinterpret_cast<cufftDoubleComplex*>(in),
                            reinterpret_cast<cufftDoubleComplex*>(out), dir));
    }
  }

  // 2D: the 2D transforms as row and column passes that skip what is zero
  // or never read.  The input of the type-2 transform is non-zero only on the
  // rows of the grid modes (k1 in [-n1/2, n1/2)), and the interpolation reads
  // only the columns that the tiles of the k-points' bins reach (found here
  // from the k-point sort, which never changes); the type-1 input is
  // non-zero only on those columns and the extraction reads only the mode
  // rows.  So: type 2 = row FFTs of the mode rows (H -> T2, whose other rows
  // stay zero) + column FFTs of the reached columns (in place); type 1 =
  // column FFTs of the reached columns + row FFTs of the mode rows (in place).
  void setup_pruned() {
    pruned_ = false;
    const int nf0 = int(geom_.nf[0]), nf1 = int(geom_.nf[1]);
    const int nbins = int(geom_.nbins());
    std::vector<int> bs(nbins + 1);
    FB_CUDA(cudaMemcpy(bs.data(), sort_.bin_start.p, sizeof(int) * (nbins + 1), cudaMemcpyDeviceToHost));
    std::vector<char> col(nf0, 0);
    const int w = es_.w;
    for (int b = 0; b < nbins; ++b) {
      if (bs[b + 1] == bs[b]) continue;
      const int c0 = (b % geom_.nb[0]) * kTile2D;
      for (int c = c0 - w - 4; c < c0 + kTile2D + w + 4; ++c) col[((c % nf0) + nf0) % nf0] = 1;
    }
    std::vector<std::pair<int, int>> cr;  // [start, length) column ranges
    for (int c = 0; c < nf0;) {
      if (!col[c]) { ++c; continue; }
      int e = c;
      while (e < nf0 && col[e]) ++e;
      cr.push_back({c, e - c});
      c = e;
    }
    int ncols = 0;
    for (auto& r : cr) ncols += r.second;
    if (cr.size() > 4 || 2 * ncols > 3 * nf0 / 2 + 1) return;  // not worth it
    col_ranges_ = cr;
    const int rpos = n_[1] - n_[1] / 2, rneg = n_[1] / 2;  // mode rows [0, rpos) and [nf1 - rneg, nf1)
    row_ranges_.clear();
    if (rpos > 0) row_ranges_.push_back({0, rpos});
    if (rneg > 0) row_ranges_.push_back({nf1 - rneg, rneg});
    T2_.alloc(geom_.G());
    FB_CUDA(cudaMemset(T2_.p, 0, T2_.bytes()));
    const cufftType ty = sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z;
    for (auto& r : row_ranges_) plan_for(1, r.second, ty);
    for (auto& r : col_ranges_) plan_for(0, r.second, ty);
    pruned_ = true;
  }

  // batched 1D plan: kind 1 = rows (length nf0, contiguous), 0 = columns (length nf1, stride nf0)
  cufftHandle plan_for(int kind, int batch, cufftType ty) {
    const int64_t key = int64_t(kind) << 32 | uint32_t(batch);
    auto it = plans_.find(key);
    if (it != plans_.end()) return it->second;
    const int nf0 = int(geom_.nf[0]), nf1 = int(geom_.nf[1]);
    cufftHandle h = 0;
    if (kind == 1) {
      int n = nf0, emb = nf0;
      FB_CUFFT(cufftPlanMany(&h, 1, &n, &emb, 1, nf0, &emb, 1, nf0, ty, batch));
    } else {
      int n = nf1, emb = nf1;
      FB_CUFFT(cufftPlanMany(&h, 1, &n, &emb, nf0, 1, &emb, nf0, 1, ty, batch));
    }
    plans_[key] = h;
    return h;
  }

  void exec1(cufftHandle plan, cplx_t<T>* in, cplx_t<T>* out, int dir, cudaStream_t s) {
    FB_CUFFT(cufftSetStream(plan, s));
    if (sizeof(T) == 4) {
      FB_CUFFT(cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftComplex*>(out), dir));
    } else {
      FB_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(in),
                            reinterpret_cast<cufftDoubleComplex*>(out), dir));
    }
  }

  void rows_pass(cplx_t<T>* in, cplx_t<T>* out, int dir, cudaStream_t s) {
    const cufftType ty = sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z;
    const int64_t nf0 = geom_.nf[0];
    for (auto& r : row_ranges_) exec1(plan_for(1, r.second, ty), in + r.first * nf0, out + r.first * nf0, dir, s);
  }
  void cols_pass(cplx_t<T>* buf, int dir, cudaStream_t s) {
    const cufftType ty = sizeof(T) == 4 ? CUFFT_C2C : CUFFT_Z2Z;
    for (auto& r : col_ranges_) exec1(plan_for(0, r.second, ty), buf + r.first, buf + r.first, dir, s);
  }

  void run(const double* x, double* g, double* e, bool acc, cudaStream_t s) {
    timer_begin(s);
    begin_eval_status(s);
    if (!acc) FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double), s));
    const int grid = int(std::min<int64_t>(ceil_div(G_, kThreads), int64_t(sm_count()) * 8));
    uwnu_precorrect_kernel<T><<<grid, kThreads, 0, s>>>(x, G_, D_, n_[0], n_[1], n_[2], geom_, corr_[0].p, corr_[1].p,
                                                        corr_[2].p, H_.p, status_.p);
    FB_LAUNCH_CHECK();
    cplx_t<T>* t2 = Gf_.p;
    if (pruned_) {
      t2 = T2_.p;
      rows_pass(H_.p, t2, CUFFT_INVERSE, s);  // sign +1
      cols_pass(t2, CUFFT_INVERSE, s);
    } else {
      exec(H_.p, Gf_.p, CUFFT_INVERSE, s);  // sign +1
    }
    timer_mark("type2_fft", s);
    interp<T>(recs_.p, M_, nullptr, T(1), sort_, geom_, poly_, t2, 1, INTERP_CPLX, nullptr, rho_.p, 0, nullptr,
              s);
    timer_mark("type2_interp", s);
    const int mg = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(M_, kThreads), int64_t(sm_count()) * 4)));
    uwnu_loss_kernel<T><<<mg, kThreads, 0, s>>>(rho_.p, M_, sk_.p, v_.p, e, f_.p, g != nullptr);
    FB_LAUNCH_CHECK();
    timer_mark("loss", s);
    if (!g) return;
    FB_CUDA(cudaMemsetAsync(Gf_.p, 0, Gf_.bytes(), s));
    spread_cplx<T>(recs_.p, f_.p, sort_, geom_, poly_, Gf_.p, s);
    timer_mark("type1_spread", s);
    if (pruned_) {
      cols_pass(Gf_.p, CUFFT_FORWARD, s);  // sign -1, in place
      rows_pass(Gf_.p, Gf_.p, CUFFT_FORWARD, s);
    } else {
      exec(Gf_.p, Gf_.p, CUFFT_FORWARD, s);  // sign -1, in place
    }
    uwnu_extract_kernel<T><<<grid, kThreads, 0, s>>>(Gf_.p, G_, D_, n_[0], n_[1], n_[2], geom_, corr_[0].p,
                                                     corr_[1].p, corr_[2].p, g, acc ? 1 : 0,
                                                     grad_mode_ == 1 ? 1.0 : 1.0 / kTwoPi);
    FB_LAUNCH_CHECK();
    timer_mark("type1_fft_extract", s);
  }

  int D_;
  int n_[3] = {1, 1, 1};
  int64_t G_ = 1, M_ = 0;
  ESParams es_;
  std::vector<double> poly_;
  Geom geom_;
  SortBufs sort_;
  DevBuf<unsigned char> recs_;
  DevBuf<cplx_t<T>> H_, Gf_, f_;
  DevBuf<double> corr_[3], sk_, v_;
  DevBuf<double2> rho_;
  cufftHandle plan_ = 0;
  bool pruned_ = false;
  DevBuf<cplx_t<T>> T2_;  // type-2 transform output (pruned passes; rows outside the mode rows stay zero)
  std::vector<std::pair<int, int>> row_ranges_, col_ranges_;
  std::map<int64_t, cufftHandle> plans_;
};

}  // namespace

PotentialPtr make_uwnu(const std::vector<int>& grid, const std::vector<double>& kpts, const std::vector<double>& sk,
                       const std::vector<double>& v, const std::vector<double>& L, double eps, int precision) {
  if (precision == 1) return PotentialPtr(new UwNUImpl<float>(grid, kpts, sk, v, L, eps));
  return PotentialPtr(new UwNUImpl<double>(grid, kpts, sk, v, L, eps));
}

}  // namespace fb
