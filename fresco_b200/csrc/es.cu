// Host-side ES kernel set-up: parameters, smooth FFT sizes and the Fourier
// correction factors (see es.cuh for the method and its source).
#include "es.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace fb {

ESParams es_params(double eps, int wmax) {
  if (!(eps > 0.0) || !std::isfinite(eps)) throw std::invalid_argument("eps must be positive and finite");
  ESParams p;
  int w = int(std::ceil(std::log10(1.0 / eps))) + 1;
  w = std::max(2, std::min(w, wmax));
  p.w = w;
  double beta_over_w = 2.30;
  if (w == 2) beta_over_w = 2.20;
  else if (w == 3) beta_over_w = 2.26;
  else if (w == 4) beta_over_w = 2.38;
  p.beta = beta_over_w * w;
  p.eps_eff = std::pow(10.0, -(w - 1));
  return p;
}

static bool smooth7(int64_t n) {
  for (int64_t f : {2, 3, 5, 7})
    while (n % f == 0) n /= f;
  return n == 1;
}

int64_t next_smooth_even(int64_t n) {
  if (n < 2) n = 2;
  if (n % 2) ++n;
  while (!smooth7(n)) n += 2;
  return n;
}

int64_t fine_grid_size(int64_t n_modes, int w) {
  const int64_t kmax = n_modes / 2;
  int64_t target = std::max<int64_t>({4 * kmax, n_modes + 1, 2 * int64_t(w)});
  return next_smooth_even(target);
}

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& wts) {
  x.assign(n, 0.0);
  wts.assign(n, 0.0);
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    wts[i] = wts[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

std::vector<double> es_correction(const ESParams& es, int64_t nf, int64_t kmin, int64_t count) {
  const int nq = std::max(64, 8 * es.w + 64);
  std::vector<double> xq, wq;
  gauss_legendre(nq, xq, wq);
  std::vector<double> phiq(nq);
  for (int q = 0; q < nq; ++q) phiq[q] = wq[q] * es_phi(xq[q], es.beta);
  const double pi = 3.14159265358979323846;
  const double scale = es.w * pi / double(nf);
  std::vector<double> out(count);
  for (int64_t i = 0; i < count; ++i) {
    const double k = double(kmin + i);
    double s = 0.0;
    for (int q = 0; q < nq; ++q) s += phiq[q] * std::cos(k * scale * xq[q]);
    out[i] = 0.5 * es.w * s;
  }
  return out;
}

std::vector<double> es_poly_coefficients(const ESParams& es, int W) {
  const int Q = W + 2;
  const int n = 4 * Q + 40;  // Chebyshev nodes for the fit
  const double pi = 3.14159265358979323846;
  std::vector<double> out(size_t(W) * (Q + 1), 0.0);
  std::vector<double> xk(n), cheb(Q + 1);
  for (int j = 0; j < n; ++j) xk[j] = std::cos(pi * (j + 0.5) / n);  // in [-1, 1], u = x / 2
  for (int m = 0; m < W; ++m) {
    const double a = m - 0.5 * (W - 1);
    // Chebyshev coefficients of g(x) = phi((a - x/2) * 2/W) from the discrete orthogonality sums
    for (int k = 0; k <= Q; ++k) {
      double sum = 0.0;
      for (int j = 0; j < n; ++j) sum += es_phi((a - 0.5 * xk[j]) * 2.0 / W, es.beta) * std::cos(k * pi * (j + 0.5) / n);
      cheb[k] = (k == 0 ? 1.0 : 2.0) * sum / n;
    }
    // sum_k cheb_k T_k(x) -> monomials in x (T_{k+1} = 2x T_k - T_{k-1}) -> monomials in u (x = 2u)
    std::vector<double> tkm1(Q + 1, 0.0), tk(Q + 1, 0.0), mono(Q + 1, 0.0);
    tkm1[0] = 1.0;      // T_0
    tk[1] = 1.0;        // T_1
    mono[0] += cheb[0];
    if (Q >= 1) mono[1] += cheb[1];
    for (int k = 1; k < Q; ++k) {
      std::vector<double> tn(Q + 1, 0.0);
      for (int d = 0; d < Q; ++d) tn[d + 1] += 2.0 * tk[d];
      for (int d = 0; d <= Q; ++d) tn[d] -= tkm1[d];
      for (int d = 0; d <= Q; ++d) mono[d] += cheb[k + 1] * tn[d];
      tkm1 = tk;
      tk = tn;
    }
    double scale = 1.0;
    for (int d = 0; d <= Q; ++d) {
      out[size_t(m) * (Q + 1) + d] = mono[d] * scale;
      scale *= 2.0;
    }
  }
  return out;
}

double es_fourier(const ESParams& es, double z) {
  static thread_local int cached_n = 0;
  static thread_local std::vector<double> xq, wq;
  const int nq = std::max(64, 8 * es.w + 64) + int(std::ceil(std::fabs(z)));
  if (nq != cached_n) {
    gauss_legendre(nq, xq, wq);
    cached_n = nq;
  }
  double s = 0.0;
  for (int q = 0; q < nq; ++q) s += wq[q] * es_phi(xq[q], es.beta) * std::cos(z * xq[q]);
  return s;
}

std::vector<double> es_fourier_chebyshev(const ESParams& es, double zmax) {
  const double pi = 3.14159265358979323846;
  // F is entire and of exponential type 1 in z: on [-zmax, zmax] its Chebyshev
  // coefficients fall off once the degree passes zmax; 40 more terms reach
  // the FP64 level
  const int n = int(std::ceil(zmax)) + 40;
  const int m = 2 * n + 16;  // Chebyshev nodes of the interpolant
  std::vector<double> f(m);
  for (int j = 0; j < m; ++j) f[j] = es_fourier(es, zmax * std::cos(pi * (j + 0.5) / m));
  std::vector<double> c(n + 1);
  for (int k = 0; k <= n; ++k) {
    double sum = 0.0;
    for (int j = 0; j < m; ++j) sum += f[j] * std::cos(k * pi * (j + 0.5) / m);
    c[k] = (k == 0 ? 1.0 : 2.0) * sum / m;
  }
  return c;
}

}  // namespace fb
