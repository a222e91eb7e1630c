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

}  // namespace fb
