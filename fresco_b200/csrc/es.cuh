// "Exponential of semicircle" (ES) spreading kernel: parameters, device
// evaluation and the Fourier-side correction factors.
//
// Written from Barnett, Magland & af Klinteberg, "A parallel non-uniform fast
// Fourier transform library based on an exponential of semicircle kernel",
// SIAM J. Sci. Comput. 41(5), 2019: phi(t) = exp(beta*(sqrt(1-t^2)-1)) on
// |t| <= 1, a kernel of w fine-grid points, beta = 2.30 w at upsampling 2,
// and correction by the kernel's Fourier transform evaluated by quadrature.
// FINUFFT v2.2.0 (the library the reference calls at source/fresco/nuwu.hpp:
// 50-51, 191-192, 256-258, 291-309) implements the same published method.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace fb {

struct ESParams {
  int w = 7;            // kernel width in fine-grid points
  double beta = 16.1;   // shape parameter
  double eps_eff = 1e-6;
};

// Kernel width / shape for tolerance eps.  w = ceil(log10(1/eps)) + 1,
// clamped to [2, wmax]; beta = 2.30 w (slightly adjusted for w <= 4).
ESParams es_params(double eps, int wmax);

// Smallest even integer >= n whose only prime factors are 2, 3, 5, 7
// (sizes cuFFT transforms without a Bluestein pass).
int64_t next_smooth_even(int64_t n);

// Fine-grid size for n modes: large enough that the highest mode |k|max =
// floor(n/2) and its alias nf - |k|max are as far apart as at upsampling 2
// (nf >= 4 |k|max), at least n + 1 and at least 2w.
int64_t fine_grid_size(int64_t n_modes, int w);

// Correction factors p(k) = psi_hat(k) / h for k = kmin .. kmin + count - 1,
// where psi(x) = phi(2x / (w h)), h = 2 pi / nf.  Computed in FP64 by
// Gauss-Legendre quadrature: p(k) = (w/2) int_{-1}^{1} phi(t) cos(k w pi t / nf) dt.
std::vector<double> es_correction(const ESParams& es, int64_t nf, int64_t kmin, int64_t count);

// Gauss-Legendre nodes/weights on [-1, 1] (Newton iteration on P_n).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& wts);

// Fourier transform of the kernel on its own support, F(z) = int_{-1}^{1}
// phi(t) cos(z t) dt (Gauss-Legendre quadrature, FP64).  A kernel of
// half-width a in some coordinate has the transform a F(xi a) at xi.
double es_fourier(const ESParams& es, double z);

// Chebyshev coefficients c_0..c_n of F on [-zmax, zmax] (F(z) = sum_k c_k
// T_k(z / zmax)), n large enough that the series matches F to about 1e-15
// relative to F(0) there; evaluated on the device by Clenshaw's recurrence.
std::vector<double> es_fourier_chebyshev(const ESParams& es, double zmax);

// Host evaluation of phi(t) (for tests and the quadrature).
inline double es_phi(double t, double beta) {
  const double a = 1.0 - t * t;
  return a >= 0.0 ? std::exp(beta * (std::sqrt(a) - 1.0)) : 0.0;
}

// Piecewise-polynomial form of the kernel taps (the approach of the ES paper,
// section on fast kernel evaluation): with the fractional cell offset f of a
// point, the W taps sit at z_m = (m - (W-1)/2) - u, where u = f - 1/2 for even
// W and u = f (f <= 1/2) or f - 1 (f > 1/2) for odd W, so u lies in
// [-1/2, 1/2].  Each tap is a degree-(W+2) polynomial in u, fitted at set-up
// by Chebyshev interpolation and evaluated with Horner's rule; the fit error
// is about 30x below the kernel's own truncation error for every W.
template <int W>
struct EsPolyDeg {
  static constexpr int Q = W + 2;
};

// Monomial coefficients c[m * (Q+1) + d] of tap m in powers u^d.
std::vector<double> es_poly_coefficients(const ESParams& es, int W);

template <int W, typename T>
struct EsPoly {
  T c[W][EsPolyDeg<W>::Q + 1];
};

template <int W, typename T>
inline EsPoly<W, T> make_es_poly(const std::vector<double>& coef) {
  constexpr int Q = EsPolyDeg<W>::Q;
  EsPoly<W, T> p;
  for (int m = 0; m < W; ++m)
    for (int d = 0; d <= Q; ++d) p.c[m][d] = T(coef[size_t(m) * (Q + 1) + d]);
  return p;
}

#ifdef __CUDACC__
// Start offset s of the W taps (relative to the point's cell) and the
// polynomial variable u for a fractional offset f in [0, 1).
template <int W, typename T>
__device__ __forceinline__ int es_start(T f, T& u) {
  if (W % 2 == 0) {
    u = f - T(0.5);
    return -W / 2 + 1;
  }
  const bool hi = f > T(0.5);
  u = hi ? f - T(1) : f;
  return -(W - 1) / 2 + (hi ? 1 : 0);
}

template <int W, typename T>
__device__ __forceinline__ T es_poly_tap(const EsPoly<W, T>& p, int m, T u) {
  constexpr int Q = EsPolyDeg<W>::Q;
  T v = p.c[m][Q];
#pragma unroll
  for (int d = Q - 1; d >= 0; --d) v = fma(v, u, p.c[m][d]);
  return v;
}

// All W tap values of a point at fractional offset f; returns the start offset.
template <int W, typename T>
__device__ __forceinline__ int es_taps(T f, const EsPoly<W, T>& p, T (&kv)[W]) {
  T u;
  const int s = es_start<W, T>(f, u);
#pragma unroll
  for (int m = 0; m < W; ++m) kv[m] = es_poly_tap<W, T>(p, m, u);
  return s;
}
#endif

}  // namespace fb
