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

// Host evaluation of phi(t) (for tests and the quadrature).
inline double es_phi(double t, double beta) {
  const double a = 1.0 - t * t;
  return a >= 0.0 ? std::exp(beta * (std::sqrt(a) - 1.0)) : 0.0;
}

#ifdef __CUDACC__
// Device evaluation of the w kernel values for a point at fractional cell
// offset f in [0, 1): taps m = 0..w-1 sit at grid offsets s+m relative to the
// point's cell, with z = s + m - f in (-w/2, w/2].  Returns s.
template <int W, typename T>
__device__ __forceinline__ int es_taps(T f, T beta, T (&kv)[W]) {
  int s;
  if (W % 2 == 0) {
    s = -W / 2 + (f > T(0) ? 1 : 0);
  } else {
    s = -(W - 1) / 2 + (f > T(0.5) ? 1 : 0);
  }
  const T inv_half = T(2) / T(W);
#pragma unroll
  for (int m = 0; m < W; ++m) {
    const T z = (T(s + m) - f) * inv_half;
    const T a = T(1) - z * z;
    T v;
    if (sizeof(T) == 4) {
      v = a >= T(0) ? expf(float(beta) * (sqrtf(float(a)) - 1.0f)) : T(0);
    } else {
      v = a >= T(0) ? exp(double(beta) * (sqrt(double(a)) - 1.0)) : T(0);
    }
    kv[m] = v;
  }
  return s;
}
#endif

}  // namespace fb
