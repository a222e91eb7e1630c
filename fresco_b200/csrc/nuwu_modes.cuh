// The NUwU mode pass shared by the single-pattern potential and the batched
// ensemble: the active-mode table (source/fresco/nuwu.hpp:260-287) and the
// per-mode device arithmetic (deconvolution, S, d, phi, packed type-2 field).
//
// For real weights, Re T2(f) = T2(f^H) with f^H(k) = (f(k) + conj f(-k))/2, so
// the field h = f_x^H + i f_y^H returns both gradient components of 2D as the
// real and imaginary parts of one type-2 transform (3D adds a second field
// for z).  f_a^H = -i k_a F^H with F^H(k) = (2/N) rho(k) [A(k) q - B(k)],
// q = |rho|^2/N, where A and B fold V and S0 at k and -k.
#pragma once

#include <vector>

#include "common.cuh"

namespace fb {

struct ModeCoef {
  double A, B, w2, s0;  // A, B as above; w2 = V/S0'^2, s0 = S0 (phi = w2 (q - s0)^2)
};

// Active modes (V(k) != 0 or V(-k) != 0) of the n^D mode grid, x fastest
// (flat = ix + n iy [+ n^2 iz], nuwu.hpp:277-285), with their coefficients.
inline void nuwu_mode_table(int D, int n, const double* v, const double* sk, std::vector<int>& idx,
                            std::vector<ModeCoef>& coef) {
  int64_t nm = 1;
  for (int a = 0; a < D; ++a) nm *= n;
  idx.clear();
  coef.clear();
  for (int64_t m = 0; m < nm; ++m) {
    int64_t r = m, mm = 0, stride = 1;
    for (int a = 0; a < D; ++a) {  // the mode -k
      const int64_t ia = r % n;
      r /= n;
      mm += (n - 1 - ia) * stride;
      stride *= n;
    }
    const double vk = v[m], vm = v[mm];
    if (vk == 0.0 && vm == 0.0) continue;
    const double s0k = sk[m], s0m = sk[mm];
    const double dk = s0k != 0.0 ? s0k : 1.0, dm = s0m != 0.0 ? s0m : 1.0;
    ModeCoef cc;
    cc.A = vk / (dk * dk) + vm / (dm * dm);
    cc.B = vk * s0k / (dk * dk) + vm * s0m / (dm * dm);
    cc.w2 = vk / (dk * dk);
    cc.s0 = s0k;
    idx.push_back(int(m));
    coef.push_back(cc);
  }
}

#ifdef __CUDACC__
// rho(k) of active mode m (flat index on the n^D grid, K = n/2) read from the
// R2C output bhat (sign -1, so rho(k) = conj(B(k)) for k_x >= 0 and B(-k)
// otherwise), before the deconvolution.  It is linear in the points, so the
// values of disjoint point sets add up to the value of their union.
template <int D, typename T>
__device__ __forceinline__ double2 nuwu_mode_rho(int m, int n, int K, const cplx_t<T>* __restrict__ bhat, int nh0,
                                                 int nf1, int nf2) {
  const int kx = m % n - K;
  const int ky = (D >= 2) ? (m / n) % n - K : 0;
  const int kz = (D >= 3) ? m / (n * n) - K : 0;
  int64_t bi;
  bool cj;
  if (kx >= 0) {
    const int yy = ky < 0 ? ky + nf1 : ky;
    const int zz = kz < 0 ? kz + nf2 : kz;
    bi = kx + int64_t(nh0) * (yy + int64_t(nf1) * zz);
    cj = true;
  } else {
    const int yy = ky > 0 ? nf1 - ky : -ky;
    const int zz = kz > 0 ? nf2 - kz : -kz;
    bi = -kx + int64_t(nh0) * (yy + int64_t(nf1) * zz);
    cj = false;
  }
  const cplx_t<T> b = bhat[bi];
  return make_double2(double(b.x), cj ? -double(b.y) : double(b.y));
}

// The mode's phi term from rho(k) (undeconvolved): deconvolves it by
// p(k) = prod corr_a(k_a) and, with want_grad, writes the packed field at k
// (hgrid; in 3D the z field's half spectrum k_x >= 0 follows at hgrid + G).
template <int D, typename T>
__device__ __forceinline__ double nuwu_mode_apply(int m, int n, int K, const ModeCoef& c, double2 rho, int nf0,
                                                  int nf1, int nf2, const double* __restrict__ corr0,
                                                  const double* __restrict__ corr1, const double* __restrict__ corr2,
                                                  double invN, cplx_t<T>* hgrid, int64_t G, bool want_grad) {
  const int kx = m % n - K;
  const int ky = (D >= 2) ? (m / n) % n - K : 0;
  const int kz = (D >= 3) ? m / (n * n) - K : 0;
  double p = corr0[kx + K];
  if (D >= 2) p *= corr1[ky + K];
  if (D >= 3) p *= corr2[kz + K];
  const double rr = rho.x / p;
  const double ri = rho.y / p;
  const double q = (rr * rr + ri * ri) * invN;
  const double dq = q - c.s0;
  if (want_grad) {
    const double a = (c.A * q - c.B) * (2.0 * invN) / p;  // includes the type-2 pre-correction 1/p
    const double fr = rr * a, fi = ri * a;                 // F^H / p
    const int x0 = kx < 0 ? kx + nf0 : kx;
    const int y0 = ky < 0 ? ky + nf1 : ky;
    const int z0 = kz < 0 ? kz + nf2 : kz;
    const int64_t hi = x0 + int64_t(nf0) * (y0 + int64_t(nf1) * z0);
    cplx_t<T> h;
    if (D == 1) {
      // -i kx F
      h.x = T(fi * kx);
      h.y = T(-fr * kx);
    } else {
      // F (ky - i kx)
      h.x = T(fr * ky + fi * kx);
      h.y = T(fi * ky - fr * kx);
    }
    hgrid[hi] = h;
    if (D == 3 && kx >= 0) {
      // -i kz F^H is Hermitian, so its type-2 transform (exponent -i) is real:
      // the C2R transform (exponent +i) of the conjugate, stored as the half
      // spectrum k_x >= 0 (nf0 / 2 + 1 cells per row)
      cplx_t<T> h2;
      h2.x = T(fi * kz);
      h2.y = T(fr * kz);
      hgrid[G + x0 + int64_t(nf0 / 2 + 1) * (y0 + int64_t(nf1) * z0)] = h2;
    }
  }
  return c.w2 * dq * dq;
}

// One active mode m: reads rho(k) from bhat, returns the mode's phi term and,
// with want_grad, writes the packed field at k.
template <int D, typename T>
__device__ __forceinline__ double nuwu_mode_term(int m, int n, int K, const ModeCoef& c,
                                                 const cplx_t<T>* __restrict__ bhat, int nh0, int nf0, int nf1,
                                                 int nf2, const double* __restrict__ corr0,
                                                 const double* __restrict__ corr1, const double* __restrict__ corr2,
                                                 double invN, cplx_t<T>* hgrid, int64_t G, bool want_grad) {
  return nuwu_mode_apply<D, T>(m, n, K, c, nuwu_mode_rho<D, T>(m, n, K, bhat, nh0, nf1, nf2), nf0, nf1, nf2, corr0,
                               corr1, corr2, invN, hgrid, G, want_grad);
}
#endif

}  // namespace fb
