// One-dimensional complex FFTs of a power-of-two length N (512..8192)
// computed by TPB = N / 16 threads in registers and shared memory, for the 2D
// NUwU transforms that only touch a band of modes.
//
// Algorithm: self-sorting (Stockham) decimation in frequency.  With
// N = p_1 p_2 ... p_r, stage t splits each of the s current sub-transforms of
// length L = p m (p = p_t) as j = j1 + m j2, k = p k1 + k2:
//   out[(j1 p + k2) s + q] = W_L^(j1 k2) sum_j2 in[(j1 + m j2) s + q] W_p^(j2 k2)
// with W_N = exp(-2 pi i / N) (the forward, sign -1 transform of cuFFT and
// FFTW); the output is in natural order.  The radices are 16 (as long as 16
// divides what is left) and then 8, 4 or 2, all compile-time constants, so a
// thread holds 16 elements, runs its butterflies in registers and exchanges
// data through shared memory once per stage.  Element i of a shared buffer
// lives at i + i / 16, which puts the radix-strided stores of the first stage
// in distinct banks.
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"

namespace fb {

// exp(-2 pi i j / n), j = 0..n-1, interleaved (re, im), computed in FP64.
inline std::vector<double> fft_twiddles(int n) {
  std::vector<double> t(2 * size_t(n));
  for (int j = 0; j < n; ++j) {
    const double a = -2.0 * 3.14159265358979323846 * double(j) / double(n);
    t[2 * size_t(j)] = std::cos(a);
    t[2 * size_t(j) + 1] = std::sin(a);
  }
  return t;
}

// Shared-memory elements a padded buffer of n entries occupies.
__host__ __device__ constexpr int fft_padded(int n) { return n + (n >> 4) + 1; }

#ifdef __CUDACC__
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

// complex helpers for float2 / double2 (cplx_t<T> is not deducible)
#define FB_CPLX_OPS(C)                                                                       \
  __device__ __forceinline__ C cmul(C a, C b) {                                              \
    C r;                                                                                     \
    r.x = a.x * b.x - a.y * b.y;                                                             \
    r.y = a.x * b.y + a.y * b.x;                                                             \
    return r;                                                                                \
  }                                                                                          \
  __device__ __forceinline__ C cadd(C a, C b) {                                              \
    C r;                                                                                     \
    r.x = a.x + b.x;                                                                         \
    r.y = a.y + b.y;                                                                         \
    return r;                                                                                \
  }                                                                                          \
  __device__ __forceinline__ C csub(C a, C b) {                                              \
    C r;                                                                                     \
    r.x = a.x - b.x;                                                                         \
    r.y = a.y - b.y;                                                                         \
    return r;                                                                                \
  }                                                                                          \
  /* multiplication by -i */                                                                 \
  __device__ __forceinline__ C cmul_mi(C a) {                                                \
    C r;                                                                                     \
    r.x = a.y;                                                                               \
    r.y = -a.x;                                                                              \
    return r;                                                                                \
  }
FB_CPLX_OPS(float2)
FB_CPLX_OPS(double2)
#undef FB_CPLX_OPS

// Forward DFT of P points in registers (W_P = exp(-2 pi i / P)).
template <typename T, int P>
struct SmallDft;

template <typename T>
struct SmallDft<T, 2> {
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[2], const cplx_t<T>*, int) {
    const cplx_t<T> a = u[0], b = u[1];
    u[0] = cadd(a, b);
    u[1] = csub(a, b);
  }
};

template <typename T>
struct SmallDft<T, 4> {
  __device__ __forceinline__ static void run4(cplx_t<T>& u0, cplx_t<T>& u1, cplx_t<T>& u2, cplx_t<T>& u3) {
    const cplx_t<T> t0 = cadd(u0, u2), t1 = csub(u0, u2), t2 = cadd(u1, u3), t3 = cmul_mi(csub(u1, u3));
    u0 = cadd(t0, t2);
    u2 = csub(t0, t2);
    u1 = cadd(t1, t3);
    u3 = csub(t1, t3);
  }
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[4], const cplx_t<T>*, int) { run4(u[0], u[1], u[2], u[3]); }
};

template <typename T>
struct SmallDft<T, 8> {
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[8], const cplx_t<T>*, int) {
    // even and odd halves, then X[k] = E[k] + W8^k O[k], X[k+4] = E[k] - W8^k O[k]
    cplx_t<T> e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
    cplx_t<T> o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
    SmallDft<T, 4>::run4(e0, e1, e2, e3);
    SmallDft<T, 4>::run4(o0, o1, o2, o3);
    const T h = T(0.70710678118654752440);  // 1 / sqrt(2)
    cplx_t<T> w1, w3;
    w1.x = (o1.x + o1.y) * h;  // o1 (1 - i) / sqrt 2
    w1.y = (o1.y - o1.x) * h;
    const cplx_t<T> w2 = cmul_mi(o2);
    w3.x = (o3.y - o3.x) * h;  // o3 (-1 - i) / sqrt 2
    w3.y = -(o3.x + o3.y) * h;
    u[0] = cadd(e0, o0);
    u[4] = csub(e0, o0);
    u[1] = cadd(e1, w1);
    u[5] = csub(e1, w1);
    u[2] = cadd(e2, w2);
    u[6] = csub(e2, w2);
    u[3] = cadd(e3, w3);
    u[7] = csub(e3, w3);
  }
};

template <typename T>
struct SmallDft<T, 3> {
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[3], const cplx_t<T>*, int) {
    const T s3 = T(-0.86602540378443864676);  // -sqrt(3)/2: imaginary part of W_3
    const cplx_t<T> t1 = cadd(u[1], u[2]);
    cplx_t<T> t2;
    t2.x = u[0].x - T(0.5) * t1.x;
    t2.y = u[0].y - T(0.5) * t1.y;
    const cplx_t<T> d = csub(u[1], u[2]);
    cplx_t<T> t3;  // d * (i s3)
    t3.x = -d.y * s3;
    t3.y = d.x * s3;
    u[0] = cadd(u[0], t1);
    u[1] = cadd(t2, t3);
    u[2] = csub(t2, t3);
  }
};

template <typename T>
struct SmallDft<T, 16> {
  // j = 4a + b, k = c + 4d: X[c + 4d] = sum_b W4^(bd) W16^(bc) sum_a x[4a + b] W4^(ac)
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[16], const cplx_t<T>*, int) {
    const T c1 = T(0.92387953251128675613), s1 = T(0.38268343236508977173), h = T(0.70710678118654752440);
#pragma unroll
    for (int b = 0; b < 4; ++b) SmallDft<T, 4>::run4(u[b], u[4 + b], u[8 + b], u[12 + b]);
    // Y_b[c] sits in u[4c + b]; multiply by W16^(bc)
    auto rot = [](cplx_t<T> v, T wr, T wi) {
      cplx_t<T> r;
      r.x = v.x * wr - v.y * wi;
      r.y = v.x * wi + v.y * wr;
      return r;
    };
    u[5] = rot(u[5], c1, -s1);    // b=1 c=1: W16^1
    u[9] = rot(u[9], h, -h);      // b=1 c=2: W16^2
    u[13] = rot(u[13], s1, -c1);  // b=1 c=3: W16^3
    u[6] = rot(u[6], h, -h);      // b=2 c=1: W16^2
    u[10] = cmul_mi(u[10]);       // b=2 c=2: W16^4 = -i
    u[14] = rot(u[14], -h, -h);   // b=2 c=3: W16^6
    u[7] = rot(u[7], s1, -c1);    // b=3 c=1: W16^3
    u[11] = rot(u[11], -h, -h);   // b=3 c=2: W16^6
    u[15] = rot(u[15], -c1, s1);  // b=3 c=3: W16^9
#pragma unroll
    for (int c = 0; c < 4; ++c) SmallDft<T, 4>::run4(u[4 * c], u[4 * c + 1], u[4 * c + 2], u[4 * c + 3]);
    // X[c + 4d] is now in u[4c + d]: transpose the 4 x 4 index
    cplx_t<T> v[16];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int d = 0; d < 4; ++d) v[c + 4 * d] = u[4 * c + d];
#pragma unroll
    for (int k = 0; k < 16; ++k) u[k] = v[k];
  }
};

// P = 5, 7: direct sums with W_P^r = tw[r n / P] from the length-n table.
template <typename T, int P>
struct SmallDft {
  __device__ __forceinline__ static void run(cplx_t<T> (&u)[P], const cplx_t<T>* __restrict__ tw, int n) {
    cplx_t<T> w[P];
#pragma unroll
    for (int r = 0; r < P; ++r) w[r] = tw[r * (n / P)];
    cplx_t<T> v[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      cplx_t<T> acc = u[0];
#pragma unroll
      for (int j = 1; j < P; ++j) acc = cadd(acc, cmul(u[j], w[(j * k) % P]));
      v[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < P; ++k) u[k] = v[k];
  }
};

// Barrier over the `count` threads of one transform (named barrier `id`, 1..15;
// count is a multiple of 32 and the participating warps are whole).
__device__ __forceinline__ void group_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// W^1..W^(P-1) from W^1 and W^4 (table entries) by at most four products.
template <typename T, int P>
__device__ __forceinline__ void twiddle_powers(cplx_t<T> (&w)[P], cplx_t<T> w1, cplx_t<T> w4) {
  w[1] = w1;
  if (P > 2) w[2] = cmul(w1, w1);
  if (P > 3) w[3] = cmul(w[2], w1);
  if (P > 4) {
    w[4] = w4;
    w[5] = cmul(w4, w1);
    w[6] = cmul(w4, w[2]);
    w[7] = cmul(w4, w[3]);
  }
  if (P > 8) {
    const cplx_t<T> w8 = cmul(w4, w4);
    w[8] = w8;
#pragma unroll
    for (int k = 9; k < 12; ++k) w[k % P] = cmul(w8, w[(k - 8) % P]);
    const cplx_t<T> w12 = cmul(w8, w4);
    w[12 % P] = w12;
#pragma unroll
    for (int k = 13; k < 16; ++k) w[k % P] = cmul(w12, w[(k - 12) % P]);
  }
}

// Forward FFT of length N by the TPB = N / 16 threads with lane index t.
// run() takes the 16 first-stage inputs of the thread (element t + j (N/16),
// j = 0..15) in v, leaves the natural-order result in the padded shared buffer
// buf, and synchronises the group (barrier id, TPB threads) before returning.
template <typename T, int N>
struct RegFft {
  static_assert(N >= 512 && N <= 8192 && (N & (N - 1)) == 0, "power-of-two length 512..8192");
  static constexpr int E = 16;
  static constexpr int TPB = N / E;
  // bar.sync counts whole warps, and a transform must own its warps
  static_assert(TPB % 32 == 0, "a transform needs a multiple of 32 threads");

  template <int S>
  static constexpr int radix() {
    return (N / S) % 16 == 0 ? 16 : N / S;
  }

  template <int S>
  __device__ static void stage(cplx_t<T> (&v)[E], cplx_t<T>* buf, const cplx_t<T>* __restrict__ tw, int t,
                               int bar) {
    constexpr int P = radix<S>();
    constexpr int NB = E / P;  // butterflies per thread
    constexpr int SP = S * P;
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const int idx = t + i * TPB;
      const int j1 = idx / S, q = idx % S;
      cplx_t<T> u[P];
#pragma unroll
      for (int j2 = 0; j2 < P; ++j2) u[j2] = v[i * P + j2];
      SmallDft<T, P>::run(u, tw, N);
      const int ob = j1 * SP + q;
      buf[fpad(ob)] = u[0];
      if (SP < N) {  // the last stage has j1 = 0: no twiddles
        cplx_t<T> w[P];
        twiddle_powers<T, P>(w, tw[j1 * S], P > 4 ? tw[(4 * j1 * S) % N] : tw[0]);
#pragma unroll
        for (int k2 = 1; k2 < P; ++k2) u[k2] = cmul(u[k2], w[k2]);
      }
#pragma unroll
      for (int k2 = 1; k2 < P; ++k2) buf[fpad(ob + k2 * S)] = u[k2];
    }
    group_sync(bar, TPB);
    if constexpr (SP < N) {
      constexpr int P2 = radix<SP>();
      constexpr int NB2 = E / P2;
#pragma unroll
      for (int i = 0; i < NB2; ++i)
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) v[i * P2 + j2] = buf[fpad(t + i * TPB + j2 * (N / P2))];
      group_sync(bar, TPB);
      stage<SP>(v, buf, tw, t, bar);
    }
  }

  __device__ static void run(cplx_t<T> (&v)[E], cplx_t<T>* buf, const cplx_t<T>* __restrict__ tw, int t, int bar) {
    stage<1>(v, buf, tw, t, bar);
  }
};
#endif

}  // namespace fb
