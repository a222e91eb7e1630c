// Oracle implementation of the FINUFFT and FFTW entry points the reference
// calls (test infrastructure only; see finufft.h / fftw3.h in this folder).
//
//  * exact mode: direct FP64 sums, the quantity FINUFFT approximates;
//  * ES mode: a CPU ES-kernel NUFFT (types 1 and 2) restated from Barnett,
//    Magland & af Klinteberg, SIAM J. Sci. Comput. 41(5), 2019: fine grid
//    nf = smallest 2,3,5-smooth even number >= max(2n, 2w), kernel
//    exp(beta (sqrt(1 - t^2) - 1)) of w = ceil(log10(10/tol)) points,
//    beta = 2.30 w, correction by Gauss-Legendre quadrature of the kernel's
//    Fourier transform.  Spreading uses a tile colouring so that OpenMP
//    threads never write the same grid cell; everything is FP64.
//  * the FFT is a self-sorting mixed-radix (4, 2, 3 and generic odd primes)
//    transform on the CPU.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "fftw3.h"
#include "finufft.h"

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;

int g_mode = 0;  // 0 auto, 1 exact, 2 ES

// Wall seconds spent per ES stage since the last reset: setpts (coordinate
// map and bin sort), spread, FFT, mode copy with correction, interpolation.
enum { kProfSetpts, kProfSpread, kProfFft, kProfModes, kProfInterp, kProfN };
double g_prof[kProfN] = {0, 0, 0, 0, 0};
struct ProfScope {
  int slot;
  double t0;
  explicit ProfScope(int s) : slot(s), t0(omp_get_wtime()) {}
  ~ProfScope() { g_prof[slot] += omp_get_wtime() - t0; }
};

// ---------------------------------------------------------------------------
// mixed-radix FFT
// ---------------------------------------------------------------------------

// Self-sorting (Stockham) mixed-radix FFT.  Stage t splits each of the s
// current sub-transforms of length L = p m as j = j1 + m j2, k = p k1 + k2:
//   C[j1 s p + s k2 + q] = W_L^(j1 k2) sum_j2 B[(j1 + m j2) s + q] W_p^(j2 k2),
// so the sub-transform index q stays the fastest-varying part of the output
// index and no bit reversal is needed.
struct Fft1 {
  int n = 1;
  int sign = 1;
  std::vector<cd> tw;  // exp(sign 2 pi i j / n)
  std::vector<int> fac;

  Fft1(int n_, int sign_) : n(n_), sign(sign_) {
    tw.resize(n);
    for (int j = 0; j < n; ++j) {
      const double a = sign * 2.0 * kPi * double(j) / double(n);
      tw[j] = cd(std::cos(a), std::sin(a));
    }
    int r = n;
    while (r % 4 == 0) { fac.push_back(4); r /= 4; }
    while (r % 2 == 0) { fac.push_back(2); r /= 2; }
    for (int p = 3; p * p <= r; p += 2)
      while (r % p == 0) { fac.push_back(p); r /= p; }
    if (r > 1) fac.push_back(r);
  }

  // In-place transforms of B interleaved lines (element j of line b at
  // x[j B + b]); work holds n B elements.  Interleaving scales every index
  // stride of the recursion by B while the twiddles stay those of one line,
  // so the innermost loops run over s B contiguous elements.
  void exec(cd* x, cd* work, int B = 1) const {
    cd* a = x;
    cd* b = work;
    long s = 1, L = n;
    const cd wi(0.0, double(sign));
    const double s3 = sign * 0.86602540378443864676;
    std::vector<cd> gen;
    for (int p : fac) {
      const long m = L / p;
      const long sb = s * B;
      if (p > 4 && p != 3 && int(gen.size()) < p) gen.resize(2 * p);
      for (long j1 = 0; j1 < m; ++j1) {
        const cd* in = a + j1 * sb;
        cd* out = b + j1 * sb * p;
        if (p == 4) {
          const cd w1 = tw[size_t(j1 * s)], w2 = tw[size_t(2 * j1 * s)], w3 = tw[size_t(3 * j1 * s)];
          for (long q = 0; q < sb; ++q) {
            const cd u0 = in[q], u1 = in[m * sb + q], u2 = in[2 * m * sb + q], u3 = in[3 * m * sb + q];
            const cd t0 = u0 + u2, t1 = u0 - u2, t2 = u1 + u3, t3 = (u1 - u3) * wi;
            out[q] = t0 + t2;
            out[sb + q] = (t1 + t3) * w1;
            out[2 * sb + q] = (t0 - t2) * w2;
            out[3 * sb + q] = (t1 - t3) * w3;
          }
        } else if (p == 2) {
          const cd w1 = tw[size_t(j1 * s)];
          for (long q = 0; q < sb; ++q) {
            const cd u0 = in[q], u1 = in[m * sb + q];
            out[q] = u0 + u1;
            out[sb + q] = (u0 - u1) * w1;
          }
        } else if (p == 3) {
          const cd w1 = tw[size_t(j1 * s)], w2 = tw[size_t(2 * j1 * s)];
          for (long q = 0; q < sb; ++q) {
            const cd u0 = in[q], u1 = in[m * sb + q], u2 = in[2 * m * sb + q];
            const cd t1 = u1 + u2, t2 = u0 - 0.5 * t1, t3 = (u1 - u2) * cd(0.0, s3);
            out[q] = u0 + t1;
            out[sb + q] = (t2 + t3) * w1;
            out[2 * sb + q] = (t2 - t3) * w2;
          }
        } else {
          cd* u = gen.data();
          cd* v = gen.data() + p;
          const int np = n / p;
          for (long q = 0; q < sb; ++q) {
            for (int j2 = 0; j2 < p; ++j2) u[j2] = in[j2 * m * sb + q];
            for (int k2 = 0; k2 < p; ++k2) {
              cd acc = 0.0;
              for (int j2 = 0; j2 < p; ++j2) acc += u[j2] * tw[size_t((j2 * k2) % p) * np];
              v[k2] = acc;
            }
            for (int k2 = 0; k2 < p; ++k2) out[sb * k2 + q] = v[k2] * tw[size_t(j1 * k2 * s)];
          }
        }
      }
      std::swap(a, b);
      s *= p;
      L = m;
    }
    if (a != x) std::memcpy(x, a, sizeof(cd) * size_t(n) * B);
  }
};

// Twiddle tables are built once per (size, sign).
const Fft1& fft_plan_cached(int n, int sign) {
  static std::vector<std::unique_ptr<Fft1>> cache;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  for (auto& f : cache)
    if (f->n == n && f->sign == sign) return *f;
  cache.emplace_back(new Fft1(n, sign));
  return *cache.back();
}

// In-place unnormalised multi-dimensional DFT, row-major dims (last fastest).
// Lines are transformed kBlk at a time, interleaved (Fft1::exec with B =
// kBlk): along a strided axis kBlk neighbouring lines are gathered so that
// every cache line read is fully used; along the contiguous axis kBlk rows
// are transposed into the interleaved layout.
void fft_nd(cd* data, const std::vector<int>& dims, int sign) {
  constexpr int kBlk = 16;
  const int r = int(dims.size());
  size_t total = 1;
  for (int d : dims) total *= size_t(d);
  for (int a = 0; a < r; ++a) {
    const int n = dims[a];
    if (n == 1) continue;
    size_t stride = 1;
    for (int b = a + 1; b < r; ++b) stride *= size_t(dims[b]);
    const size_t nouter = total / (size_t(n) * stride);
    const Fft1& f = fft_plan_cached(n, sign);
    if (stride == 1) {
      const size_t nblk = (nouter + kBlk - 1) / kBlk;
#pragma omp parallel
      {
        std::vector<cd> blk(size_t(n) * kBlk, cd(0.0, 0.0)), work(size_t(n) * kBlk);
#pragma omp for schedule(static)
        for (long bi = 0; bi < long(nblk); ++bi) {
          const size_t l0 = size_t(bi) * kBlk;
          const int w = int(std::min<size_t>(kBlk, nouter - l0));
          for (int b = 0; b < w; ++b) {
            const cd* line = data + (l0 + b) * size_t(n);
            for (int j = 0; j < n; ++j) blk[size_t(j) * kBlk + b] = line[j];
          }
          f.exec(blk.data(), work.data(), kBlk);
          for (int b = 0; b < w; ++b) {
            cd* line = data + (l0 + b) * size_t(n);
            for (int j = 0; j < n; ++j) line[j] = blk[size_t(j) * kBlk + b];
          }
        }
      }
      continue;
    }
    const size_t nblk = (stride + kBlk - 1) / kBlk;
#pragma omp parallel
    {
      std::vector<cd> blk(size_t(n) * kBlk, cd(0.0, 0.0)), work(size_t(n) * kBlk);
#pragma omp for schedule(static)
      for (long bi = 0; bi < long(nouter * nblk); ++bi) {
        const size_t outer = size_t(bi) / nblk, i0 = (size_t(bi) % nblk) * kBlk;
        const int w = int(std::min<size_t>(kBlk, stride - i0));
        cd* base = data + outer * stride * n + i0;
        for (int j = 0; j < n; ++j)
          for (int b = 0; b < w; ++b) blk[size_t(j) * kBlk + b] = base[size_t(j) * stride + b];
        f.exec(blk.data(), work.data(), kBlk);
        for (int j = 0; j < n; ++j)
          for (int b = 0; b < w; ++b) base[size_t(j) * stride + b] = blk[size_t(j) * kBlk + b];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// ES kernel helpers
// ---------------------------------------------------------------------------

int64_t next235even(int64_t n) {
  if (n < 2) n = 2;
  if (n % 2) ++n;
  for (;; n += 2) {
    int64_t r = n;
    for (int f : {2, 3, 5})
      while (r % f == 0) r /= f;
    if (r == 1) return n;
  }
}

void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), pp = 0.0;
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
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

inline double es_phi(double t, double beta) {
  const double a = 1.0 - t * t;
  return a >= 0.0 ? std::exp(beta * (std::sqrt(a) - 1.0)) : 0.0;
}

// Fourier correction p(k) = psi_hat(k)/h for k = -n/2 .. (n-1)/2.
std::vector<double> correction(int w, double beta, int64_t nf, int64_t n) {
  const int nq = std::max(64, 8 * w + 64);
  std::vector<double> xq, wq;
  gauss_legendre(nq, xq, wq);
  std::vector<double> out(n);
  for (int64_t i = 0; i < n; ++i) {
    const double k = double(i - n / 2);
    double s = 0.0;
    for (int q = 0; q < nq; ++q) s += wq[q] * es_phi(xq[q], beta) * std::cos(k * w * kPi / double(nf) * xq[q]);
    out[i] = 0.5 * w * s;
  }
  return out;
}

// Piecewise-polynomial kernel taps, FINUFFT's default way of evaluating the
// kernel (Horner's rule on a polynomial per tap; the ES paper's section on
// fast kernel evaluation).  With the fractional cell offset f of a point the
// w taps sit at t_m = (m - (w-1)/2 - u) 2/w, where u = f - 1/2 for even w
// and u = f (f <= 1/2) or f - 1 (f > 1/2) for odd w, so u is in [-1/2, 1/2].
// Each tap is a degree-(w+3) polynomial in u, fitted once per plan by
// Chebyshev interpolation at 4(w+3)+40 nodes; the fit error is far below the
// kernel's own truncation error.
constexpr int kPolyExtra = 3;

std::vector<double> tap_polynomials(int w, double beta) {
  const int Q = w + kPolyExtra;
  const int n = 4 * Q + 40;
  std::vector<double> out(size_t(w) * (Q + 1), 0.0), cheb(Q + 1);
  for (int m = 0; m < w; ++m) {
    const double a = m - 0.5 * (w - 1);
    for (int k = 0; k <= Q; ++k) {
      double sum = 0.0;
      for (int j = 0; j < n; ++j) {
        const double xj = std::cos(kPi * (j + 0.5) / n);  // node in [-1, 1]; u = xj / 2
        sum += es_phi((a - 0.5 * xj) * 2.0 / w, beta) * std::cos(k * kPi * (j + 0.5) / n);
      }
      cheb[k] = (k == 0 ? 1.0 : 2.0) * sum / n;
    }
    // Chebyshev series in x -> monomials in x (three-term recurrence) -> monomials in u = x / 2
    std::vector<double> tkm1(Q + 1, 0.0), tk(Q + 1, 0.0), mono(Q + 1, 0.0);
    tkm1[0] = 1.0;
    tk[1] = 1.0;
    mono[0] = cheb[0];
    mono[1] = cheb[1];
    for (int k = 1; k < Q; ++k) {
      std::vector<double> tn(Q + 1, 0.0);
      for (int d = 0; d < Q; ++d) tn[d + 1] += 2.0 * tk[d];
      for (int d = 0; d <= Q; ++d) tn[d] -= tkm1[d];
      for (int d = 0; d <= Q; ++d) mono[d] += cheb[k + 1] * tn[d];
      tkm1 = tk;
      tk = tn;
    }
    double scale = 1.0;
    for (int d = 0; d <= Q; ++d, scale *= 2.0) out[size_t(m) * (Q + 1) + d] = mono[d] * scale;
  }
  return out;
}

// Kernel taps of a point at fractional cell offset f; returns the offset of
// the first tap from the point's cell.
inline int taps(int w, const double* poly, double f, double* kv) {
  const int Q = w + kPolyExtra;
  double u;
  int s;
  if (w % 2 == 0) {
    u = f - 0.5;
    s = -w / 2 + 1;
  } else {
    const bool hi = f > 0.5;
    u = hi ? f - 1.0 : f;
    s = -(w - 1) / 2 + (hi ? 1 : 0);
  }
  for (int m = 0; m < w; ++m) {
    const double* c = poly + size_t(m) * (Q + 1);
    double v = c[Q];
    for (int d = Q - 1; d >= 0; --d) v = v * u + c[d];
    kv[m] = v;
  }
  return s;
}

inline int64_t wrap(int64_t x, int64_t n) {
  x %= n;
  return x < 0 ? x + n : x;
}

}  // namespace

// ---------------------------------------------------------------------------
// FINUFFT API
// ---------------------------------------------------------------------------

struct finufft_plan_s {
  int type = 1, dim = 1, iflag = 1;
  double tol = 1e-6;
  int64_t nm[3] = {1, 1, 1};
  int64_t M = 0, Nt = 0;
  double* X[3] = {nullptr, nullptr, nullptr};
  double* S[3] = {nullptr, nullptr, nullptr};
  // ES set-up
  int w = 7;
  double beta = 16.1;
  int64_t nf[3] = {1, 1, 1};
  std::vector<double> corr[3];
  std::vector<double> poly;    // tap polynomials (tap_polynomials)
  std::vector<int64_t> cell;   // per point, per dim (M*dim)
  std::vector<double> frac;    // per point, per dim
  int tile = 32;
  int64_t nb[3] = {1, 1, 1};
  std::vector<int64_t> tstart;  // tile offsets into torder
  std::vector<int64_t> torder;  // points sorted by tile
};

extern "C" void fresco_shim_set_mode(int mode) { g_mode = mode; }
// Copies the per-stage seconds (setpts, spread, FFT, modes, interpolation)
// into out[0..4]; reset != 0 clears them afterwards.
extern "C" void fresco_shim_profile(double* out, int reset) {
  for (int i = 0; i < kProfN; ++i) {
    if (out) out[i] = g_prof[i];
    if (reset) g_prof[i] = 0.0;
  }
}
extern "C" int fresco_shim_get_mode(void) { return g_mode; }

void finufft_default_opts(finufft_opts* o) {
  if (!o) return;
  o->modeord = 0;
  o->debug = 0;
  o->upsampfac = 2.0;
}

int finufft_makeplan(int type, int dim, int64_t* n_modes, int iflag, int ntrans, double tol, finufft_plan* plan,
                     finufft_opts* o) {
  if (type < 1 || type > 3 || dim < 1 || dim > 3 || ntrans != 1) return 1;
  auto* p = new finufft_plan_s;
  p->type = type;
  p->dim = dim;
  p->iflag = iflag >= 0 ? 1 : -1;
  p->tol = tol;
  if (type != 3)
    for (int a = 0; a < dim; ++a) p->nm[a] = n_modes[a];
  int w = int(std::ceil(-std::log10(tol / 10.0)));
  w = std::max(2, std::min(16, w));
  p->w = w;
  double bw = 2.30;
  if (w == 2) bw = 2.20;
  else if (w == 3) bw = 2.26;
  else if (w == 4) bw = 2.38;
  p->beta = bw * w;
  if (type != 3) {
    for (int a = 0; a < dim; ++a) {
      p->nf[a] = next235even(std::max<int64_t>(2 * p->nm[a], 2 * w));
      p->corr[a] = correction(w, p->beta, p->nf[a], p->nm[a]);
    }
    p->poly = tap_polynomials(w, p->beta);
  }
  *plan = p;
  return 0;
}

namespace {

bool use_exact(const finufft_plan_s* p) {
  if (p->type == 3) return true;
  if (g_mode == 1) return true;
  if (g_mode == 2) return false;
  double nmt = 1.0;
  for (int a = 0; a < p->dim; ++a) nmt *= double(p->nm[a]);
  return double(p->M) * nmt <= 2e7;
}

void es_setpts(finufft_plan_s* p) {
  ProfScope prof(kProfSetpts);
  const int d = p->dim;
  const int64_t M = p->M;
  p->cell.assign(size_t(M) * d, 0);
  p->frac.assign(size_t(M) * d, 0.0);
  p->tile = std::max(p->w, d == 3 ? 16 : 32);
  for (int a = 0; a < 3; ++a) p->nb[a] = a < d ? (p->nf[a] + p->tile - 1) / p->tile : 1;
  const int64_t ntiles = p->nb[0] * p->nb[1] * p->nb[2];
  std::vector<int64_t> tid(M);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; ++j) {
    int64_t b[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
      const double nfd = double(p->nf[a]);
      double u = p->X[a][j] * (nfd / (2.0 * kPi));
      u -= nfd * std::floor(u / nfd);
      double fl = std::floor(u);
      int64_t c = int64_t(fl);
      double f = u - fl;
      if (c >= p->nf[a]) c -= p->nf[a];
      if (c < 0) c += p->nf[a];
      p->cell[size_t(j) * d + a] = c;
      p->frac[size_t(j) * d + a] = f;
      b[a] = c / p->tile;
    }
    tid[j] = b[0] + p->nb[0] * (b[1] + p->nb[1] * b[2]);
  }
  // stable counting sort by tile: per-thread histograms of contiguous point
  // ranges, offsets in (tile, thread) order, then a parallel scatter
  const int nth = omp_get_max_threads();
  std::vector<int64_t> hist(size_t(nth) * ntiles, 0);
  p->tstart.assign(ntiles + 1, 0);
  p->torder.resize(M);
#pragma omp parallel num_threads(nth)
  {
    const int t = omp_get_thread_num(), nt = omp_get_num_threads();
    const int64_t j0 = M * t / nt, j1 = M * (t + 1) / nt;
    int64_t* h = hist.data() + size_t(t) * ntiles;
    for (int64_t j = j0; j < j1; ++j) ++h[tid[j]];
#pragma omp barrier
#pragma omp single
    {
      int64_t run = 0;
      for (int64_t b = 0; b < ntiles; ++b) {
        p->tstart[b] = run;
        for (int u = 0; u < nt; ++u) {
          const int64_t c = hist[size_t(u) * ntiles + b];
          hist[size_t(u) * ntiles + b] = run;
          run += c;
        }
      }
      p->tstart[ntiles] = run;
    }
    for (int64_t j = j0; j < j1; ++j) p->torder[h[tid[j]]++] = j;
  }
}

// Spreads complex strengths c onto the fine grid (row-major, dim 0 fastest).
void es_spread(const finufft_plan_s* p, const cd* c, std::vector<cd>& grid) {
  ProfScope prof(kProfSpread);
  const int d = p->dim, w = p->w;
  const int64_t nf0 = p->nf[0], nf1 = p->nf[1], nf2 = p->nf[2];
  grid.assign(size_t(nf0 * nf1 * nf2), cd(0.0, 0.0));
  auto color = [&](int64_t b, int a) -> int {
    if (p->nb[a] % 2 == 1 && b == p->nb[a] - 1 && p->nb[a] > 1) return 2;
    return int(b % 2);
  };
  for (int col = 0; col < 27; ++col) {
    const int c0 = col % 3, c1 = (col / 3) % 3, c2 = col / 9;
    std::vector<int64_t> tl;
    for (int64_t b2 = 0; b2 < p->nb[2]; ++b2)
      for (int64_t b1 = 0; b1 < p->nb[1]; ++b1)
        for (int64_t b0 = 0; b0 < p->nb[0]; ++b0) {
          if (color(b0, 0) != c0) continue;
          if (d >= 2 && color(b1, 1) != c1) continue;
          if (d < 2 && c1 != 0) continue;
          if (d >= 3 && color(b2, 2) != c2) continue;
          if (d < 3 && c2 != 0) continue;
          tl.push_back(b0 + p->nb[0] * (b1 + p->nb[1] * b2));
        }
    if (tl.empty()) continue;
#pragma omp parallel for schedule(dynamic)
    for (long ti = 0; ti < long(tl.size()); ++ti) {
      const int64_t t = tl[ti];
      double k0[16], k1[16], k2[16];
      int64_t i0[16], i1[16], i2[16];
      for (int64_t q = p->tstart[t]; q < p->tstart[t + 1]; ++q) {
        const int64_t j = p->torder[q];
        const int s0 = taps(w, p->poly.data(), p->frac[size_t(j) * d], k0);
        for (int m = 0; m < w; ++m) i0[m] = wrap(p->cell[size_t(j) * d] + s0 + m, nf0);
        int ny = 1, nz = 1;
        k1[0] = k2[0] = 1.0;
        i1[0] = i2[0] = 0;
        if (d >= 2) {
          const int s1 = taps(w, p->poly.data(), p->frac[size_t(j) * d + 1], k1);
          for (int m = 0; m < w; ++m) i1[m] = wrap(p->cell[size_t(j) * d + 1] + s1 + m, nf1);
          ny = w;
        }
        if (d >= 3) {
          const int s2 = taps(w, p->poly.data(), p->frac[size_t(j) * d + 2], k2);
          for (int m = 0; m < w; ++m) i2[m] = wrap(p->cell[size_t(j) * d + 2] + s2 + m, nf2);
          nz = w;
        }
        const cd cj = c[j];
        for (int mz = 0; mz < nz; ++mz)
          for (int my = 0; my < ny; ++my) {
            const cd v = cj * (k2[mz] * k1[my]);
            cd* row = grid.data() + (i2[mz] * nf1 + i1[my]) * nf0;
            for (int mx = 0; mx < w; ++mx) row[i0[mx]] += v * k0[mx];
          }
      }
    }
  }
}

void es_interp(const finufft_plan_s* p, const std::vector<cd>& grid, cd* c) {
  ProfScope prof(kProfInterp);
  const int d = p->dim, w = p->w;
  const int64_t nf0 = p->nf[0], nf1 = p->nf[1], nf2 = p->nf[2];
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < p->M; ++q) {
    const int64_t j = p->torder[q];
    double k0[16], k1[16], k2[16];
    int64_t i0[16], i1[16], i2[16];
    const int s0 = taps(w, p->poly.data(), p->frac[size_t(j) * d], k0);
    for (int m = 0; m < w; ++m) i0[m] = wrap(p->cell[size_t(j) * d] + s0 + m, nf0);
    int ny = 1, nz = 1;
    k1[0] = k2[0] = 1.0;
    i1[0] = i2[0] = 0;
    if (d >= 2) {
      const int s1 = taps(w, p->poly.data(), p->frac[size_t(j) * d + 1], k1);
      for (int m = 0; m < w; ++m) i1[m] = wrap(p->cell[size_t(j) * d + 1] + s1 + m, nf1);
      ny = w;
    }
    if (d >= 3) {
      const int s2 = taps(w, p->poly.data(), p->frac[size_t(j) * d + 2], k2);
      for (int m = 0; m < w; ++m) i2[m] = wrap(p->cell[size_t(j) * d + 2] + s2 + m, nf2);
      nz = w;
    }
    cd acc(0.0, 0.0);
    for (int mz = 0; mz < nz; ++mz)
      for (int my = 0; my < ny; ++my) {
        const cd* row = grid.data() + (i2[mz] * nf1 + i1[my]) * nf0;
        cd r(0.0, 0.0);
        for (int mx = 0; mx < w; ++mx) r += row[i0[mx]] * k0[mx];
        acc += r * (k2[mz] * k1[my]);
      }
    c[j] = acc;
  }
}

std::vector<int> fft_dims(const finufft_plan_s* p) {
  std::vector<int> dims;
  for (int a = p->dim - 1; a >= 0; --a) dims.push_back(int(p->nf[a]));
  return dims;
}

// mode index -> fine index and correction
void es_type1(const finufft_plan_s* p, const cd* c, cd* f) {
  std::vector<cd> grid;
  es_spread(p, c, grid);
  {
    ProfScope prof(kProfFft);
    fft_nd(grid.data(), fft_dims(p), p->iflag);
  }
  ProfScope prof(kProfModes);
  const int64_t n0 = p->nm[0], n1 = p->nm[1], n2 = p->nm[2];
#pragma omp parallel for schedule(static)
  for (int64_t i2 = 0; i2 < n2; ++i2)
    for (int64_t i1 = 0; i1 < n1; ++i1)
      for (int64_t i0 = 0; i0 < n0; ++i0) {
        const int64_t g0 = wrap(i0 - n0 / 2, p->nf[0]);
        const int64_t g1 = p->dim >= 2 ? wrap(i1 - n1 / 2, p->nf[1]) : 0;
        const int64_t g2 = p->dim >= 3 ? wrap(i2 - n2 / 2, p->nf[2]) : 0;
        double pc = p->corr[0][i0];
        if (p->dim >= 2) pc *= p->corr[1][i1];
        if (p->dim >= 3) pc *= p->corr[2][i2];
        f[i0 + n0 * (i1 + n1 * i2)] = grid[size_t((g2 * p->nf[1] + g1) * p->nf[0] + g0)] / pc;
      }
}

void es_type2(const finufft_plan_s* p, cd* c, const cd* f) {
  std::vector<cd> grid(size_t(p->nf[0] * p->nf[1] * p->nf[2]), cd(0.0, 0.0));
  const int64_t n0 = p->nm[0], n1 = p->nm[1], n2 = p->nm[2];
  {
  ProfScope prof(kProfModes);
#pragma omp parallel for schedule(static)
  for (int64_t i2 = 0; i2 < n2; ++i2)
    for (int64_t i1 = 0; i1 < n1; ++i1)
      for (int64_t i0 = 0; i0 < n0; ++i0) {
        const int64_t g0 = wrap(i0 - n0 / 2, p->nf[0]);
        const int64_t g1 = p->dim >= 2 ? wrap(i1 - n1 / 2, p->nf[1]) : 0;
        const int64_t g2 = p->dim >= 3 ? wrap(i2 - n2 / 2, p->nf[2]) : 0;
        double pc = p->corr[0][i0];
        if (p->dim >= 2) pc *= p->corr[1][i1];
        if (p->dim >= 3) pc *= p->corr[2][i2];
        grid[size_t((g2 * p->nf[1] + g1) * p->nf[0] + g0)] = f[i0 + n0 * (i1 + n1 * i2)] / pc;
      }
  }
  {
    ProfScope prof(kProfFft);
    fft_nd(grid.data(), fft_dims(p), p->iflag);
  }
  es_interp(p, grid, c);
}

// exact direct sums
void phase_table(const double* x, int64_t M, int64_t n, int iflag, std::vector<cd>& E) {
  E.resize(size_t(M * n));
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; ++j)
    for (int64_t i = 0; i < n; ++i) {
      const double a = iflag * double(i - n / 2) * x[j];
      E[size_t(j * n + i)] = cd(std::cos(a), std::sin(a));
    }
}

void exact_type1(const finufft_plan_s* p, const cd* c, cd* f) {
  const int d = p->dim;
  const int64_t n0 = p->nm[0], n1 = p->nm[1], n2 = p->nm[2], M = p->M;
  std::vector<cd> E0, E1, E2;
  phase_table(p->X[0], M, n0, p->iflag, E0);
  if (d >= 2) phase_table(p->X[1], M, n1, p->iflag, E1);
  if (d >= 3) phase_table(p->X[2], M, n2, p->iflag, E2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t i2 = 0; i2 < n2; ++i2)
    for (int64_t i1 = 0; i1 < n1; ++i1) {
      std::vector<cd> row(n0, cd(0.0, 0.0));
      for (int64_t j = 0; j < M; ++j) {
        cd v = c[j];
        if (d >= 2) v *= E1[size_t(j * n1 + i1)];
        if (d >= 3) v *= E2[size_t(j * n2 + i2)];
        const cd* e0 = E0.data() + j * n0;
        for (int64_t i0 = 0; i0 < n0; ++i0) row[i0] += v * e0[i0];
      }
      for (int64_t i0 = 0; i0 < n0; ++i0) f[i0 + n0 * (i1 + n1 * i2)] = row[i0];
    }
}

void exact_type2(const finufft_plan_s* p, cd* c, const cd* f) {
  const int d = p->dim;
  const int64_t n0 = p->nm[0], n1 = p->nm[1], n2 = p->nm[2], M = p->M;
#pragma omp parallel
  {
    std::vector<cd> e0(n0), e1(n1), e2(n2);
#pragma omp for schedule(static)
    for (int64_t j = 0; j < M; ++j) {
      for (int64_t i = 0; i < n0; ++i) {
        const double a = p->iflag * double(i - n0 / 2) * p->X[0][j];
        e0[i] = cd(std::cos(a), std::sin(a));
      }
      for (int64_t i = 0; i < n1; ++i) {
        const double a = d >= 2 ? p->iflag * double(i - n1 / 2) * p->X[1][j] : 0.0;
        e1[i] = cd(std::cos(a), std::sin(a));
      }
      for (int64_t i = 0; i < n2; ++i) {
        const double a = d >= 3 ? p->iflag * double(i - n2 / 2) * p->X[2][j] : 0.0;
        e2[i] = cd(std::cos(a), std::sin(a));
      }
      cd acc(0.0, 0.0);
      for (int64_t i2 = 0; i2 < n2; ++i2)
        for (int64_t i1 = 0; i1 < n1; ++i1) {
          cd r(0.0, 0.0);
          const cd* fr = f + n0 * (i1 + n1 * i2);
          for (int64_t i0 = 0; i0 < n0; ++i0) r += fr[i0] * e0[i0];
          acc += r * e1[i1] * e2[i2];
        }
      c[j] = acc;
    }
  }
}

void exact_type3(const finufft_plan_s* p, const cd* c, cd* f) {
  const int d = p->dim;
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < p->Nt; ++k) {
    cd acc(0.0, 0.0);
    for (int64_t j = 0; j < p->M; ++j) {
      double ph = p->S[0][k] * p->X[0][j];
      if (d >= 2) ph += p->S[1][k] * p->X[1][j];
      if (d >= 3) ph += p->S[2][k] * p->X[2][j];
      ph *= p->iflag;
      acc += c[j] * cd(std::cos(ph), std::sin(ph));
    }
    f[k] = acc;
  }
}

}  // namespace

int finufft_setpts(finufft_plan plan, int64_t M, double* x, double* y, double* z, int64_t N, double* s, double* t,
                   double* u) {
  if (!plan) return 1;
  plan->M = M;
  plan->X[0] = x;
  plan->X[1] = y;
  plan->X[2] = z;
  if (plan->type == 3) {
    plan->Nt = N;
    plan->S[0] = s;
    plan->S[1] = t;
    plan->S[2] = u;
  }
  if (!use_exact(plan)) es_setpts(plan);
  return 0;
}

int finufft_execute(finufft_plan plan, std::complex<double>* weights, std::complex<double>* result) {
  if (!plan) return 1;
  if (plan->type == 3) {
    exact_type3(plan, weights, result);
  } else if (use_exact(plan)) {
    if (plan->type == 1) exact_type1(plan, weights, result);
    else exact_type2(plan, weights, result);
  } else {
    if (plan->cell.size() != size_t(plan->M * plan->dim)) es_setpts(plan);
    if (plan->type == 1) es_type1(plan, weights, result);
    else es_type2(plan, weights, result);
  }
  return 0;
}

int finufft_destroy(finufft_plan plan) {
  delete plan;
  return 0;
}

// ---------------------------------------------------------------------------
// FFTW API
// ---------------------------------------------------------------------------

struct fftw_plan_s {
  std::vector<int> dims;
  fftw_complex* in = nullptr;
  fftw_complex* out = nullptr;
  int sign = -1;
};

void* fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
  (void)flags;
  auto* p = new fftw_plan_s;
  p->dims.assign(n, n + rank);
  p->in = in;
  p->out = out;
  p->sign = sign;
  return p;
}

void fftw_execute(const fftw_plan p) {
  size_t total = 1;
  for (int d : p->dims) total *= size_t(d);
  cd* out = reinterpret_cast<cd*>(p->out);
  if (p->out != p->in) std::memcpy(out, p->in, total * sizeof(cd));
  fft_nd(out, p->dims, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
