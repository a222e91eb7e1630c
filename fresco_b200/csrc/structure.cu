// Structure factor and pair correlation of a point pattern on the device: the
// counterpart of fresco.utils.export_structure (fresco/utils/utils.py:16-52)
// and radial_profile (utils.py:138-152).
//
// Reference semantics: coordinates r / L, shifted by -1/2 when any exceeds 1,
// times 2 pi; weights 1, or the point volumes (pi r^2, 4/3 pi r^3) scaled to
// sum to N; rho = type-1 NUFFT on Nk^d modes (tolerance tol), S = |rho|^2 / N
// in centred order (index k + Nk/2, dimension 0 first); g = real part of the
// centred inverse DFT of (S - 1) in FFT order, times prod(L) / N (numpy's
// ifftn normalisation cancels the Nk^d factor); radial profiles average S and
// g over integer radii int(sqrt(sum_a (i_a - Nk/2)^2)) = 0..Nk/2.
//
// B200 form: one FP64 bin sort, ES spreading into the fine grid, a D2Z FFT,
// deconvolution of the Nk^d modes, one Z2Z inverse FFT of Nk^d (cuFFT), and
// block-local shared-memory bins for the radial profiles.  It runs once per
// pattern (after a minimisation), so it allocates its buffers per call.
#include <cmath>
#include <cufft.h>
#include <string>
#include <vector>

#include "es.cuh"
#include "nufft.cuh"
#include "potential.cuh"

namespace fb {

namespace {

constexpr double kPi = 3.14159265358979323846;

// S(k) from the R2C output (sign -1) of the spread grid: rho(k) (iflag +1) is
// conj(B(k)) for k_x >= 0 and B(-k) otherwise, deconvolved by the ES factors.
template <int D>
__global__ void structure_modes_kernel(const double2* __restrict__ bhat, int nh0, Geom g, int Nk, int kmin,
                                       const double* __restrict__ corr0, const double* __restrict__ corr1,
                                       const double* __restrict__ corr2, double invN, double* sk,
                                       double2* __restrict__ fft_in) {
  int64_t total = Nk;
  for (int a = 1; a < D; ++a) total *= Nk;
  const int nf1 = g.nf[1], nf2 = g.nf[2];
  for (int64_t m = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; m < total;
       m += int64_t(gridDim.x) * blockDim.x) {
    // centred output index m = ((i0 Nk) + i1) Nk + i2, dimension 0 slowest
    int idx[3] = {0, 0, 0};
    int64_t r = m;
    for (int a = D - 1; a >= 0; --a) {
      idx[a] = int(r % Nk);
      r /= Nk;
    }
    const int kx = idx[0] + kmin;
    const int ky = D >= 2 ? idx[1] + kmin : 0;
    const int kz = D >= 3 ? idx[2] + kmin : 0;
    double p = corr0[idx[0]];
    if (D >= 2) p *= corr1[idx[1]];
    if (D >= 3) p *= corr2[idx[2]];
    int64_t bi;
    if (kx >= 0) {
      const int yy = ky < 0 ? ky + nf1 : ky, zz = kz < 0 ? kz + nf2 : kz;
      bi = kx + int64_t(nh0) * (yy + int64_t(nf1) * zz);
    } else {
      const int yy = ky > 0 ? nf1 - ky : -ky, zz = kz > 0 ? nf2 - kz : -kz;
      bi = -kx + int64_t(nh0) * (yy + int64_t(nf1) * zz);
    }
    const double2 b = bhat[bi];
    const double s = (b.x * b.x + b.y * b.y) / (p * p) * invN;
    sk[m] = s;
    // the inverse-FFT input: S - 1 in FFT order (index k mod Nk per dimension)
    int64_t fi = 0;
    for (int a = 0; a < D; ++a) {
      const int k = a == 0 ? kx : (a == 1 ? ky : kz);
      fi = fi * Nk + (k < 0 ? k + Nk : k);
    }
    fft_in[fi] = make_double2(s - 1.0, 0.0);
  }
}

// g in centred order: real part of the unnormalised inverse DFT, shifted so
// that index Nk/2 holds lag 0, times prod(L) / N.
template <int D>
__global__ void structure_pair_kernel(const double2* __restrict__ fft_out, int Nk, double scale, double* gr) {
  int64_t total = Nk;
  for (int a = 1; a < D; ++a) total *= Nk;
  const int c = Nk / 2;
  for (int64_t m = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; m < total;
       m += int64_t(gridDim.x) * blockDim.x) {
    int64_t r = m, src = 0, mul = 1;
    for (int a = D - 1; a >= 0; --a) {
      const int i = int(r % Nk);
      r /= Nk;
      src += int64_t((i - c + Nk) % Nk) * mul;  // fftshift: out[i] = in[(i - Nk/2) mod Nk]
      mul *= Nk;
    }
    gr[m] = fft_out[src].x * scale;
  }
}

// Sums of a centred Nk^d array over integer radii 0..R+1 (R = Nk/2; radii
// beyond R land in bin R+1), block-local in shared memory.
template <int D>
__global__ void radial_sum_kernel(const double* __restrict__ data, int Nk, double* sums, unsigned long long* counts) {
  extern __shared__ unsigned char smem_raw[];
  const int R = Nk / 2, nb = R + 2;
  double* s_sum = reinterpret_cast<double*>(smem_raw);
  unsigned* s_cnt = reinterpret_cast<unsigned*>(s_sum + nb);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    s_sum[i] = 0.0;
    s_cnt[i] = 0u;
  }
  __syncthreads();
  int64_t total = Nk;
  for (int a = 1; a < D; ++a) total *= Nk;
  for (int64_t m = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; m < total;
       m += int64_t(gridDim.x) * blockDim.x) {
    int64_t r = m, d2 = 0;
    for (int a = D - 1; a >= 0; --a) {
      const int64_t t = int(r % Nk) - R;
      r /= Nk;
      d2 += t * t;
    }
    int bin = int(sqrt(double(d2)));  // truncation, as numpy's astype(int)
    if (bin > R) bin = R + 1;
    atomicAdd(&s_sum[bin], data[m]);
    atomicAdd(&s_cnt[bin], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    if (s_cnt[i]) {
      atomicAdd(&sums[i], s_sum[i]);
      atomicAdd(&counts[i], (unsigned long long)s_cnt[i]);
    }
  }
}

template <int D>
void export_structure_d(const double* x, int64_t N, const double* L, int Nk, const double* radii, double tol,
                        double* sk_out, double* gr_out, double* s_radial, double* g_radial) {
  if (N <= 0) throw InvalidArgument("export_structure needs at least one point");
  if (Nk < 2) throw InvalidArgument("export_structure needs Nk >= 2");
  int64_t total = Nk;
  for (int a = 1; a < D; ++a) total *= Nk;
  // coordinates: r / L, shifted by -1/2 when any exceeds 1 (utils.py:20-24);
  // the 2 pi scaling is the sort's kind-1 map x = p 2 pi / L with L = 1
  std::vector<double> xs(x, x + N * D);
  double mx = -INFINITY;
  for (int64_t j = 0; j < N; ++j)
    for (int a = 0; a < D; ++a) {
      xs[j * D + a] /= L[a];
      mx = std::max(mx, xs[j * D + a]);
    }
  if (mx > 1.0)
    for (double& v : xs) v -= 0.5;
  // weights (utils.py:26-35): area factor once, then scaled to sum to N
  std::vector<double> c(size_t(N), 1.0);
  bool uniform = true;
  if (radii) {
    double sum = 0.0;
    for (int64_t j = 0; j < N; ++j) {
      c[j] = D == 2 ? kPi * radii[j] * radii[j] : (D == 3 ? 4.0 / 3.0 * kPi * radii[j] * radii[j] * radii[j] : 1.0);
      sum += c[j];
    }
    for (auto& v : c) v *= double(N) / sum;
    for (auto& v : c) uniform &= v == c[0];
  }
  const ESParams es = es_params(tol, 16);
  const std::vector<double> poly = es_poly_coefficients(es, es.w);
  int64_t nf[3] = {1, 1, 1};
  for (int a = 0; a < D; ++a) nf[a] = fine_grid_size(Nk, es.w);
  int tile[3] = {D == 1 ? 1024 : (D == 2 ? kTile2D : 8), D == 2 ? kTile2D : 8, 8};
  const Geom g = make_geom(D, nf, es.w, tile);
  cudaStream_t s = nullptr;
  DevBuf<double> dx, dc, grid, corr[3], sk, gr, rsum;
  DevBuf<unsigned long long> rcnt;
  DevBuf<double2> bhat, fin, fout;
  DevBuf<unsigned char> recs;
  DevBuf<int> status;
  SortBufs sb;
  dx.alloc(N * D);
  FB_CUDA(cudaMemcpy(dx.p, xs.data(), sizeof(double) * N * D, cudaMemcpyHostToDevice));
  if (!uniform) {
    dc.alloc(N);
    FB_CUDA(cudaMemcpy(dc.p, c.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  }
  status.alloc(2);
  FB_CUDA(cudaMemset(status.p, 0, 2 * sizeof(int)));
  alloc_sort(sb, N, g);
  recs.alloc(N * int64_t(rec_bytes(D, false)));
  MapParams mp;
  mp.kind = 1;
  mp.stride = D;
  for (int a = 0; a < D; ++a) mp.L[a] = 1.0;
  bin_sort<double>(dx.p, N, mp, g, sb, recs.p, status.p, s);
  grid.alloc(g.G());
  FB_CUDA(cudaMemset(grid.p, 0, grid.bytes()));
  spread_real<double>(recs.p, dc.p, uniform ? c[0] : 1.0, sb, g, poly, grid.p, s);
  const int nh0 = g.nf[0] / 2 + 1;
  bhat.alloc(int64_t(nh0) * g.nf[1] * g.nf[2]);
  int dims[3];
  for (int a = 0; a < D; ++a) dims[a] = g.nf[D - 1 - a];
  cufftHandle plan = 0;
  FB_CUFFT(cufftPlanMany(&plan, D, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1));
  FB_CUFFT(cufftExecD2Z(plan, grid.p, reinterpret_cast<cufftDoubleComplex*>(bhat.p)));
  cufftDestroy(plan);
  const int kmin = -(Nk / 2);
  for (int a = 0; a < 3; ++a) {
    const std::vector<double> pc = es_correction(es, a < D ? g.nf[a] : g.nf[0], kmin, Nk);
    corr[a].alloc(Nk);
    FB_CUDA(cudaMemcpy(corr[a].p, pc.data(), sizeof(double) * Nk, cudaMemcpyHostToDevice));
  }
  sk.alloc(total);
  fin.alloc(total);
  fout.alloc(total);
  const int blocks = int(std::min<int64_t>(ceil_div(total, 256), int64_t(sm_count()) * 8));
  structure_modes_kernel<D><<<blocks, 256, 0, s>>>(bhat.p, nh0, g, Nk, kmin, corr[0].p, corr[1].p, corr[2].p,
                                                   1.0 / double(N), sk.p, fin.p);
  FB_LAUNCH_CHECK();
  int kd[3] = {Nk, Nk, Nk};
  FB_CUFFT(cufftPlanMany(&plan, D, kd, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2Z, 1));
  FB_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(fin.p),
                        reinterpret_cast<cufftDoubleComplex*>(fout.p), CUFFT_INVERSE));
  cufftDestroy(plan);
  double vol = 1.0;
  for (int a = 0; a < D; ++a) vol *= L[a];
  gr.alloc(total);
  structure_pair_kernel<D><<<blocks, 256, 0, s>>>(fout.p, Nk, vol / double(N), gr.p);
  FB_LAUNCH_CHECK();
  const int R = Nk / 2, nb = R + 2;
  rsum.alloc(2 * nb);
  rcnt.alloc(2 * nb);
  FB_CUDA(cudaMemset(rsum.p, 0, rsum.bytes()));
  FB_CUDA(cudaMemset(rcnt.p, 0, rcnt.bytes()));
  const size_t smem = size_t(nb) * (sizeof(double) + sizeof(unsigned));
  auto rk = radial_sum_kernel<D>;
  if (smem > 48 * 1024) ensure_dynamic_smem(rk, smem);
  rk<<<blocks, 256, smem, s>>>(sk.p, Nk, rsum.p, rcnt.p);
  rk<<<blocks, 256, smem, s>>>(gr.p, Nk, rsum.p + nb, rcnt.p + nb);
  FB_LAUNCH_CHECK();
  FB_CUDA(cudaMemcpy(sk_out, sk.p, sizeof(double) * total, cudaMemcpyDeviceToHost));
  FB_CUDA(cudaMemcpy(gr_out, gr.p, sizeof(double) * total, cudaMemcpyDeviceToHost));
  std::vector<double> hs(2 * nb);
  std::vector<unsigned long long> hc(2 * nb);
  FB_CUDA(cudaMemcpy(hs.data(), rsum.p, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost));
  FB_CUDA(cudaMemcpy(hc.data(), rcnt.p, sizeof(unsigned long long) * 2 * nb, cudaMemcpyDeviceToHost));
  for (int i = 0; i <= R; ++i) {
    s_radial[i] = hc[i] ? hs[i] / double(hc[i]) : NAN;
    g_radial[i] = hc[nb + i] ? hs[nb + i] / double(hc[nb + i]) : NAN;
  }
  int hst[2];
  FB_CUDA(cudaMemcpy(hst, status.p, sizeof(hst), cudaMemcpyDeviceToHost));
  if (hst[1] & STATUS_NONFINITE_INPUT) throw InvalidArgument("export_structure: non-finite coordinate");
}

}  // namespace

void export_structure(const double* x, int64_t n_points, int ndim, const double* L, int Nk, const double* radii,
                      double tol, double* sk_out, double* gr_out, double* s_radial, double* g_radial) {
  if (ndim == 2) return export_structure_d<2>(x, n_points, L, Nk, radii, tol, sk_out, gr_out, s_radial, g_radial);
  if (ndim == 3) return export_structure_d<3>(x, n_points, L, Nk, radii, tol, sk_out, gr_out, s_radial, g_radial);
  throw InvalidArgument("export_structure: dimension must be 2 or 3 (utils.py:36-49)");
}

}  // namespace fb
