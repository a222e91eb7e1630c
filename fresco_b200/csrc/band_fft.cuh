// Pruned 2D transforms of the NUwU loss ("band" transforms) on N x N fine
// grids, N a power of two in 512..8192, for one pattern or a batch of
// patterns of the same grid.
#pragma once

#include "fft_block.cuh"
#include "nuwu_modes.cuh"

namespace fb {

// ---------------------------------------------------------------------------
// 2D band transforms.  The loss only reads modes with |k_x| <= Kx and
// |k_y| <= Ky (the active band), so the 2D transforms are split into passes
// that touch only what the band needs (all forward, sign -1, as cuFFT; fine
// grid N x N with N a power of two, RegFft<T, N>):
//   rows_r2c:   per transform two real fine-grid rows (z = a + i b), keeps
//               k_x = 0..Kx of each row                        -> band1[Kx+1][N]
//   band_modes: one k_x >= 0 per block: column FFT of band1, the mode pass for
//               +k_x and -k_x (deconvolve, S, d, phi, packed field h), and the
//               column FFTs of the two h columns              -> band2[N][2Kx+1]
//   rows_c2c:   per transform one band2 row placed at k_x mod N -> the full
//               type-2 output row.
// Each block runs two transforms (threadIdx.y = 0, 1) of N / 16 threads with
// their own named barriers.  Batched: blockIdx.y selects the pattern, whose
// buffers the BandBatch descriptor locates (one pattern: all strides 0).
// ---------------------------------------------------------------------------

template <typename T>
struct BandBatch {
  T* grid;                   // real fine grids (read and zeroed by the row transform)
  int64_t grid_stride;
  cplx_t<T>* band1;          // [Kx+1][N] per pattern
  int64_t band1_stride;
  cplx_t<T>* band2;          // [N][2Kx+1] per pattern
  int64_t band2_stride;
  cplx_t<T>* out;            // type-2 output grids
  int64_t out_stride;
  const ModeCoef* coef;      // [2Kx+1][2Ky+1] per pattern
  int64_t coef_stride;
  const double* invN;        // 1/N per pattern, or null: invN_all
  double invN_all;
  double* energy;            // energy[idx], idx = index ? index[p] : 0
  const int* status;         // status[idx]: the pattern's evaluation status word
  const int* index;
};

// The rows are zeroed once read: the next evaluation spreads into a clean grid
// without a separate memset.  FP32 up to N = 2048 keeps four blocks per SM
// (64 registers, no spills); larger transforms are left to the compiler.
template <typename T, int N>
__global__ void __launch_bounds__(N / 8, (sizeof(T) == 4 && N <= 2048) ? 4 : 1) band_rows_r2c_kernel(T* __restrict__ grid, int64_t grid_stride,
                                                               const cplx_t<T>* __restrict__ tw, int KB,
                                                               cplx_t<T>* __restrict__ band1, int64_t band1_stride) {
  grid += blockIdx.y * grid_stride;
  band1 += blockIdx.y * band1_stride;
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* buf = reinterpret_cast<cplx_t<T>*>(smem_raw) + threadIdx.y * fft_padded(N);
  const int t = threadIdx.x;
  const int64_t y = 2 * (2 * int64_t(blockIdx.x) + threadIdx.y);
  T* ra = grid + y * N;
  T* rb = ra + N;
  cplx_t<T> v[F::E];
#pragma unroll
  for (int j = 0; j < F::E; ++j) {
    v[j].x = ra[t + j * (N / F::E)];
    v[j].y = rb[t + j * (N / F::E)];
  }
#pragma unroll
  for (int j = 0; j < F::E; ++j) {
    ra[t + j * (N / F::E)] = T(0);
    rb[t + j * (N / F::E)] = T(0);
  }
  F::run(v, buf, tw, t, 1 + threadIdx.y);
  // A(k) = (Z(k) + conj Z(-k)) / 2, B(k) = (Z(k) - conj Z(-k)) / (2i)
  for (int k = t; k < KB; k += F::TPB) {
    const cplx_t<T> zk = buf[fpad(k)], zm = buf[fpad(k == 0 ? 0 : N - k)];
    cplx_t<T> A, B;
    A.x = T(0.5) * (zk.x + zm.x);
    A.y = T(0.5) * (zk.y - zm.y);
    B.x = T(0.5) * (zk.y + zm.y);
    B.y = T(0.5) * (zm.x - zk.x);
    band1[int64_t(k) * N + y] = A;
    band1[int64_t(k) * N + y + 1] = B;
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(N / 8) band_modes_kernel(const BandBatch<T> bb, const cplx_t<T>* __restrict__ tw,
                                                           int Kx, int Ky, int K, const double* __restrict__ corr0,
                                                           const double* __restrict__ corr1, int want_grad) {
  const cplx_t<T>* __restrict__ band1 = bb.band1 + blockIdx.y * bb.band1_stride;
  cplx_t<T>* __restrict__ band2 = bb.band2 + blockIdx.y * bb.band2_stride;
  const ModeCoef* __restrict__ coef = bb.coef + blockIdx.y * bb.coef_stride;
  const double invN = bb.invN ? bb.invN[blockIdx.y] : bb.invN_all;
  const int eidx = bb.index ? bb.index[blockIdx.y] : 0;
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* col = reinterpret_cast<cplx_t<T>*>(smem_raw);
  cplx_t<T>* h1 = col + fft_padded(N);  // field column +k_x
  cplx_t<T>* h2 = h1 + fft_padded(N);   // field column -k_x
  const int t = threadIdx.x, grp = threadIdx.y;
  const int tid = grp * F::TPB + t, nthr = 2 * F::TPB;
  const int kx = blockIdx.x;
  const int NB2 = 2 * Kx + 1, NY = 2 * Ky + 1;
  if (want_grad)
    for (int i = tid; i < N; i += nthr) {
      h1[fpad(i)] = cplx_t<T>{T(0), T(0)};
      h2[fpad(i)] = cplx_t<T>{T(0), T(0)};
    }
  if (grp == 0) {  // B(k_x, k_y) for all k_y (mod N)
    cplx_t<T> v[F::E];
#pragma unroll
    for (int j = 0; j < F::E; ++j) v[j] = band1[int64_t(kx) * N + t + j * (N / F::E)];
    F::run(v, col, tw, t, 1);
  }
  __syncthreads();
  double phi = 0.0;
  for (int i = tid; i < NY; i += nthr) {
    const int ky = i - Ky;
    const double py = corr1[ky + K];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      if (side == 1 && kx == 0) break;
      const int kxs = side == 0 ? kx : -kx;
      const ModeCoef c = coef[int64_t(kxs + Kx) * NY + i];
      if (c.w2 == 0.0 && c.A == 0.0 && c.B == 0.0) continue;  // outside the active set
      const double p = corr0[kxs + K] * py;
      // rho(k) = conj(B(k)) for k_x >= 0; rho(-|k_x|, k_y) = B(|k_x|, -k_y)
      const int yy = side == 0 ? (ky < 0 ? ky + N : ky) : (ky > 0 ? N - ky : -ky);
      const cplx_t<T> bv = col[fpad(yy)];
      const double rr = double(bv.x) / p;
      const double ri = (side == 0 ? -double(bv.y) : double(bv.y)) / p;
      const double q = (rr * rr + ri * ri) * invN;
      const double dq = q - c.s0;
      phi += c.w2 * dq * dq;
      if (want_grad) {
        const double a = (c.A * q - c.B) * (2.0 * invN) / p;  // includes the type-2 pre-correction 1/p
        const double fr = rr * a, fi = ri * a;
        cplx_t<T> h;  // F (k_y - i k_x)
        h.x = T(fr * ky + fi * kxs);
        h.y = T(fi * ky - fr * kxs);
        (side == 0 ? h1 : h2)[fpad(ky < 0 ? ky + N : ky)] = h;
      }
    }
  }
  block_sum_atomic(phi, bb.energy + eidx);  // ends with __syncthreads
  if (blockIdx.x == 0 && tid == 0 && bb.status != nullptr && (bb.status[eidx] & STATUS_NONFINITE_INPUT))
    atomicAdd(bb.energy + eidx, __longlong_as_double(0x7ff8000000000000ULL));
  if (!want_grad) return;
  if (grp == 1 && kx == 0) return;  // k_x = 0 has one column
  cplx_t<T>* h = grp == 0 ? h1 : h2;
  cplx_t<T> v[F::E];
#pragma unroll
  for (int j = 0; j < F::E; ++j) v[j] = h[fpad(t + j * (N / F::E))];
  group_sync(1 + grp, F::TPB);  // every input is in registers before h is reused
  F::run(v, h, tw, t, 1 + grp);
  const int c = grp == 0 ? Kx + kx : Kx - kx;
  for (int y = t; y < N; y += F::TPB) band2[int64_t(y) * NB2 + c] = h[fpad(y)];
}

template <typename T, int N>
__global__ void __launch_bounds__(N / 8, sizeof(T) == 4 ? 3 : 2) band_rows_c2c_kernel(const BandBatch<T> bb, int Kx,
                                                                                  const cplx_t<T>* __restrict__ tw) {
  const cplx_t<T>* __restrict__ band2 = bb.band2 + blockIdx.y * bb.band2_stride;
  cplx_t<T>* __restrict__ out = bb.out + blockIdx.y * bb.out_stride;
  using F = RegFft<T, N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* buf = reinterpret_cast<cplx_t<T>*>(smem_raw) + threadIdx.y * fft_padded(N);
  const int t = threadIdx.x;
  const int64_t y = 2 * int64_t(blockIdx.x) + threadIdx.y;
  const int NB2 = 2 * Kx + 1;
  const cplx_t<T>* row = band2 + y * NB2;
  cplx_t<T> v[F::E];
#pragma unroll
  for (int j = 0; j < F::E; ++j) {
    const int x = t + j * (N / F::E);  // k_x = x for x <= Kx, x - N for x >= N - Kx, else no mode
    v[j] = x <= Kx ? row[Kx + x] : (x >= N - Kx ? row[Kx + x - N] : cplx_t<T>{T(0), T(0)});
  }
  F::run(v, buf, tw, t, 1 + threadIdx.y);
  cplx_t<T>* o = out + y * N;
  for (int x = t; x < N; x += F::TPB) o[x] = buf[fpad(x)];
}

}  // namespace fb
