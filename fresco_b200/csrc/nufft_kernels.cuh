// Kernel bodies and host launchers for nufft.cuh, instantiated once per
// precision in nufft_f32.cu / nufft_f64.cu.
#pragma once

#include <algorithm>

#include "nufft.cuh"

namespace fb {

namespace {
constexpr double kPi = 3.14159265358979323846;
}

__device__ __forceinline__ int wrap_index(int x, int n) {
  if (x < 0) x += n;
  else if (x >= n) x -= n;
  if (x < 0 || x >= n) {
    x %= n;
    if (x < 0) x += n;
  }
  return x;
}

// Maps coordinate a of point j to (cell, fraction).  Returns false for a
// non-finite coordinate (then cell = 0, fraction = 0 so all later accesses
// stay in bounds).
__device__ __forceinline__ bool map_coord(const double* __restrict__ pts, int64_t j, const MapParams& mp,
                                          int nf, int a, int& c, double& f) {
  const double p = pts[j * mp.stride + a];
  const double L = mp.L[a];
  double x;
  if (mp.kind == 0) {
    // same operation order as source/fresco/nuwu.hpp:219
    x = (p - round(p / L)) * 2 * kPi / L;
  } else {
    x = p * 2 * kPi / L;  // uwnu.hpp:245
  }
  double u = x * (double(nf) / (2.0 * kPi));
  if (!isfinite(u)) {
    c = 0;
    f = 0.0;
    return false;
  }
  u -= double(nf) * floor(u / double(nf));
  double fl = floor(u);
  int ci = int(fl);
  f = u - fl;
  if (ci >= nf) ci -= nf;
  if (ci < 0) ci += nf;
  if (ci < 0 || ci >= nf) { ci = 0; f = 0.0; }
  c = ci;
  return true;
}

template <int D>
__global__ void __launch_bounds__(kSortThreads) bin_count_kernel(const double* __restrict__ pts, int64_t N,
                                                                 MapParams mp, Geom g, int* bin_count,
                                                                 uint32_t* rank, int* status) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    int c[3] = {0, 0, 0};
    bool ok = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      double f;
      ok &= map_coord(pts, j, mp, g.nf[a], a, c[a], f);
    }
    if (!ok) raise_status(status, STATUS_NONFINITE_INPUT);
    const int bin = c[0] / g.tile[0] + g.nb[0] * (c[1] / g.tile[1] + g.nb[1] * (c[2] / g.tile[2]));
    rank[j] = uint32_t(atomicAdd(&bin_count[bin], 1));
  }
}

// One block: bin offsets (exclusive scan of counts) and the subproblem table
// (each bin cut into chunks of at most kMaxSub points).
static __global__ void __launch_bounds__(1024) build_subproblems_kernel(int nbins, const int* __restrict__ bin_count,
                                                                 int* bin_start, int* sub_bin, int* sub_start,
                                                                 int* sub_count, int* num_sub, int max_sub) {
  __shared__ int s_pts[1024];
  __shared__ int s_sub[1024];
  const int tid = threadIdx.x;
  const int per = (nbins + blockDim.x - 1) / blockDim.x;
  const int b0 = min(nbins, tid * per), b1 = min(nbins, b0 + per);
  int np = 0, ns = 0;
  for (int b = b0; b < b1; ++b) {
    const int c = bin_count[b];
    np += c;
    ns += (c + kMaxSub - 1) / kMaxSub;
  }
  s_pts[tid] = np;
  s_sub[tid] = ns;
  __syncthreads();
  for (int off = 1; off < int(blockDim.x); off <<= 1) {
    const int a = tid >= off ? s_pts[tid - off] : 0;
    const int b = tid >= off ? s_sub[tid - off] : 0;
    __syncthreads();
    s_pts[tid] += a;
    s_sub[tid] += b;
    __syncthreads();
  }
  int pbase = s_pts[tid] - np, sbase = s_sub[tid] - ns;
  for (int b = b0; b < b1; ++b) {
    const int c = bin_count[b];
    bin_start[b] = pbase;
    const int nsub = (c + kMaxSub - 1) / kMaxSub;
    for (int s = 0; s < nsub; ++s) {
      if (sbase < max_sub) {
        sub_bin[sbase] = b;
        sub_start[sbase] = pbase + s * kMaxSub;
        sub_count[sbase] = min(kMaxSub, c - s * kMaxSub);
      }
      ++sbase;
    }
    pbase += c;
  }
  if (tid == int(blockDim.x) - 1) *num_sub = min(s_sub[tid], max_sub);
}

template <int D, typename T>
__global__ void __launch_bounds__(kSortThreads) scatter_kernel(const double* __restrict__ pts, int64_t N,
                                                               MapParams mp, Geom g,
                                                               const double* __restrict__ weights,
                                                               double uniform_weight,
                                                               const uint32_t* __restrict__ rank,
                                                               const int* __restrict__ bin_start,
                                                               SortedPts<T> out) {
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    int c[3] = {0, 0, 0};
    double f[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < D; ++a) map_coord(pts, j, mp, g.nf[a], a, c[a], f[a]);
    const int bin = c[0] / g.tile[0] + g.nb[0] * (c[1] / g.tile[1] + g.nb[1] * (c[2] / g.tile[2]));
    const int64_t dest = int64_t(bin_start[bin]) + rank[j];
    out.cell[dest] = pack_cell(D, c[0], c[1], c[2]);
#pragma unroll
    for (int a = 0; a < D; ++a) out.frac[a][dest] = T(f[a]);
    out.cw[dest] = T(weights ? weights[j] : uniform_weight);
    out.idx[dest] = uint32_t(j);
  }
}

template <typename T>
__device__ __forceinline__ void atomic_add_cplx(cplx_t<T>* p, T re, T im);
template <>
__device__ __forceinline__ void atomic_add_cplx<float>(float2* p, float re, float im) {
  atomicAdd(p, make_float2(re, im));  // vector atomic (sm_90+, global memory)
}
template <>
__device__ __forceinline__ void atomic_add_cplx<double>(double2* p, double re, double im) {
  atomicAdd(&p->x, re);
  atomicAdd(&p->y, im);
}

// One block per subproblem: spread its points into a shared tile (tile +
// halo of w/2 cells on each side), then add the tile to the fine grid with
// global atomics (periodic wrap).
template <int D, int W, typename T, bool CPLX>
__global__ void __launch_bounds__(256) spread_kernel(SortedPts<T> sp, const int* __restrict__ sub_bin,
                                                     const int* __restrict__ sub_start,
                                                     const int* __restrict__ sub_count,
                                                     const int* __restrict__ num_sub, Geom g, T beta,
                                                     const cplx_t<T>* __restrict__ strengths, T* grid_real,
                                                     cplx_t<T>* grid_cplx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  constexpr int NC = CPLX ? 2 : 1;
  const int tw0 = g.tw[0], tw1 = g.tw[1];
  const int tsize = int(g.tile_cells());
  for (int i = threadIdx.x; i < tsize * NC; i += blockDim.x) tile[i] = T(0);
  __syncthreads();

  const int bin = sub_bin[sub];
  const int start = sub_start[sub], cnt = sub_count[sub];
  const int bx = bin % g.nb[0];
  const int brem = bin / g.nb[0];
  const int by = brem % g.nb[1];
  const int bz = brem / g.nb[1];
  const int org0 = bx * g.tile[0], org1 = by * g.tile[1], org2 = bz * g.tile[2];
  constexpr int PAD = W / 2;

  for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
    const int j = start + p;
    int c0, c1, c2;
    unpack_cell(D, sp.cell[j], c0, c1, c2);
    T sr, si = T(0);
    if (CPLX) {
      const cplx_t<T> v = strengths[sp.idx[j]];
      sr = v.x;
      si = v.y;
    } else {
      sr = sp.cw[j];
    }
    T k0[W];
    const int l0 = c0 - org0 + es_taps<W, T>(sp.frac[0][j], beta, k0) + PAD;
    if (D == 1) {
#pragma unroll
      for (int m0 = 0; m0 < W; ++m0) {
        if (CPLX) {
          atomicAdd(&tile[2 * (l0 + m0)], sr * k0[m0]);
          atomicAdd(&tile[2 * (l0 + m0) + 1], si * k0[m0]);
        } else {
          atomicAdd(&tile[l0 + m0], sr * k0[m0]);
        }
      }
      continue;
    }
    T k1[W];
    const int l1 = c1 - org1 + es_taps<W, T>(sp.frac[1][j], beta, k1) + PAD;
    int nz = 1;
    T k2[W];
    int l2 = 0;
    if (D == 3) {
      l2 = c2 - org2 + es_taps<W, T>(sp.frac[2][j], beta, k2) + PAD;
      nz = W;
    }
    for (int m2 = 0; m2 < nz; ++m2) {
      const T wz = (D == 3) ? k2[m2] : T(1);
#pragma unroll
      for (int m1 = 0; m1 < W; ++m1) {
        const T wyr = sr * wz * k1[m1];
        const T wyi = si * wz * k1[m1];
        const int row = ((l2 + m2) * tw1 + (l1 + m1)) * tw0 + l0;
#pragma unroll
        for (int m0 = 0; m0 < W; ++m0) {
          if (CPLX) {
            atomicAdd(&tile[2 * (row + m0)], wyr * k0[m0]);
            atomicAdd(&tile[2 * (row + m0) + 1], wyi * k0[m0]);
          } else {
            atomicAdd(&tile[row + m0], wyr * k0[m0]);
          }
        }
      }
    }
  }
  __syncthreads();

  const int o0 = org0 - PAD;
  const int o1 = (D >= 2) ? org1 - PAD : 0;
  const int o2 = (D >= 3) ? org2 - PAD : 0;
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  for (int i = threadIdx.x; i < tsize; i += blockDim.x) {
    const int i0 = i % tw0;
    const int r = i / tw0;
    const int i1 = r % tw1;
    const int i2 = r / tw1;
    const int a0 = wrap_index(o0 + i0, nf0);
    const int a1 = (D >= 2) ? wrap_index(o1 + i1, nf1) : 0;
    const int a2 = (D >= 3) ? wrap_index(o2 + i2, nf2) : 0;
    const int64_t gi = (int64_t(a2) * nf1 + a1) * nf0 + a0;
    if (CPLX) {
      const T re = tile[2 * i], im = tile[2 * i + 1];
      if (re != T(0) || im != T(0)) atomic_add_cplx<T>(grid_cplx + gi, re, im);
    } else {
      const T v = tile[i];
      if (v != T(0)) atomicAdd(grid_real + gi, v);
    }
  }
}

// Thread per sorted point: gathers W^D fine-grid values directly from HBM/L2
// (the bin-sorted order gives neighbouring threads overlapping footprints).
template <int D, int W, typename T, int NF>
__global__ void __launch_bounds__(256) interp_kernel(SortedPts<T> sp, int64_t N, Geom g, T beta,
                                                     const cplx_t<T>* __restrict__ fields, int64_t G,
                                                     int mode, double* grad, double2* out2, int accumulate,
                                                     const int* __restrict__ status) {
  const bool bad = status != nullptr && ((*status) & STATUS_NONFINITE_INPUT);
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    int c0, c1, c2;
    unpack_cell(D, sp.cell[j], c0, c1, c2);
    T k0[W], k1[W], k2[W];
    int ix[W];
    const int s0 = es_taps<W, T>(sp.frac[0][j], beta, k0);
#pragma unroll
    for (int m = 0; m < W; ++m) ix[m] = wrap_index(c0 + s0 + m, nf0);
    int s1 = 0, s2 = 0;
    if (D >= 2) s1 = es_taps<W, T>(sp.frac[1][j], beta, k1);
    if (D >= 3) s2 = es_taps<W, T>(sp.frac[2][j], beta, k2);
    T v0r = 0, v0i = 0, v1r = 0, v1i = 0;
    const int nz = (D == 3) ? W : 1;
    const int ny = (D >= 2) ? W : 1;
    for (int m2 = 0; m2 < nz; ++m2) {
      const int iz = (D == 3) ? wrap_index(c2 + s2 + m2, nf2) : 0;
      const T wz = (D == 3) ? k2[m2] : T(1);
#pragma unroll
      for (int m1 = 0; m1 < ny; ++m1) {
        const int iy = (D >= 2) ? wrap_index(c1 + s1 + m1, nf1) : 0;
        const T wy = (D >= 2) ? wz * k1[m1] : T(1);
        const cplx_t<T>* row = fields + (int64_t(iz) * nf1 + iy) * nf0;
        T rr = 0, ri = 0, qr = 0, qi = 0;
#pragma unroll
        for (int m0 = 0; m0 < W; ++m0) {
          const cplx_t<T> a = __ldg(row + ix[m0]);
          rr += a.x * k0[m0];
          ri += a.y * k0[m0];
          if (NF == 2) {
            const cplx_t<T> b = __ldg(row + G + ix[m0]);
            qr += b.x * k0[m0];
            qi += b.y * k0[m0];
          }
        }
        v0r += wy * rr;
        v0i += wy * ri;
        if (NF == 2) {
          v1r += wy * qr;
          v1i += wy * qi;
        }
      }
    }
    const uint32_t o = sp.idx[j];
    if (mode == INTERP_GRAD) {
      const double cw = double(sp.cw[j]);
      double gv[3] = {cw * double(v0r), cw * double(v0i), cw * double(v1r)};
#pragma unroll
      for (int a = 0; a < D; ++a) {
        double val = bad ? __longlong_as_double(0x7ff8000000000000ULL) : gv[a];
        double* dst = grad + int64_t(o) * D + a;
        *dst = accumulate ? *dst + val : val;
      }
    } else {
      out2[o] = make_double2(double(v0r), double(v0i));
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

inline int point_grid(int64_t n, int per_sm = 8) {
  const int64_t want = std::max<int64_t>(1, ceil_div(n, 256));
  return int(std::min<int64_t>(want, int64_t(sm_count()) * per_sm));
}

template <typename T>
void bin_sort(const double* pts, int64_t N, const MapParams& mp, const Geom& g, const double* weights,
              double uniform_weight, SortBufs& sb, SortedStore<T>& out, int* status, cudaStream_t s) {
  const int nbins = int(g.nbins());
  FB_CUDA(cudaMemsetAsync(sb.bin_count.p, 0, sizeof(int) * nbins, s));
  if (N > 0) {
    const int grid = point_grid(N);
    switch (g.D) {
      case 1: bin_count_kernel<1><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, sb.bin_count.p, sb.rank.p, status); break;
      case 2: bin_count_kernel<2><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, sb.bin_count.p, sb.rank.p, status); break;
      default: bin_count_kernel<3><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, sb.bin_count.p, sb.rank.p, status); break;
    }
    FB_LAUNCH_CHECK();
  }
  build_subproblems_kernel<<<1, 1024, 0, s>>>(nbins, sb.bin_count.p, sb.bin_start.p, sb.sub_bin.p, sb.sub_start.p,
                                              sb.sub_count.p, sb.num_sub.p, int(sb.max_sub));
  FB_LAUNCH_CHECK();
  if (N > 0) {
    const int grid = point_grid(N);
    SortedPts<T> v = out.view();
    switch (g.D) {
      case 1: scatter_kernel<1, T><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, weights, uniform_weight, sb.rank.p, sb.bin_start.p, v); break;
      case 2: scatter_kernel<2, T><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, weights, uniform_weight, sb.rank.p, sb.bin_start.p, v); break;
      default: scatter_kernel<3, T><<<grid, kSortThreads, 0, s>>>(pts, N, mp, g, weights, uniform_weight, sb.rank.p, sb.bin_start.p, v); break;
    }
    FB_LAUNCH_CHECK();
  }
}

template <int D, int W, typename T, bool CPLX>
void launch_spread_w(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta,
                     const cplx_t<T>* strengths, T* grid_real, cplx_t<T>* grid_cplx, cudaStream_t s) {
  const size_t smem = size_t(g.tile_cells()) * sizeof(T) * (CPLX ? 2 : 1);
  auto kern = spread_kernel<D, W, T, CPLX>;
  if (smem > 48 * 1024) FB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kern<<<unsigned(sb.max_sub), 256, smem, s>>>(sp, sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                T(beta), strengths, grid_real, grid_cplx);
  FB_LAUNCH_CHECK();
}

template <int D, int W, typename T>
void launch_interp_w(const SortedPts<T>& sp, int64_t N, const Geom& g, double beta, const cplx_t<T>* fields,
                     int nfields, int mode, double* grad, double2* out2, int acc, const int* status,
                     cudaStream_t s) {
  if (N <= 0) return;
  const int grid = point_grid(N, 16);
  if (nfields == 2) {
    interp_kernel<D, W, T, 2><<<grid, 256, 0, s>>>(sp, N, g, T(beta), fields, g.G(), mode, grad, out2, acc, status);
  } else {
    interp_kernel<D, W, T, 1><<<grid, 256, 0, s>>>(sp, N, g, T(beta), fields, g.G(), mode, grad, out2, acc, status);
  }
  FB_LAUNCH_CHECK();
}

#define FB_FOR_W(T, X)                                                                    \
  switch (g.w) {                                                                          \
    case 2: X(2); break;                                                                  \
    case 3: X(3); break;                                                                  \
    case 4: X(4); break;                                                                  \
    case 5: X(5); break;                                                                  \
    case 6: X(6); break;                                                                  \
    case 7: X(7); break;                                                                  \
    case 8: X(8); break;                                                                  \
    case 9: X(9); break;                                                                  \
    case 10: X(10); break;                                                                \
    default:                                                                              \
      if (sizeof(T) == 8) {                                                               \
        switch (g.w) {                                                                    \
          case 11: X(11); break;                                                          \
          case 12: X(12); break;                                                          \
          case 13: X(13); break;                                                          \
          case 14: X(14); break;                                                          \
          case 15: X(15); break;                                                          \
          case 16: X(16); break;                                                          \
          default: throw InvalidArgument("unsupported kernel width");                     \
        }                                                                                 \
      } else {                                                                            \
        throw InvalidArgument("unsupported kernel width for FP32");                       \
      }                                                                                   \
  }

template <typename T, int D, bool CPLX>
void spread_dispatch(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta,
                     const cplx_t<T>* strengths, T* grid_real, cplx_t<T>* grid_cplx, cudaStream_t s) {
#define FB_SPREAD_W(WW)                                                                       \
  launch_spread_w<D, (sizeof(T) == 4 && WW > 10) ? 10 : WW, T, CPLX>(sp, sb, g, beta, strengths, \
                                                                      grid_real, grid_cplx, s)
  FB_FOR_W(T, FB_SPREAD_W)
#undef FB_SPREAD_W
}

template <typename T, int D>
void interp_dispatch(const SortedPts<T>& sp, int64_t N, const Geom& g, double beta, const cplx_t<T>* fields,
                     int nfields, int mode, double* grad, double2* out2, int acc, const int* status,
                     cudaStream_t s) {
#define FB_INTERP_W(WW)                                                                           \
  launch_interp_w<D, (sizeof(T) == 4 && WW > 10) ? 10 : WW, T>(sp, N, g, beta, fields, nfields, mode, \
                                                                grad, out2, acc, status, s)
  FB_FOR_W(T, FB_INTERP_W)
#undef FB_INTERP_W
}

template <typename T>
void spread_real(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta, T* grid,
                 cudaStream_t s) {
  switch (g.D) {
    case 1: spread_dispatch<T, 1, false>(sp, sb, g, beta, nullptr, grid, nullptr, s); break;
    case 2: spread_dispatch<T, 2, false>(sp, sb, g, beta, nullptr, grid, nullptr, s); break;
    default: spread_dispatch<T, 3, false>(sp, sb, g, beta, nullptr, grid, nullptr, s); break;
  }
}

template <typename T>
void spread_cplx(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta,
                 const cplx_t<T>* strengths, cplx_t<T>* grid, cudaStream_t s) {
  switch (g.D) {
    case 1: spread_dispatch<T, 1, true>(sp, sb, g, beta, strengths, nullptr, grid, s); break;
    case 2: spread_dispatch<T, 2, true>(sp, sb, g, beta, strengths, nullptr, grid, s); break;
    default: spread_dispatch<T, 3, true>(sp, sb, g, beta, strengths, nullptr, grid, s); break;
  }
}

template <typename T>
void interp(const SortedPts<T>& sp, int64_t N, const Geom& g, double beta, const cplx_t<T>* fields, int nfields,
            int mode, double* grad, double2* out2, int accumulate, const int* status, cudaStream_t s) {
  switch (g.D) {
    case 1: interp_dispatch<T, 1>(sp, N, g, beta, fields, nfields, mode, grad, out2, accumulate, status, s); break;
    case 2: interp_dispatch<T, 2>(sp, N, g, beta, fields, nfields, mode, grad, out2, accumulate, status, s); break;
    default: interp_dispatch<T, 3>(sp, N, g, beta, fields, nfields, mode, grad, out2, accumulate, status, s); break;
  }
}

#define FB_INSTANTIATE_NUFFT(T)                                                                           \
  template void bin_sort<T>(const double*, int64_t, const MapParams&, const Geom&, const double*, double,    \
                            SortBufs&, SortedStore<T>&, int*, cudaStream_t);                                 \
  template void spread_real<T>(const SortedPts<T>&, const SortBufs&, const Geom&, double, T*, cudaStream_t); \
  template void spread_cplx<T>(const SortedPts<T>&, const SortBufs&, const Geom&, double, const cplx_t<T>*, \
                               cplx_t<T>*, cudaStream_t);                                                    \
  template void interp<T>(const SortedPts<T>&, int64_t, const Geom&, double, const cplx_t<T>*, int, int,     \
                          double*, double2*, int, const int*, cudaStream_t);

}  // namespace fb
