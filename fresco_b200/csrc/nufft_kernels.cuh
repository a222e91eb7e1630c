// Kernel bodies and host launchers for nufft.cuh, instantiated once per
// precision in nufft_f32.cu / nufft_f64.cu.
#pragma once

#include <algorithm>
#include <vector>

#include "nufft.cuh"
#include "scan.cuh"

namespace fb {

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr int kSortThreads = 512;
}  // namespace

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
__device__ __forceinline__ bool map_coord(const double* __restrict__ pts, int64_t j, const MapParams& mp, int nf, int a,
                                          int& c, double& f) {
  // Every operation is an explicitly rounded intrinsic: the counting and the
  // scattering pass of the sort evaluate this map separately and must agree
  // bit for bit, whatever the compiler's contraction choices in each kernel.
  const double p = pts[j * mp.stride + a];
  const double L = mp.L[a];
  double x;
  if (mp.kind == 0) {
    // same operation order as source/fresco/nuwu.hpp:219
    x = __ddiv_rn(__dmul_rn(__dmul_rn(__dsub_rn(p, round(__ddiv_rn(p, L))), 2.0), kPi), L);
  } else {
    x = __ddiv_rn(__dmul_rn(__dmul_rn(p, 2.0), kPi), L);  // uwnu.hpp:245
  }
  double u = __dmul_rn(x, double(nf) / (2.0 * kPi));
  if (!isfinite(u)) {
    c = 0;
    f = 0.0;
    return false;
  }
  u = __dsub_rn(u, __dmul_rn(double(nf), floor(__ddiv_rn(u, double(nf)))));
  const double fl = floor(u);
  int ci = int(fl);
  f = __dsub_rn(u, fl);
  if (ci >= nf) ci -= nf;
  if (ci < 0) ci += nf;
  if (ci < 0 || ci >= nf) {
    ci = 0;
    f = 0.0;
  }
  c = ci;
  return true;
}

template <int D>
__device__ __forceinline__ int point_bin(const double* __restrict__ pts, int64_t j, const MapParams& mp, const Geom& g,
                                         int (&c)[3], double (&f)[3], bool& ok) {
  ok = true;
#pragma unroll
  for (int a = 0; a < D; ++a) ok &= map_coord(pts, j, mp, g.nf[a], a, c[a], f[a]);
  return c[0] / g.tile[0] + g.nb[0] * (c[1] / g.tile[1] + g.nb[1] * (c[2] / g.tile[2]));
}

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of
// 32, at most 1024); returns the prefix and writes the block total.
__device__ __forceinline__ int block_exclusive_scan(int v, int* total, int* s_warp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int w = lane < nw ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < nw) s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const int before = wid > 0 ? s_warp[wid - 1] : 0;
  *total = s_warp[nw - 1];
  __syncthreads();
  return before + inc - v;
}

// Sort pass 1: block-local histogram of the block's chunk of points in
// shared memory, then one global atomic per non-empty bin reserves the
// block's segment inside that bin (blk_off, block-major).
template <int D>
__global__ void __launch_bounds__(kSortThreads) sort_count_kernel(const double* __restrict__ pts, int64_t N,
                                                                  int64_t chunk, MapParams mp, Geom g, int* bin_total,
                                                                  int* blk_off, int* status) {
  extern __shared__ int sh_hist[];
  const int nbins = int(g.nbins());
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  const int64_t j0 = int64_t(blockIdx.x) * chunk, j1 = min(N, j0 + chunk);
  bool bad = false;
  for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    int c[3] = {0, 0, 0};
    double f[3];
    bool ok;
    const int bin = point_bin<D>(pts, j, mp, g, c, f, ok);
    bad |= !ok;
    atomicAdd(&sh_hist[bin], 1);
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
  __syncthreads();
  int* my_off = blk_off + int64_t(blockIdx.x) * nbins;
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
    const int cnt = sh_hist[i];
    if (cnt) my_off[i] = atomicAdd(&bin_total[i], cnt);
  }
}

// Sort pass 2 (one block of 1024 threads): bin starts (exclusive scan of the
// bin totals), the subproblem table (each bin cut into chunks of at most
// kMaxSub points), and bin_total cleared for the next sort.
static __global__ void __launch_bounds__(1024) sort_plan_kernel(int nbins, int* bin_total, int* bin_start,
                                                                int* sub_bin, int* sub_start, int* sub_count,
                                                                int* num_sub, int max_sub) {
  __shared__ int s_warp[32];
  const int per = (nbins + int(blockDim.x) - 1) / int(blockDim.x);
  const int b0 = min(nbins, int(threadIdx.x) * per), b1 = min(nbins, b0 + per);
  int npts = 0, nsub = 0;
  for (int b = b0; b < b1; ++b) {
    const int c = bin_total[b];
    npts += c;
    nsub += (c + kMaxSub - 1) / kMaxSub;
  }
  int tot_pts, tot_sub;
  int start = block_exclusive_scan(npts, &tot_pts, s_warp);
  int sbase = block_exclusive_scan(nsub, &tot_sub, s_warp);
  for (int b = b0; b < b1; ++b) {
    const int c = bin_total[b];
    bin_start[b] = start;
    bin_total[b] = 0;
    for (int q = 0; q * kMaxSub < c; ++q) {
      if (sbase < max_sub) {
        sub_bin[sbase] = b;
        sub_start[sbase] = start + q * kMaxSub;
        sub_count[sbase] = min(kMaxSub, c - q * kMaxSub);
      }
      ++sbase;
    }
    start += c;
  }
  if (threadIdx.x == 0) {
    bin_start[nbins] = tot_pts;
    *num_sub = min(tot_sub, max_sub);
  }
}

// Sort pass 3: each block hands out the slots of its segments again with
// shared-memory cursors (the counts are those of pass 1, so every slot is
// written exactly once) and stores the packed records.
template <int D, typename T>
__global__ void __launch_bounds__(kSortThreads) sort_scatter_kernel(const double* __restrict__ pts, int64_t N,
                                                                    int64_t chunk, MapParams mp, Geom g,
                                                                    const int* __restrict__ bin_start,
                                                                    const int* __restrict__ blk_off, Rec<D, T>* out,
                                                                    int* status) {
  extern __shared__ int sh_cur[];
  const int nbins = int(g.nbins());
  const int* my_off = blk_off + int64_t(blockIdx.x) * nbins;
  // bins this block has no points in hold stale offsets that are never used
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh_cur[i] = bin_start[i] + my_off[i];
  __syncthreads();
  const int64_t j0 = int64_t(blockIdx.x) * chunk, j1 = min(N, j0 + chunk);
  for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    int c[3] = {0, 0, 0};
    double f[3] = {0, 0, 0};
    bool ok;
    const int bin = point_bin<D>(pts, j, mp, g, c, f, ok);
    const int dest = atomicAdd(&sh_cur[bin], 1);
    if (dest < 0 || int64_t(dest) >= N) {
      raise_status(status, STATUS_OVERFLOW);
      continue;
    }
    Rec<D, T> r;
    r.cell = pack_cell(D, c[0], c[1], c[2]);
#pragma unroll
    for (int a = 0; a < D; ++a) r.f[a] = T(f[a]);
    r.idx = uint32_t(j);
    out[dest] = r;
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

// Adds a shared tile (origin org - pad per used dimension) to the fine grid
// with global atomics and periodic wrap.
template <int D, typename T, bool CPLX>
__device__ __forceinline__ void flush_tile(const T* tile, const Geom& g, int org0, int org1, int org2, int pad,
                                           T* grid_real, cplx_t<T>* grid_cplx) {
  const int tw0 = g.tw[0], tw1 = g.tw[1];
  const int tsize = int(g.tile_cells());
  const int o0 = org0 - pad;
  const int o1 = (D >= 2) ? org1 - pad : 0;
  const int o2 = (D >= 3) ? org2 - pad : 0;
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

// ---------------------------------------------------------------------------
// 2D spreading without shared-memory atomics.
//
// The 64 x 64-cell tile is cut into sub-blocks of SB x SB cells (SB = 8 for
// w <= 8, 16 for w <= 16).  A point's w x w footprint only reaches the
// neighbouring sub-blocks, so sub-blocks whose (a, b) indices have the same
// parities never touch the same cell: the tile is spread in four phases, one
// per parity class.  Within a phase a warp handles GPW sub-blocks at once,
// one point from each, with one lane per footprint row; a lane adds its row
// with plain shared-memory read-modify-writes.  Points of one sub-block are
// taken one after another by the same lane group (__syncwarp between them),
// so no two lanes ever update the same cell concurrently.
// ---------------------------------------------------------------------------

template <int W>
struct Phased2D {
  static constexpr int SB = W <= 8 ? 8 : 16;
  static constexpr int NSB = kTile2D / SB;       // sub-blocks per tile edge
  static constexpr int GROUP = W <= 8 ? 8 : 16;  // lanes per point (one per footprint row)
  static constexpr int GPW = 32 / GROUP;         // points per warp step
  static constexpr int PER_PHASE = (NSB / 2) * (NSB / 2);
  static constexpr int NWARP = PER_PHASE / GPW;
  static constexpr int THREADS = 32 * NWARP;
};

template <int W, typename T, bool CPLX>
__global__ void __launch_bounds__(Phased2D<W>::THREADS) spread2d_phased_kernel(
    const Rec<2, T>* __restrict__ recs, const T* __restrict__ weights, T uniform,
    const cplx_t<T>* __restrict__ strengths, const int* __restrict__ sub_bin, const int* __restrict__ sub_start,
    const int* __restrict__ sub_count, const int* __restrict__ num_sub, Geom g, const EsPoly<W, T> poly, T* grid_real,
    cplx_t<T>* grid_cplx) {
  using P = Phased2D<W>;
  constexpr int NC = CPLX ? 2 : 1;
  constexpr int PAD = W / 2;
  constexpr int TW = kTile2D + W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Rec<2, T>* srec = reinterpret_cast<Rec<2, T>*>(smem_raw);  // subproblem's records, grouped by sub-block
  T* tile = reinterpret_cast<T*>(srec + kMaxSub);
  int* code = reinterpret_cast<int*>(tile + TW * TW * NC);
  int* sb_count = code + kMaxSub;
  int* sb_start = sb_count + P::NSB * P::NSB;

  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  const int bin = sub_bin[sub];
  const int start = sub_start[sub], cnt = sub_count[sub];
  const int org0 = (bin % g.nb[0]) * kTile2D, org1 = (bin / g.nb[0]) * kTile2D;

  for (int i = threadIdx.x; i < TW * TW * NC; i += blockDim.x) tile[i] = T(0);
  for (int i = threadIdx.x; i < P::NSB * P::NSB; i += blockDim.x) sb_count[i] = 0;
  __syncthreads();
  // group the subproblem's points by sub-block (integer shared atomics)
  for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
    int c0, c1, c2;
    unpack_cell(2, recs[start + p].cell, c0, c1, c2);
    const int sbi = ((c0 - org0) / P::SB) + P::NSB * ((c1 - org1) / P::SB);
    code[p] = (sbi << 16) | atomicAdd(&sb_count[sbi], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int i = 0; i < P::NSB * P::NSB; ++i) {
      sb_start[i] = acc;
      acc += sb_count[i];
    }
  }
  __syncthreads();
  for (int p = threadIdx.x; p < cnt; p += blockDim.x) srec[sb_start[code[p] >> 16] + (code[p] & 0xffff)] = recs[start + p];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / P::GROUP, row = lane % P::GROUP;
  const int q = warp * P::GPW + grp;  // this lane group's slot within a phase
  const int qa = q % (P::NSB / 2), qb = q / (P::NSB / 2);
  // each lane evaluates one tap (its footprint row) for every point: keep that
  // tap's polynomial in registers (idle lanes take a valid row)
  constexpr int Q = EsPolyDeg<W>::Q;
  T cr[Q + 1];
  {
    const int trow = row < W ? row : W - 1;
#pragma unroll
    for (int m = 0; m < W; ++m)
      if (m == trow) {
#pragma unroll
        for (int d = 0; d <= Q; ++d) cr[d] = poly.c[m][d];
      }
  }
  for (int phase = 0; phase < 4; ++phase) {
    const int sbi = (2 * qa + (phase & 1)) + P::NSB * (2 * qb + (phase >> 1));
    const int my_n = sb_count[sbi], my_base = sb_start[sbi];
    int n_max = my_n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_max = max(n_max, __shfl_xor_sync(0xffffffffu, n_max, o));
    // software pipeline: the taps of point it+1 are formed before point it is added
    T kx = T(0), wr = T(0), wi = T(0);
    int base = 0;
    bool active = false;
#define FB_PHASED_LOAD(IT, KX, WR, WI, BASE, ACT)                                      \
  {                                                                                    \
    ACT = (IT) < my_n;                                                                 \
    KX = T(0);                                                                         \
    WR = T(0);                                                                         \
    WI = T(0);                                                                         \
    BASE = 0;                                                                          \
    if (ACT) {                                                                         \
      const Rec<2, T> r_ = srec[my_base + (IT)];                                       \
      int c0_, c1_, c2_;                                                               \
      unpack_cell(2, r_.cell, c0_, c1_, c2_);                                          \
      T u0_, u1_;                                                                      \
      const int s0_ = es_start<W, T>(r_.f[0], u0_);                                    \
      const int s1_ = es_start<W, T>(r_.f[1], u1_);                                    \
      T a_ = cr[Q], b_ = cr[Q];                                                        \
      _Pragma("unroll") for (int d_ = Q - 1; d_ >= 0; --d_) {                          \
        a_ = fma(a_, u0_, cr[d_]);                                                     \
        b_ = fma(b_, u1_, cr[d_]);                                                     \
      }                                                                                \
      KX = a_;                                                                         \
      T sr_, si_ = T(0);                                                               \
      if (CPLX) {                                                                      \
        const cplx_t<T> v_ = strengths[r_.idx];                                        \
        sr_ = v_.x;                                                                    \
        si_ = v_.y;                                                                    \
      } else {                                                                         \
        sr_ = weights ? weights[r_.idx] : uniform;                                     \
      }                                                                                \
      WR = sr_ * b_;                                                                   \
      WI = si_ * b_;                                                                   \
      BASE = ((c1_ - org1 + s1_ + PAD + row) * TW + (c0_ - org0 + s0_ + PAD)) * NC;    \
    }                                                                                  \
  }
    FB_PHASED_LOAD(0, kx, wr, wi, base, active)
    for (int it = 0; it < n_max; ++it) {
      T nkx, nwr, nwi;
      int nbase;
      bool nact;
      FB_PHASED_LOAD(it + 1, nkx, nwr, nwi, nbase, nact)
      T* rowp = tile + base;
#pragma unroll
      for (int m = 0; m < W; ++m) {
        const T km = __shfl_sync(0xffffffffu, kx, grp * P::GROUP + m);
        if (active && row < W) {
          if (CPLX) {
            rowp[2 * m] += wr * km;
            rowp[2 * m + 1] += wi * km;
          } else {
            rowp[m] += wr * km;
          }
        }
      }
      __syncwarp();
      kx = nkx;
      wr = nwr;
      wi = nwi;
      base = nbase;
      active = nact;
    }
#undef FB_PHASED_LOAD
    __syncthreads();
  }
  Geom gt = g;
  gt.tw[0] = TW;
  gt.tw[1] = TW;
  gt.tw[2] = 1;
  flush_tile<2, T, CPLX>(tile, gt, org0, org1, 0, PAD, grid_real, grid_cplx);
}

// Generic spreading (1D, 3D): one thread per point, shared-memory atomics.
template <int D, int W, typename T, bool CPLX>
__global__ void __launch_bounds__(256) spread_kernel(const Rec<D, T>* __restrict__ recs, const T* __restrict__ weights,
                                                     T uniform, const cplx_t<T>* __restrict__ strengths,
                                                     const int* __restrict__ sub_bin, const int* __restrict__ sub_start,
                                                     const int* __restrict__ sub_count, const int* __restrict__ num_sub,
                                                     Geom g, const EsPoly<W, T> poly, T* grid_real,
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
    const Rec<D, T> rec = recs[start + p];
    int c0, c1, c2;
    unpack_cell(D, rec.cell, c0, c1, c2);
    T sr, si = T(0);
    if (CPLX) {
      const cplx_t<T> v = strengths[rec.idx];
      sr = v.x;
      si = v.y;
    } else {
      sr = weights ? weights[rec.idx] : uniform;
    }
    T k0[W];
    const int l0 = c0 - org0 + es_taps<W, T>(rec.f[0], poly, k0) + PAD;
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
    const int l1 = c1 - org1 + es_taps<W, T>(rec.f[D >= 2 ? 1 : 0], poly, k1) + PAD;
    int nz = 1;
    T k2[W];
    int l2 = 0;
    if (D == 3) {
      l2 = c2 - org2 + es_taps<W, T>(rec.f[D >= 3 ? 2 : 0], poly, k2) + PAD;
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
  flush_tile<D, T, CPLX>(tile, g, org0, org1, org2, PAD, grid_real, grid_cplx);
}

// Epilogue shared by the interpolation kernels.
template <int D, typename T>
__device__ __forceinline__ void interp_store(int mode, uint32_t o, T wgt, T v0r, T v0i, T v1r, bool bad, double* grad,
                                             double2* out2, int accumulate, const GradScale& gs) {
  if (mode == INTERP_GRAD) {
    const double cw = double(wgt);
    const double gv[3] = {cw * double(v0r) * gs.s[0], cw * double(v0i) * gs.s[1], cw * double(v1r) * gs.s[2]};
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const double val = bad ? __longlong_as_double(0x7ff8000000000000ULL) : gv[a];
      double* dst = grad + int64_t(o) * D + a;
      *dst = accumulate ? *dst + val : val;
    }
  } else {
    out2[o] = make_double2(double(v0r), double(v0i));
  }
}

// 2D interpolation: one block per subproblem stages the tile (+ halo) of the
// field in shared memory, then one thread per point sums its w x w taps.
template <int W, typename T>
__global__ void __launch_bounds__(256) interp2d_tile_kernel(
    const Rec<2, T>* __restrict__ recs, const T* __restrict__ weights, T uniform, const int* __restrict__ sub_bin,
    const int* __restrict__ sub_start, const int* __restrict__ sub_count, const int* __restrict__ num_sub, Geom g,
    const EsPoly<W, T> poly, const cplx_t<T>* __restrict__ field, int mode, double* grad, double2* out2, int accumulate,
    const int* __restrict__ status, const GradScale gs) {
  constexpr int PAD = W / 2;
  constexpr int TW = kTile2D + W;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx_t<T>* tile = reinterpret_cast<cplx_t<T>*>(smem_raw);
  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  const bool bad = status != nullptr && ((*status) & STATUS_NONFINITE_INPUT);
  const int bin = sub_bin[sub];
  const int start = sub_start[sub], cnt = sub_count[sub];
  const int org0 = (bin % g.nb[0]) * kTile2D, org1 = (bin / g.nb[0]) * kTile2D;
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  for (int i = threadIdx.x; i < TW * TW; i += blockDim.x) {
    const int i0 = i % TW, i1 = i / TW;
    const int a0 = wrap_index(org0 - PAD + i0, nf0), a1 = wrap_index(org1 - PAD + i1, nf1);
    tile[i] = field[int64_t(a1) * nf0 + a0];
  }
  __syncthreads();
  for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
    const Rec<2, T> r = recs[start + p];
    int c0, c1, c2;
    unpack_cell(2, r.cell, c0, c1, c2);
    T k0[W], k1[W];
    const int s0 = es_taps<W, T>(r.f[0], poly, k0);
    const int s1 = es_taps<W, T>(r.f[1], poly, k1);
    const int l0 = c0 - org0 + s0 + PAD, l1 = c1 - org1 + s1 + PAD;
    T vr = 0, vi = 0;
#pragma unroll
    for (int m1 = 0; m1 < W; ++m1) {
      const cplx_t<T>* rowp = tile + (l1 + m1) * TW + l0;
      T rr = 0, ri = 0;
#pragma unroll
      for (int m0 = 0; m0 < W; ++m0) {
        const cplx_t<T> a = rowp[m0];
        rr += a.x * k0[m0];
        ri += a.y * k0[m0];
      }
      vr += k1[m1] * rr;
      vi += k1[m1] * ri;
    }
    const T wgt = (mode == INTERP_GRAD) ? (weights ? weights[r.idx] : uniform) : T(1);
    interp_store<2, T>(mode, r.idx, wgt, vr, vi, T(0), bad, grad, out2, accumulate, gs);
  }
}

// Generic interpolation (1D, 3D): thread per sorted point, taps gathered
// directly from HBM/L2 (neighbouring threads share footprints).
template <int D, int W, typename T, int NF>
__global__ void __launch_bounds__(256) interp_kernel(const Rec<D, T>* __restrict__ recs, int64_t N,
                                                     const T* __restrict__ weights, T uniform, Geom g,
                                                     const EsPoly<W, T> poly, const cplx_t<T>* __restrict__ fields,
                                                     int64_t G, int mode,
                                                     double* grad, double2* out2, int accumulate,
                                                     const int* __restrict__ status, const GradScale gs) {
  const bool bad = status != nullptr && ((*status) & STATUS_NONFINITE_INPUT);
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < N; j += int64_t(gridDim.x) * blockDim.x) {
    const Rec<D, T> rec = recs[j];
    int c0, c1, c2;
    unpack_cell(D, rec.cell, c0, c1, c2);
    T k0[W], k1[W], k2[W];
    int ix[W];
    const int s0 = es_taps<W, T>(rec.f[0], poly, k0);
#pragma unroll
    for (int m = 0; m < W; ++m) ix[m] = wrap_index(c0 + s0 + m, nf0);
    int s1 = 0, s2 = 0;
    if (D >= 2) s1 = es_taps<W, T>(rec.f[D >= 2 ? 1 : 0], poly, k1);
    if (D >= 3) s2 = es_taps<W, T>(rec.f[D >= 3 ? 2 : 0], poly, k2);
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
        const cplx_t<T>* rowp = fields + (int64_t(iz) * nf1 + iy) * nf0;
        T rr = 0, ri = 0, qr = 0, qi = 0;
#pragma unroll
        for (int m0 = 0; m0 < W; ++m0) {
          const cplx_t<T> a = __ldg(rowp + ix[m0]);
          rr += a.x * k0[m0];
          ri += a.y * k0[m0];
          if (NF == 2) {
            const cplx_t<T> b = __ldg(rowp + G + ix[m0]);
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
    const T wgt = (mode == INTERP_GRAD) ? (weights ? weights[rec.idx] : uniform) : T(1);
    interp_store<D, T>(mode, rec.idx, wgt, v0r, v0i, v1r, bad, grad, out2, accumulate, gs);
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

inline int point_grid(int64_t n, int per_sm = 8) {
  const int64_t want = std::max<int64_t>(1, ceil_div(n, 256));
  return int(std::min<int64_t>(want, int64_t(sm_count()) * per_sm));
}

template <int D, typename T>
void bin_sort_d(const double* pts, int64_t N, const MapParams& mp, const Geom& g, SortBufs& sb, void* recs, int* status,
                cudaStream_t s) {
  const int nbins = int(g.nbins());
  const size_t smem = sizeof(int) * size_t(nbins);
  auto k1 = sort_count_kernel<D>;
  auto k3 = sort_scatter_kernel<D, T>;
  if (smem > 48 * 1024) {
    FB_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    FB_CUDA(cudaFuncSetAttribute(k3, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  }
  if (N > 0) {
    k1<<<sb.NB, kSortThreads, smem, s>>>(pts, N, sb.chunk, mp, g, sb.bin_total.p, sb.blk_off.p, status);
    FB_LAUNCH_CHECK();
  }
  sort_plan_kernel<<<1, 1024, 0, s>>>(nbins, sb.bin_total.p, sb.bin_start.p, sb.sub_bin.p, sb.sub_start.p,
                                      sb.sub_count.p, sb.num_sub.p, int(sb.max_sub));
  FB_LAUNCH_CHECK();
  if (N > 0) {
    k3<<<sb.NB, kSortThreads, smem, s>>>(pts, N, sb.chunk, mp, g, sb.bin_start.p, sb.blk_off.p,
                                         static_cast<Rec<D, T>*>(recs), status);
    FB_LAUNCH_CHECK();
  }
}

template <typename T>
void bin_sort(const double* pts, int64_t N, const MapParams& mp, const Geom& g, SortBufs& sb, void* recs, int* status,
              cudaStream_t s) {
  switch (g.D) {
    case 1: bin_sort_d<1, T>(pts, N, mp, g, sb, recs, status, s); break;
    case 2: bin_sort_d<2, T>(pts, N, mp, g, sb, recs, status, s); break;
    default: bin_sort_d<3, T>(pts, N, mp, g, sb, recs, status, s); break;
  }
}

template <int W, typename T, bool CPLX>
void launch_spread2d(const void* recs, const T* weights, T uniform, const cplx_t<T>* strengths, const SortBufs& sb,
                     const Geom& g, const std::vector<double>& poly, T* grid_real, cplx_t<T>* grid_cplx,
                     cudaStream_t s) {
  using P = Phased2D<W>;
  constexpr int TW = kTile2D + W;
  const size_t smem = sizeof(Rec<2, T>) * kMaxSub + sizeof(T) * TW * TW * (CPLX ? 2 : 1) +
                      sizeof(int) * (kMaxSub + 2 * P::NSB * P::NSB);
  auto kern = spread2d_phased_kernel<W, T, CPLX>;
  if (smem > 48 * 1024) FB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kern<<<unsigned(sb.max_sub), P::THREADS, smem, s>>>(static_cast<const Rec<2, T>*>(recs), weights, uniform, strengths,
                                                       sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                       make_es_poly<W, T>(poly), grid_real, grid_cplx);
  FB_LAUNCH_CHECK();
}

template <int D, int W, typename T, bool CPLX>
void launch_spread_generic(const void* recs, const T* weights, T uniform, const cplx_t<T>* strengths,
                           const SortBufs& sb, const Geom& g, const std::vector<double>& poly, T* grid_real,
                           cplx_t<T>* grid_cplx, cudaStream_t s) {
  const size_t smem = size_t(g.tile_cells()) * sizeof(T) * (CPLX ? 2 : 1);
  auto kern = spread_kernel<D, W, T, CPLX>;
  if (smem > 48 * 1024) FB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kern<<<unsigned(sb.max_sub), 256, smem, s>>>(static_cast<const Rec<D, T>*>(recs), weights, uniform, strengths,
                                                sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                make_es_poly<W, T>(poly), grid_real, grid_cplx);
  FB_LAUNCH_CHECK();
}

template <int W, typename T>
void launch_interp2d(const void* recs, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
                     const std::vector<double>& poly, const cplx_t<T>* field, int mode, double* grad, double2* out2,
                     int acc, const int* status, cudaStream_t s, const GradScale& gs) {
  constexpr int TW = kTile2D + W;
  const size_t smem = sizeof(cplx_t<T>) * TW * TW;
  auto kern = interp2d_tile_kernel<W, T>;
  if (smem > 48 * 1024) FB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kern<<<unsigned(sb.max_sub), 256, smem, s>>>(static_cast<const Rec<2, T>*>(recs), weights, uniform, sb.sub_bin.p,
                                                sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                make_es_poly<W, T>(poly), field, mode, grad, out2, acc, status, gs);
  FB_LAUNCH_CHECK();
}

template <int D, int W, typename T>
void launch_interp_generic(const void* recs, int64_t N, const T* weights, T uniform, const Geom& g,
                           const std::vector<double>& poly, const cplx_t<T>* fields, int nfields, int mode,
                           double* grad, double2* out2, int acc, const int* status, cudaStream_t s,
                           const GradScale& gs) {
  if (N <= 0) return;
  const int grid = point_grid(N, 16);
  const Rec<D, T>* r = static_cast<const Rec<D, T>*>(recs);
  if (nfields == 2) {
    interp_kernel<D, W, T, 2><<<grid, 256, 0, s>>>(r, N, weights, uniform, g, make_es_poly<W, T>(poly), fields, g.G(),
                                                   mode, grad, out2, acc, status, gs);
  } else {
    interp_kernel<D, W, T, 1><<<grid, 256, 0, s>>>(r, N, weights, uniform, g, make_es_poly<W, T>(poly), fields, g.G(),
                                                   mode, grad, out2, acc, status, gs);
  }
  FB_LAUNCH_CHECK();
}

#define FB_FOR_W(T, X)                                                \
  switch (g.w) {                                                      \
    case 2: X(2); break;                                              \
    case 3: X(3); break;                                              \
    case 4: X(4); break;                                              \
    case 5: X(5); break;                                              \
    case 6: X(6); break;                                              \
    case 7: X(7); break;                                              \
    case 8: X(8); break;                                              \
    case 9: X(9); break;                                              \
    case 10: X(10); break;                                            \
    default:                                                          \
      if (sizeof(T) == 8) {                                           \
        switch (g.w) {                                                \
          case 11: X(11); break;                                      \
          case 12: X(12); break;                                      \
          case 13: X(13); break;                                      \
          case 14: X(14); break;                                      \
          case 15: X(15); break;                                      \
          case 16: X(16); break;                                      \
          default: throw InvalidArgument("unsupported kernel width"); \
        }                                                             \
      } else {                                                        \
        throw InvalidArgument("unsupported kernel width for FP32");   \
      }                                                               \
  }

#define FB_WCLAMP(T, WW) ((sizeof(T) == 4 && (WW) > 10) ? 10 : (WW))

template <typename T, bool CPLX>
void spread_dispatch(const void* recs, const T* weights, T uniform, const cplx_t<T>* strengths, const SortBufs& sb,
                     const Geom& g, const std::vector<double>& poly, T* grid_real, cplx_t<T>* grid_cplx, cudaStream_t s) {
  if (g.D == 2) {
#define FB_S2(WW) \
  launch_spread2d<FB_WCLAMP(T, WW), T, CPLX>(recs, weights, uniform, strengths, sb, g, poly, grid_real, grid_cplx, s)
    FB_FOR_W(T, FB_S2)
#undef FB_S2
  } else if (g.D == 1) {
#define FB_S1(WW)                                                                                                \
  launch_spread_generic<1, FB_WCLAMP(T, WW), T, CPLX>(recs, weights, uniform, strengths, sb, g, poly, grid_real, \
                                                      grid_cplx, s)
    FB_FOR_W(T, FB_S1)
#undef FB_S1
  } else {
#define FB_S3(WW)                                                                                                \
  launch_spread_generic<3, FB_WCLAMP(T, WW), T, CPLX>(recs, weights, uniform, strengths, sb, g, poly, grid_real, \
                                                      grid_cplx, s)
    FB_FOR_W(T, FB_S3)
#undef FB_S3
  }
}

template <typename T>
void spread_real(const void* recs, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
                 const std::vector<double>& poly, T* grid, cudaStream_t s) {
  spread_dispatch<T, false>(recs, weights, uniform, nullptr, sb, g, poly, grid, nullptr, s);
}

template <typename T>
void spread_cplx(const void* recs, const cplx_t<T>* strengths, const SortBufs& sb, const Geom& g,
                 const std::vector<double>& poly, cplx_t<T>* grid, cudaStream_t s) {
  spread_dispatch<T, true>(recs, nullptr, T(1), strengths, sb, g, poly, nullptr, grid, s);
}

template <typename T>
void interp(const void* recs, int64_t N, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
            const std::vector<double>& poly, const cplx_t<T>* fields, int nfields, int mode, double* grad,
            double2* out2, int accumulate, const int* status, cudaStream_t s, GradScale gs) {
  if (g.D == 2 && nfields == 1) {
#define FB_I2(WW)                                                                                                  \
  launch_interp2d<FB_WCLAMP(T, WW), T>(recs, weights, uniform, sb, g, poly, fields, mode, grad, out2, accumulate, \
                                       status, s, gs)
    FB_FOR_W(T, FB_I2)
#undef FB_I2
  } else if (g.D == 1) {
#define FB_I1(WW)                                                                                             \
  launch_interp_generic<1, FB_WCLAMP(T, WW), T>(recs, N, weights, uniform, g, poly, fields, nfields, mode, grad, \
                                                out2, accumulate, status, s, gs)
    FB_FOR_W(T, FB_I1)
#undef FB_I1
  } else if (g.D == 2) {
#define FB_I2G(WW)                                                                                            \
  launch_interp_generic<2, FB_WCLAMP(T, WW), T>(recs, N, weights, uniform, g, poly, fields, nfields, mode, grad, \
                                                out2, accumulate, status, s, gs)
    FB_FOR_W(T, FB_I2G)
#undef FB_I2G
  } else {
#define FB_I3(WW)                                                                                             \
  launch_interp_generic<3, FB_WCLAMP(T, WW), T>(recs, N, weights, uniform, g, poly, fields, nfields, mode, grad, \
                                                out2, accumulate, status, s, gs)
    FB_FOR_W(T, FB_I3)
#undef FB_I3
  }
}

#define FB_INSTANTIATE_NUFFT(T)                                                                                     \
  template void bin_sort<T>(const double*, int64_t, const MapParams&, const Geom&, SortBufs&, void*, int*,          \
                            cudaStream_t);                                                                           \
  template void spread_real<T>(const void*, const T*, T, const SortBufs&, const Geom&, const std::vector<double>&,    \
                               T*, cudaStream_t);                                                                    \
  template void spread_cplx<T>(const void*, const cplx_t<T>*, const SortBufs&, const Geom&,                         \
                               const std::vector<double>&, cplx_t<T>*, cudaStream_t);                                \
  template void interp<T>(const void*, int64_t, const T*, T, const SortBufs&, const Geom&, const std::vector<double>&, \
                          const cplx_t<T>*, int, int, double*, double2*, int, const int*, cudaStream_t, GradScale);

}  // namespace fb
