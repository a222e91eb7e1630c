// Kernel bodies and host launchers for nufft.cuh, instantiated once per
// precision in nufft_f32.cu / nufft_f64.cu.
#pragma once

#include <cuda.h>  // CUtensorMap (the encoder is fetched from the driver at run time)

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

// Maps coordinate a of a point to (fine-grid cell, fraction in [0, 1)).
// Returns false for a non-finite coordinate (then cell = 0, fraction = 0 so
// all later accesses stay in bounds).
//
// NUwU/NUwNU (kind 0) use x = (p - round(p/L)) 2 pi / L (source/fresco/
// nuwu.hpp:219: the period count is subtracted, not its multiple of L); UwNU
// k-points (kind 1) use x = p 2 pi / L (uwnu.hpp:245).  The fine-grid
// coordinate x nf / (2 pi) is formed as t * (nf / L) with t = p - round(p/L)
// (or p): one multiplication instead of the reference's divide-and-rescale
// chain, within a few ulp of it.  round(p/L) keeps the exact division, so a
// coordinate on a half period rounds as in the reference.
// round(p / L): the quotient is formed with the reciprocal, which is within an
// ulp of p / L and so rounds the same way unless p / L lies within 1e-9 of a
// half-integer; there the exact division decides.
static __device__ __noinline__ double round_exact_quotient(double p, double L) { return round(p / L); }

__device__ __forceinline__ double round_quotient(double p, double L, double invL) {
  const double q = p * invL;
  const double fr = q - floor(q);
  if (fabs(fr - 0.5) < 1e-9) return round_exact_quotient(p, L);  // rare: a call, never speculated
  return round(q);
}

__device__ __forceinline__ bool map_coord(double p, const MapParams& mp, int nf, int a, int& c, double& f) {
  const double t = mp.kind == 0 ? p - round_quotient(p, mp.L[a], mp.invL[a]) : p;
  double u = t * mp.scale[a];
  if (!(fabs(u) < 1.0e9)) {
    if (!isfinite(u)) {
      c = 0;
      f = 0.0;
      return false;
    }
    u -= double(nf) * floor(u / double(nf));  // far outside the box: fold first
  }
  const double fl = floor(u);
  f = u - fl;  // exact
  int ci = int(fl);
  if (ci < 0) ci += nf;
  else if (ci >= nf) ci -= nf;
  if (ci < 0 || ci >= nf) {
    ci %= nf;
    if (ci < 0) ci += nf;
  }
  c = ci;
  return true;
}

template <int D>
__device__ __forceinline__ int bin_of_cell(const int (&c)[3], const Geom& g) {
  if (D == 2) return (c[0] / kTile2D) + g.nb[0] * (c[1] / kTile2D);
  return c[0] / g.tile[0] + g.nb[0] * (c[1] / g.tile[1] + g.nb[1] * (c[2] / g.tile[2]));
}

template <int D>
__device__ __forceinline__ int point_bin(const double (&p)[D], const MapParams& mp, const Geom& g, int (&c)[3],
                                         double (&f)[3], bool& ok) {
  ok = true;
#pragma unroll
  for (int a = 0; a < D; ++a) ok &= map_coord(p[a], mp, g.nf[a], a, c[a], f[a]);
  return bin_of_cell<D>(c, g);
}

// Points per thread per round in the sort passes: the coordinates of a round
// are loaded before any of them is used, so their latencies overlap.
constexpr int kSortBatch = 4;

template <int D>
__device__ __forceinline__ void load_batch(const double* __restrict__ pts, int64_t jb, int64_t j1, int64_t step,
                                           int stride, double (&p)[kSortBatch][D]) {
#pragma unroll
  for (int u = 0; u < kSortBatch; ++u) {
    const int64_t j = jb + u * step;
#pragma unroll
    for (int a = 0; a < D; ++a) p[u][a] = j < j1 ? pts[j * stride + a] : 0.0;
  }
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

// Sort pass 1: maps every point once (cell, fraction), writes its packed
// record in input order, and counts the block's points per bin in shared
// memory; one global atomic per non-empty bin then reserves the block's
// segment inside that bin (blk_off, block-major).
template <int D, typename T>
__global__ void __launch_bounds__(kSortThreads, 2) sort_count_kernel(const double* __restrict__ pts, int64_t N,
                                                                  int64_t chunk, MapParams mp, Geom g, int* bin_total,
                                                                  int* blk_off, Rec<D, T>* unsorted, int* status) {
  extern __shared__ int sh_hist[];
  const int nbins = int(g.nbins());
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh_hist[i] = 0;
  __syncthreads();
  const int64_t j0 = int64_t(blockIdx.x) * chunk, j1 = min(N, j0 + chunk);
  bool bad = false;
  for (int64_t jb = j0 + threadIdx.x; jb < j1; jb += kSortBatch * int64_t(blockDim.x)) {
    double p[kSortBatch][D];
    load_batch<D>(pts, jb, j1, blockDim.x, mp.stride, p);
#pragma unroll
    for (int u = 0; u < kSortBatch; ++u) {
      const int64_t j = jb + u * int64_t(blockDim.x);
      if (j >= j1) break;
      int c[3] = {0, 0, 0};
      double f[3] = {0, 0, 0};
      bool ok;
      const int bin = point_bin<D>(p[u], mp, g, c, f, ok);
      bad |= !ok;
      atomicAdd(&sh_hist[bin], 1);
      Rec<D, T> r;
      r.cell = pack_cell(D, c[0], c[1], c[2]);
#pragma unroll
      for (int a = 0; a < D; ++a) r.f[a] = T(f[a]);
      r.idx = uint32_t(j);
      unsorted[j] = r;
    }
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
  __syncthreads();
  int* my_off = blk_off + int64_t(blockIdx.x) * nbins;
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
    const int cnt = sh_hist[i];
    if (cnt) my_off[i] = atomicAdd(&bin_total[i], cnt);
  }
}

// Bin starts from the bin totals, computed by every block of a sort (each
// thread scans a contiguous share of the bins); the block with `publish` also
// writes them and the subproblem table (each bin cut into equal parts of at
// most kMaxSub points).  on_bin(b, start) is called for each bin of the
// thread's share.
template <typename F>
__device__ __forceinline__ void scan_bins(const int* bin_total, int nbins, bool publish, int* bin_start, int* sub_bin,
                                          int* sub_start, int* sub_count, int* num_sub, int max_sub, int* s_warp,
                                          F&& on_bin) {
  const int tid = threadIdx.x;
  const int per = (nbins + int(blockDim.x) - 1) / int(blockDim.x);
  const int b0 = min(nbins, tid * per), b1 = min(nbins, b0 + per);
  int npts = 0, nsub = 0;
  for (int b = b0; b < b1; ++b) {
    const int c = bin_total[b];
    npts += c;
    nsub += (c + kMaxSub - 1) / kMaxSub;
  }
  int tot_pts;
  int run = block_exclusive_scan(npts, &tot_pts, s_warp);
  const int first_start = run;
  for (int b = b0; b < b1; ++b) {
    on_bin(b, run);
    if (publish) bin_start[b] = run;
    run += bin_total[b];
  }
  if (publish) {
    int tot_sub;
    int sbase = block_exclusive_scan(nsub, &tot_sub, s_warp);
    int st = first_start;
    for (int b = b0; b < b1; ++b) {
      const int c = bin_total[b];
      const int parts = (c + kMaxSub - 1) / kMaxSub;  // equal parts of at most kMaxSub points
      for (int q = 0; q < parts; ++q) {
        if (sbase < max_sub) {
          const int lo = int(int64_t(q) * c / parts), hi = int(int64_t(q + 1) * c / parts);
          sub_bin[sbase] = b;
          sub_start[sbase] = st + lo;
          sub_count[sbase] = hi - lo;
        }
        ++sbase;
      }
      st += c;
    }
    if (tid == 0) {
      bin_start[nbins] = tot_pts;
      *num_sub = min(tot_sub, max_sub);
    }
  }
}

// Sort pass 2: every block scans the bin totals itself (bin starts), block 0
// also publishes them and the subproblem table; then each block hands out the
// slots of its segments with shared-memory cursors (the counts are those of
// pass 1, so every slot is written exactly once) and moves its records
// there.  The last block to finish clears bin_total for the next sort.
template <int D, typename T>
__global__ void __launch_bounds__(kSortThreads, 2) sort_scatter_kernel(
    const Rec<D, T>* __restrict__ unsorted, int64_t N, int64_t chunk, Geom g, int* bin_total,
    const int* __restrict__ blk_off, int* bin_start, int* sub_bin, int* sub_start, int* sub_count, int* num_sub,
    int max_sub, unsigned* done, Rec<D, T>* out, int* status) {
  extern __shared__ int sh_cur[];
  __shared__ int s_warp[32];
  __shared__ bool s_last;
  const int nbins = int(g.nbins());
  const int tid = threadIdx.x;
  const int* my_off = blk_off + int64_t(blockIdx.x) * nbins;
  // bins this block has no points in get stale offsets that are never used
  scan_bins(bin_total, nbins, blockIdx.x == 0, bin_start, sub_bin, sub_start, sub_count, num_sub, max_sub, s_warp,
            [&](int b, int start) { sh_cur[b] = start + my_off[b]; });
  __syncthreads();
  const int64_t j0 = int64_t(blockIdx.x) * chunk, j1 = min(N, j0 + chunk);
  for (int64_t jb = j0 + tid; jb < j1; jb += kSortBatch * int64_t(blockDim.x)) {
    Rec<D, T> r[kSortBatch];
#pragma unroll
    for (int u = 0; u < kSortBatch; ++u) {
      const int64_t j = jb + u * int64_t(blockDim.x);
      if (j < j1) r[u] = unsorted[j];
    }
#pragma unroll
    for (int u = 0; u < kSortBatch; ++u) {
      if (jb + u * int64_t(blockDim.x) >= j1) break;
      int c[3];
      unpack_cell(D, r[u].cell, c[0], c[1], c[2]);
      const int dest = atomicAdd(&sh_cur[bin_of_cell<D>(c, g)], 1);
      if (dest < 0 || int64_t(dest) >= N) {
        raise_status(status, STATUS_OVERFLOW);
        continue;
      }
      out[dest] = r[u];
    }
  }
  // every block has read bin_total before it counts itself done
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    for (int b = tid; b < nbins; b += blockDim.x) bin_total[b] = 0;
    if (tid == 0) *done = 0u;
  }
}

// ---------------------------------------------------------------------------
// One-pass bin sort: one cooperative launch (every block resident at once)
// does what the two passes above do, with each point's record crossing HBM
// once each way.  Block b maps the points [b chunk, (b + 1) chunk) and keeps
// them in shared memory (cell, fractions; struct of arrays) with their rank
// inside the block's share of their bin (shared histogram atomics).  It
// reserves its segment in every non-empty bin with one global atomic, lists
// its points in bin order (block-local exclusive scan of its histogram) and
// waits at a grid-wide barrier (a monotonic arrival counter, bounded by
// kGridBarrierNs).  Then every block scans the bin totals, block 0 publishes
// the bin starts and the subproblem table, and each block writes its records
// in bin order, so that its run of points in one bin goes out as one
// contiguous stretch.  The last block to finish clears the bin totals.  A
// barrier that gives up raises STATUS_TIMEOUT together with
// STATUS_NONFINITE_INPUT, which makes the evaluation's energy and gradient
// NaN, and the block writes no records.
// ---------------------------------------------------------------------------
constexpr int kOneThreads = 1024;
// Shared memory of the one-pass sort: three int arrays of nbins (rounded up
// to 16 bytes) and, per point, its fractions, cell, rank and bin-order index.
template <int D, typename T>
__host__ __device__ constexpr size_t onepass_point_bytes() {
  return D * sizeof(T) + sizeof(uint32_t) + 2 * sizeof(uint16_t);
}
__host__ __device__ inline size_t onepass_bin_bytes(int nbins) { return (size_t(3 * nbins) * sizeof(int) + 15) & ~size_t(15); }

template <int D, typename T>
__global__ void __launch_bounds__(kOneThreads, 1) sort_onepass_kernel(
    const double* __restrict__ pts, int64_t N, int64_t chunk, MapParams mp, Geom g, int* bin_total, int* bin_start,
    int* sub_bin, int* sub_start, int* sub_count, int* num_sub, int max_sub, unsigned* done,
    unsigned long long* bar, Rec<D, T>* out, int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_warp[32];
  __shared__ bool s_last;
  const int nbins = int(g.nbins());
  const int tid = threadIdx.x;
  int* hist = reinterpret_cast<int*>(smem_raw);  // block's bin counts, then its segment offsets
  int* lstart = hist + nbins;                    // block-local bin starts
  int* gstart = lstart + nbins;                  // global bin starts
  T* fr = reinterpret_cast<T*>(smem_raw + onepass_bin_bytes(nbins));  // D arrays of chunk fractions
  uint32_t* cell = reinterpret_cast<uint32_t*>(fr + D * chunk);
  uint16_t* rank = reinterpret_cast<uint16_t*>(cell + chunk);
  uint16_t* inv = rank + chunk;

  for (int b = tid; b < nbins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  const int64_t j0 = int64_t(blockIdx.x) * chunk, j1 = min(N, j0 + chunk);
  const int cnt = j1 > j0 ? int(j1 - j0) : 0;
  bool bad = false;
  for (int64_t jb = j0 + tid; jb < j1; jb += kSortBatch * int64_t(blockDim.x)) {
    double p[kSortBatch][D];
    load_batch<D>(pts, jb, j1, blockDim.x, mp.stride, p);
#pragma unroll
    for (int u = 0; u < kSortBatch; ++u) {
      const int64_t j = jb + u * int64_t(blockDim.x);
      if (j >= j1) break;
      int c[3] = {0, 0, 0};
      double f[3] = {0, 0, 0};
      bool ok;
      const int bin = point_bin<D>(p[u], mp, g, c, f, ok);
      bad |= !ok;
      const int i = int(j - j0);
      rank[i] = uint16_t(atomicAdd(&hist[bin], 1));
      cell[i] = pack_cell(D, c[0], c[1], c[2]);
#pragma unroll
      for (int a = 0; a < D; ++a) fr[a * chunk + i] = T(f[a]);
    }
  }
  if (bad) raise_status(status, STATUS_NONFINITE_INPUT);
  __syncthreads();
  {  // block-local bin starts
    const int per = (nbins + int(blockDim.x) - 1) / int(blockDim.x);
    const int b0 = min(nbins, tid * per), b1 = min(nbins, b0 + per);
    int mine = 0;
    for (int b = b0; b < b1; ++b) mine += hist[b];
    int tot;
    int run = block_exclusive_scan(mine, &tot, s_warp);
    for (int b = b0; b < b1; ++b) {
      lstart[b] = run;
      run += hist[b];
    }
  }
  __syncthreads();
  for (int b = tid; b < nbins; b += blockDim.x) {
    const int c = hist[b];
    if (c) hist[b] = atomicAdd(&bin_total[b], c);  // the block's segment inside bin b
  }
  for (int i = tid; i < cnt; i += blockDim.x) {
    int c[3];
    unpack_cell(D, cell[i], c[0], c[1], c[2]);
    inv[lstart[bin_of_cell<D>(c, g)] + rank[i]] = uint16_t(i);
  }
  const bool arrived = grid_barrier(bar, gridDim.x);
  if (!arrived) {
    if (tid == 0) raise_status(status, STATUS_TIMEOUT | STATUS_NONFINITE_INPUT);
  } else {
    scan_bins(bin_total, nbins, blockIdx.x == 0, bin_start, sub_bin, sub_start, sub_count, num_sub, max_sub, s_warp,
              [&](int b, int start) { gstart[b] = start; });
    __syncthreads();
    for (int q = tid; q < cnt; q += blockDim.x) {
      const int i = inv[q];
      int c[3];
      unpack_cell(D, cell[i], c[0], c[1], c[2]);
      const int bin = bin_of_cell<D>(c, g);
      const int64_t dest = int64_t(gstart[bin]) + hist[bin] + (q - lstart[bin]);
      if (dest < 0 || dest >= N) {
        raise_status(status, STATUS_OVERFLOW);
        continue;
      }
      Rec<D, T> r;
      r.cell = cell[i];
#pragma unroll
      for (int a = 0; a < D; ++a) r.f[a] = fr[a * chunk + i];
      r.idx = uint32_t(j0 + i);
      out[dest] = r;
    }
  }
  // every block has read bin_total before it counts itself done
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    for (int b = tid; b < nbins; b += blockDim.x) bin_total[b] = 0;
    if (tid == 0) *done = 0u;
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
// One block per subproblem (the points of one 64 x 64-cell tile).  The tile
// is cut into sub-blocks of SB x SB cells (SB = 8 for w <= 8, 16 for
// w <= 16).  A point's w x w footprint only reaches the neighbouring
// sub-blocks, so sub-blocks whose (a, b) indices have the same parities never
// touch the same cell: the tile is spread in four phases, one per parity
// class, and within a phase every warp owns whole sub-blocks, whose points
// it adds one after another (program order within the warp, __syncwarp
// between rounds).  So no two threads ever update one cell concurrently and
// plain shared-memory read-modify-writes suffice.
//
// Per point, the whole warp works on its footprint: lanes hold the x and y
// tap values (one polynomial each, coefficients in registers), the products
// are formed after two shuffles, and the w x w cells are covered in passes
// of R = 32 / w rows.  The tile pitch P = 64 + w is congruent to w modulo
// 32, so the R * w cells of one pass fall in R * w distinct banks: every
// access is conflict-free.  With w <= 8 two points, one from each of two
// sub-blocks of the phase, share one round of tap evaluation (lanes 0-15 and
// 16-31).
//
// Before the phases, the block stages its points in shared memory grouped by
// sub-block, already converted to (tile offset, polynomial variables,
// weight).  At the end the tile is added to the fine grid with vector
// atomics (float4: four real or two complex cells); cells that no
// neighbouring tile can reach are stored plainly when the subproblem is its
// tile's only one.
// ---------------------------------------------------------------------------

template <int W>
struct Tile2D {
  static constexpr int SB = W <= 8 ? 8 : 16;
  static constexpr int NSB = kTile2D / SB;  // sub-blocks per tile edge
  static constexpr int PER_PHASE = (NSB / 2) * (NSB / 2);
  static constexpr int NWARP = 8;
  static constexpr int THREADS = 32 * NWARP;
  static constexpr int PAD = W / 2;
  static constexpr int EDGE = kTile2D + W;  // tile rows and pitch (cells), origin org - PAD
  static constexpr int PPW = W <= 8 ? 2 : 1;  // points per tap round
  static constexpr int HL = 32 / PPW;         // lanes per point in a tap round
  static constexpr int R = 32 / W;            // footprint rows per pass
  static constexpr int NPASS = (W + R - 1) / R;
};

template <typename T, bool CPLX>
struct alignas(16) Staged2D {
  int base;  // tile offset (cells) of the footprint's first cell
  T u0, u1;  // polynomial variables along x and y
  T wr;      // weight (real part)
};
template <typename T>
struct alignas(16) Staged2D<T, true> {
  int base;
  T u0, u1;
  T wr, wi;
};

template <int W, typename T, bool CPLX>
__host__ __device__ constexpr size_t spread2d_smem_bytes() {
  using P = Tile2D<W>;
  return sizeof(Staged2D<T, CPLX>) * kMaxSub + sizeof(T) * (CPLX ? 2 : 1) * P::EDGE * P::EDGE +
         sizeof(int) * 2 * P::NSB * P::NSB;
}

// Adds VW consecutive cells (VW = 4 real or 2 complex: one float4) of the
// shared tile row to the fine grid; the group's first global column gc is a
// multiple of VW.
template <typename T, bool CPLX>
__device__ __forceinline__ void flush_group_f32(const T* trow, int tc0, int edge, float* gdst, bool plain) {
  constexpr int NC = CPLX ? 2 : 1;
  constexpr int VW = 4 / NC;
  float v[4];
#pragma unroll
  for (int e = 0; e < VW; ++e) {
    const int tc = tc0 + e;
    const bool in = tc >= 0 && tc < edge;
#pragma unroll
    for (int q = 0; q < NC; ++q) v[e * NC + q] = in ? float(trow[tc * NC + q]) : 0.f;
  }
  if (v[0] == 0.f && v[1] == 0.f && v[2] == 0.f && v[3] == 0.f) return;
  const float4 val = make_float4(v[0], v[1], v[2], v[3]);
  if (plain) {
    *reinterpret_cast<float4*>(gdst) = val;
  } else {
    atomicAdd(reinterpret_cast<float4*>(gdst), val);
  }
}

// Work of one block of the 2D tile kernels: the cnt sorted records from
// `start` lie in the 64 x 64-cell tile with origin (org0, org1); bin_range
// points at the tile's bin start (bin_range[1] - bin_range[0] is the tile's
// point count, so the subproblem is its tile's only one when it equals cnt);
// the fine grid starts grid_off cells after the kernel's grid pointer;
// uniform is the weight when there are no per-point weights.
template <typename T>
struct TileWork {
  int start, cnt, org0, org1;
  const int* bin_range;
  int64_t grid_off;
  T uniform;
};

// Block -> work of one pattern's subproblem table (the single-pattern
// potentials).
template <typename T>
struct TileMap1 {
  const int* __restrict__ sub_bin;
  const int* __restrict__ sub_start;
  const int* __restrict__ sub_count;
  const int* __restrict__ num_sub;
  const int* __restrict__ bin_start;
  const int* __restrict__ status;  // evaluation status word (interpolation), may be null
  T uniform;
  int has_tmap = 0;  // interpolation: tmap describes the interpolated fine grid
  int polls = 0;     // first bounded wait for a tile copy (mbarrier polls)
  double* energy = nullptr;  // the evaluation's energy, made NaN if a tile copy never lands (may be null)
  CUtensorMap tmap;
  // tensor map of the fine grid for tile copies (the kernel parameter must be
  // __grid_constant__ for its address to be usable), or null
  __device__ __forceinline__ const CUtensorMap* tile_tmap() const { return has_tmap ? &tmap : nullptr; }
  __device__ __forceinline__ int* err_status() const { return const_cast<int*>(status); }
  __device__ __forceinline__ int wait_polls() const { return polls; }
  __device__ __forceinline__ double* fail_energy() const { return energy; }
  __device__ __forceinline__ bool fetch(const Geom& g, TileWork<T>& w) const {
    const int sub = blockIdx.x;
    if (sub >= *num_sub) return false;
    const int bin = sub_bin[sub];
    w.start = sub_start[sub];
    w.cnt = sub_count[sub];
    w.org0 = (bin % g.nb[0]) * kTile2D;
    w.org1 = (bin / g.nb[0]) * kTile2D;
    w.bin_range = bin_start + bin;
    w.grid_off = 0;
    w.uniform = uniform;
    return true;
  }
  __device__ __forceinline__ bool nonfinite(const TileWork<T>&) const {
    return status != nullptr && ((*status) & STATUS_NONFINITE_INPUT);
  }
};

// Staging shared by the 2D spreading kernels: zeroes the tile, groups the
// block's points by 8 x 8-cell sub-block (counts, exclusive scan) and stores
// each as (tile offset of its footprint, polynomial variables, weight) in
// sub-block order.
template <int W, typename T, bool CPLX>
__device__ __forceinline__ void spread2d_stage(const Rec<2, T>* __restrict__ recs, const T* __restrict__ weights,
                                               const cplx_t<T>* __restrict__ strengths, const TileWork<T>& wk,
                                               Staged2D<T, CPLX>* srec, T* tile, int* sb_count, int* sb_start) {
  using P = Tile2D<W>;
  using S = Staged2D<T, CPLX>;
  constexpr int NC = CPLX ? 2 : 1;
  constexpr int E = P::EDGE;
  constexpr int NSB2 = P::NSB * P::NSB;
  const int start = wk.start, cnt = wk.cnt, org0 = wk.org0, org1 = wk.org1;
  const int tid = threadIdx.x;
  for (int i = tid; i < E * E * NC; i += P::THREADS) tile[i] = T(0);
  for (int i = tid; i < NSB2; i += P::THREADS) sb_count[i] = 0;
  // this thread's points are p = tid + THREADS k; their cells are loaded
  // together (one round of load latency), and their sub-block and rank in it
  // stay in registers until the sub-block starts are known
  constexpr int PPT = (kMaxSub + P::THREADS - 1) / P::THREADS;
  uint32_t cellk[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k)
    if (tid + P::THREADS * k < cnt) cellk[k] = recs[start + tid + P::THREADS * k].cell;
  int slot[PPT];  // sub-block << 16 | rank in sub-block, or -1
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    slot[k] = -1;
    if (tid + P::THREADS * k >= cnt) continue;
    int c0, c1, c2;
    unpack_cell(2, cellk[k], c0, c1, c2);
    const int sbi = ((c0 - org0) / P::SB) + P::NSB * ((c1 - org1) / P::SB);
    slot[k] = (sbi << 16) | atomicAdd(&sb_count[sbi], 1);
  }
  __syncthreads();
  if (tid < 32) {  // exclusive scan of the sub-block counts (one warp)
    constexpr int PER = (NSB2 + 31) / 32;
    int v[PER], tot = 0;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const int i = tid * PER + e;
      v[e] = i < NSB2 ? sb_count[i] : 0;
      tot += v[e];
    }
    int inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (tid >= o) inc += t;
    }
    int run = inc - tot;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const int i = tid * PER + e;
      if (i < NSB2) sb_start[i] = run;
      run += v[e];
    }
  }
  __syncthreads();
  // stage: grouped by sub-block, converted to (tile offset, u0, u1, weight);
  // the records are loaded together as well
  {
    Rec<2, T> rk[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k)
      if (slot[k] >= 0) rk[k] = recs[start + tid + P::THREADS * k];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      if (slot[k] < 0) continue;
      const Rec<2, T>& r = rk[k];
      int c0, c1, c2;
      unpack_cell(2, r.cell, c0, c1, c2);
      S st;
      const int s0 = es_start<W, T>(r.f[0], st.u0);
      const int s1 = es_start<W, T>(r.f[1], st.u1);
      st.base = (c1 - org1 + s1 + P::PAD) * E + (c0 - org0 + s0 + P::PAD);
      if constexpr (CPLX) {
        const cplx_t<T> v = strengths[r.idx];
        st.wr = v.x;
        st.wi = v.y;
      } else {
        st.wr = weights ? weights[r.idx] : wk.uniform;
      }
      srec[sb_start[slot[k] >> 16] + (slot[k] & 0xffff)] = st;
    }
  }
  __syncthreads();
}

// Adds the shared tile of one 2D subproblem to the fine grid: float4 vector
// atomics (four real or two complex cells) for FP32, scalar atomics for FP64;
// cells that no neighbouring tile can reach are stored plainly when the
// subproblem is its tile's only one.
template <int W, typename T, bool CPLX>
__device__ __forceinline__ void spread2d_flush(const T* tile, const TileWork<T>& wk, const Geom& g, T* grid_real,
                                               cplx_t<T>* grid_cplx) {
  using P = Tile2D<W>;
  constexpr int NC = CPLX ? 2 : 1;
  constexpr int E = P::EDGE;
  const int org0 = wk.org0, org1 = wk.org1, tid = threadIdx.x;
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  if (sizeof(T) == 4 && nf0 % (4 / NC) == 0) {
    constexpr int VW = 4 / NC;                          // cells per float4
    constexpr int LEFT = (VW - P::PAD % VW) % VW;       // cells left of the tile origin in the first group
    constexpr int NG = (E + LEFT + VW - 1) / VW;        // groups per tile row
    // cells [W, 64) of the tile (relative to org - PAD) along both axes are
    // out of reach of every other tile; with one subproblem in the bin and
    // whole tiles (nf a multiple of 64) they are written with plain stores
    const bool sole = wk.cnt == wk.bin_range[1] - wk.bin_range[0] && nf0 % kTile2D == 0 && nf1 % kTile2D == 0;
    for (int i = tid; i < E * NG; i += P::THREADS) {
      const int ty = i / NG, j = i - ty * NG;
      const int tc0 = j * VW - LEFT;
      const int gy = wrap_index(org1 - P::PAD + ty, nf1);
      const int gx = wrap_index(org0 - P::PAD + tc0, nf0);
      const bool plain = sole && ty >= W && ty < kTile2D && tc0 >= W && tc0 + VW <= kTile2D;
      float* dst = CPLX ? reinterpret_cast<float*>(grid_cplx + int64_t(gy) * nf0 + gx)
                        : reinterpret_cast<float*>(grid_real + int64_t(gy) * nf0 + gx);
      flush_group_f32<T, CPLX>(tile + ty * E * NC, tc0, E, dst, plain);
    }
  } else {
    for (int i = tid; i < E * E; i += P::THREADS) {
      const int ty = i / E, tc = i - ty * E;
      const int64_t gi = int64_t(wrap_index(org1 - P::PAD + ty, nf1)) * nf0 + wrap_index(org0 - P::PAD + tc, nf0);
      if constexpr (CPLX) {
        const T re = tile[2 * i], im = tile[2 * i + 1];
        if (re != T(0) || im != T(0)) atomic_add_cplx<T>(grid_cplx + gi, re, im);
      } else {
        const T v = tile[i];
        if (v != T(0)) atomicAdd(grid_real + gi, v);
      }
    }
  }
}

template <int W, typename T, bool CPLX, typename Map>
__global__ void __launch_bounds__(Tile2D<W>::THREADS) spread2d_tile_kernel(
    const Rec<2, T>* __restrict__ recs, const T* __restrict__ weights, const cplx_t<T>* __restrict__ strengths,
    const Map map, Geom g, const EsPoly<W, T> poly, T* grid_real, cplx_t<T>* grid_cplx) {
  using P = Tile2D<W>;
  using S = Staged2D<T, CPLX>;
  constexpr int NC = CPLX ? 2 : 1;
  constexpr int E = P::EDGE;
  constexpr int NSB2 = P::NSB * P::NSB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* srec = reinterpret_cast<S*>(smem_raw);
  T* tile = reinterpret_cast<T*>(srec + kMaxSub);
  int* sb_count = reinterpret_cast<int*>(tile + E * E * NC);
  int* sb_start = sb_count + NSB2;

  TileWork<T> wk;
  if (!map.fetch(g, wk)) return;
  if (grid_real) grid_real += wk.grid_off;
  if (grid_cplx) grid_cplx += wk.grid_off;
  spread2d_stage<W, T, CPLX>(recs, weights, strengths, wk, srec, tile, sb_count, sb_start);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  // tap roles: lane hl of each half evaluates x tap hl (hl < W) or y tap hl - W
  const int half = lane / P::HL, hl = lane % P::HL;
  const bool xl = hl < W;
  const int m = xl ? hl : (hl < 2 * W ? hl - W : 0);
  constexpr int Q = EsPolyDeg<W>::Q;
  T cr[Q + 1];
#pragma unroll
  for (int mm = 0; mm < W; ++mm)
    if (mm == m) {
#pragma unroll
      for (int d = 0; d <= Q; ++d) cr[d] = poly.c[mm][d];
    }
  // cell roles: lane = rr * W + cc covers row rr (+ k R) and column cc
  const int rr = lane / W, cc = lane % W;
  const bool cell_lane = lane < P::R * W;
  const int lane_off = rr * E + cc;

  // Within a phase the PPW lane halves of a warp take different sub-blocks,
  // whose footprints never overlap, so their points are added without a
  // barrier between them; the taps of the next points are formed before the
  // current ones are added.
  auto taps = [&](int n, int b0, int it, T& tr, T& ti, int& base) {
    const S st = srec[it < n ? b0 + it : 0];
    const T u = xl ? st.u0 : st.u1;
    T tap = cr[Q];
#pragma unroll
    for (int d = Q - 1; d >= 0; --d) tap = fma(tap, u, cr[d]);
    tr = xl ? tap * st.wr : tap;
    ti = T(0);
    if constexpr (CPLX) ti = xl ? tap * st.wi : T(0);
    base = st.base;
  };
  for (int phase = 0; phase < 4; ++phase) {
    for (int q0 = warp * P::PPW; q0 < P::PER_PHASE; q0 += P::NWARP * P::PPW) {
      const int q = q0 + half;
      int n = 0, b0 = 0;
      if (q < P::PER_PHASE) {
        const int qa = q % (P::NSB / 2), qb = q / (P::NSB / 2);
        const int sbi = (2 * qa + (phase & 1)) + P::NSB * (2 * qb + (phase >> 1));
        n = sb_count[sbi];
        b0 = sb_start[sbi];
      }
      int nh[P::PPW], nmax = 0;
#pragma unroll
      for (int h = 0; h < P::PPW; ++h) {
        nh[h] = __shfl_sync(0xffffffffu, n, h * P::HL);
        nmax = max(nmax, nh[h]);
      }
      T tr, ti;
      int base;
      taps(n, b0, 0, tr, ti, base);
      for (int it = 0; it < nmax; ++it) {
        T ntr, nti;
        int nbase;
        taps(n, b0, it + 1, ntr, nti, nbase);
#pragma unroll
        for (int h = 0; h < P::PPW; ++h) {
          if (it >= nh[h]) continue;  // warp-uniform
          const int src = h * P::HL;
          const int bh = __shfl_sync(0xffffffffu, base, src);
          const T kxr = __shfl_sync(0xffffffffu, tr, src + cc);
          T kxi = T(0);
          if constexpr (CPLX) kxi = __shfl_sync(0xffffffffu, ti, src + cc);
#pragma unroll
          for (int k = 0; k < P::NPASS; ++k) {
            const int row = k * P::R + rr;
            const T ky = __shfl_sync(0xffffffffu, tr, src + W + (row < W ? row : W - 1));
            if (cell_lane && row < W) {
              T* c = tile + (bh + lane_off + k * P::R * E) * NC;
              c[0] += kxr * ky;
              if constexpr (CPLX) c[1] += kxi * ky;
            }
          }
        }
        __syncwarp();
        tr = ntr;
        ti = nti;
        base = nbase;
      }
    }
    __syncthreads();
  }

  spread2d_flush<W, T, CPLX>(tile, wk, g, grid_real, grid_cplx);
}

// FP32 2D spreading of real weights, thread per point (4 <= W <= 8), with
// fixed-point shared accumulation: contributions are scaled by 2^21 over the
// power of two above the block's largest |weight| and rounded to integers by
// one FMA against 1.5 * 2^23 (round to nearest); a cell gets at most one
// contribution per point (<= kMaxSub < 2^10), so its 32-bit sum stays below
// 2^31 and is exact in any order, and an integer shared atomic add is one
// instruction.  A non-finite weight makes the block add NaN to the grid.
// One block of 256 threads per subproblem (Map: block -> subproblem, as for
// the phased kernel).  Staging: each thread maps its points (at most 3) to
// (tile offset of the footprint, u0, u1, weight) and ranks them by bank
// class, the tile offset mod 32 (a footprint cell at (r, c) lies at offset
// base + r P + c, so two points of different class never share a bank for the
// same (r, c)); the points are stored in class order, laid out so that round k
// of thread (warp w, lane l) reads the point at class-order position
// (8 l + w) R + k (R = rounds, ceil(cnt / 256)): consecutive lanes take points
// about a class apart, and each round's records are 32 consecutive entries.
// Accumulation: the thread evaluates its W x taps (times the scaled weight) and
// W y taps from the polynomial coefficients in the kernel parameters and adds
// the W^2 cells with 32-bit integer shared atomics.  The tile columns are
// shifted by LEFT so that the flush reads aligned groups of four cells with
// one 16-byte load.
template <int W>
struct Tpp2D {
  static constexpr int PAD = W / 2;
  static constexpr int E = kTile2D + W;                  // tile rows and used columns
  static constexpr int LEFT = (4 - PAD % 4) % 4;        // column shift: grid-aligned groups of four
  static constexpr int P = (E + LEFT + 3) / 4 * 4;       // row pitch (cells)
  static constexpr int NT = 256;
  static constexpr int RMAX = (kMaxSub + NT - 1) / NT;  // rounds per thread at most
};

template <int W>
__host__ __device__ constexpr size_t spread2d_tpp_smem_bytes() {
  using C = Tpp2D<W>;
  return sizeof(float4) * C::RMAX * C::NT + sizeof(int) * size_t(C::E) * C::P;
}

template <int W, typename Map>
__global__ void __launch_bounds__(256) spread2d_tpp_kernel(const Rec<2, float>* __restrict__ recs,
                                                           const float* __restrict__ weights, const Map map, Geom g,
                                                           const EsPoly<W, float> poly, float* grid_real) {
  using C = Tpp2D<W>;
  static_assert(W >= 4 && W <= 8, "kernel widths of the FP32 2D spread");
  static_assert(kMaxSub < 1024, "fixed-point sums of at most kMaxSub contributions below 2^21 fit 31 bits");
  constexpr int Q = EsPolyDeg<W>::Q;
  constexpr int PAD = C::PAD, E = C::E, LEFT = C::LEFT, P = C::P, NT = C::NT, RMAX = C::RMAX;
  constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound holds round(x) in its low mantissa bits
  constexpr int kRoundBits = 0x4B400000;  // the bits of kRound
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* srec = reinterpret_cast<float4*>(smem_raw);  // (tile offset bits, u0, u1, weight), round-major
  int* itile = reinterpret_cast<int*>(srec + RMAX * NT);
  __shared__ int cls_count[32], cls_start[32];
  __shared__ float s_red[8];

  TileWork<float> wk;
  if (!map.fetch(g, wk)) return;
  grid_real += wk.grid_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int start = wk.start, cnt = wk.cnt, org0 = wk.org0, org1 = wk.org1;
  const float uniform = wk.uniform;

  {
    int4* t4 = reinterpret_cast<int4*>(itile);
    for (int i = tid; i < E * P / 4; i += NT) t4[i] = make_int4(0, 0, 0, 0);
  }
  if (tid < 32) cls_count[tid] = 0;
  __syncthreads();
  float4 mine[RMAX];
  int key[RMAX];  // class << 16 | rank in class, or -1
  float wm = 0.0f;  // largest |weight| of this thread's points, NaN if one is not finite
#pragma unroll
  for (int k = 0; k < RMAX; ++k) {
    key[k] = -1;
    const int p = tid + k * NT;
    if (p >= cnt) continue;
    const Rec<2, float> r = recs[start + p];
    int c0, c1, c2;
    unpack_cell(2, r.cell, c0, c1, c2);
    float u0, u1;
    const int s0 = es_start<W, float>(r.f[0], u0);
    const int s1 = es_start<W, float>(r.f[1], u1);
    const int base = (c1 - org1 + s1 + PAD) * P + (c0 - org0 + s0 + PAD + LEFT);
    const float w = weights ? weights[r.idx] : uniform;
    wm = (isfinite(w) && !isnan(wm)) ? fmaxf(wm, fabsf(w)) : __int_as_float(0x7fc00000);
    mine[k] = make_float4(__int_as_float(base), u0, u1, w);
    const int cls = base & 31;
    key[k] = (cls << 16) | atomicAdd(&cls_count[cls], 1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float t = __shfl_xor_sync(0xffffffffu, wm, o);
    wm = (isnan(wm) || isnan(t)) ? __int_as_float(0x7fc00000) : fmaxf(wm, t);
  }
  if (lane == 0) s_red[warp] = wm;
  __syncthreads();
  if (warp == 0) {  // exclusive scan of the class counts
    const int v = cls_count[lane];
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    cls_start[lane] = inc - v;
  }
  __syncthreads();
  const int R = (cnt + NT - 1) / NT;
#pragma unroll
  for (int k = 0; k < RMAX; ++k) {
    if (key[k] < 0) continue;
    const int q = cls_start[key[k] >> 16] + (key[k] & 0xffff);  // class-order position
    const int s = q / R, kk = q - s * R;                          // thread slot s = 8 lane + warp, round kk
    srec[kk * NT + (s & 7) * 32 + (s >> 3)] = mine[k];
  }
  wm = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) wm = (isnan(wm) || isnan(s_red[k])) ? __int_as_float(0x7fc00000) : fmaxf(wm, s_red[k]);
  const bool bad_weight = isnan(wm);
  float scale = 1.0f, inv_scale = 1.0f;
  if (!bad_weight && wm > 0.0f) {
    int e = 0;
    frexpf(wm, &e);  // wm < 2^e
    e = max(-100, min(100, e));
    scale = ldexpf(1.0f, 21 - e);
    inv_scale = ldexpf(1.0f, e - 21);
  }
  __syncthreads();

  const int slot = lane * 8 + warp;
  for (int kk = 0; kk < R; ++kk) {
    if (slot * R + kk >= cnt) continue;
    const float4 st = srec[kk * NT + warp * 32 + lane];
    const float ws = st.w * scale;
    float tx[W], ty[W];
#pragma unroll
    for (int m = 0; m < W; ++m) {
      float a = poly.c[m][Q], b = poly.c[m][Q];
#pragma unroll
      for (int d = Q - 1; d >= 0; --d) {
        a = fmaf(a, st.y, poly.c[m][d]);
        b = fmaf(b, st.z, poly.c[m][d]);
      }
      tx[m] = a * ws;
      ty[m] = b;
    }
    int* cell = itile + __float_as_int(st.x);
#pragma unroll
    for (int r = 0; r < W; ++r)
#pragma unroll
      for (int c = 0; c < W; ++c) atomicAdd(cell + r * P + c, __float_as_int(fmaf(tx[c], ty[r], kRound)) - kRoundBits);
  }
  __syncthreads();

  // flush: aligned groups of four cells (grid x = org0 - PAD - LEFT + 4 j, nf0 % 4 == 0)
  constexpr int NG = P / 4;
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  const bool sole = cnt == wk.bin_range[1] - wk.bin_range[0] && nf0 % kTile2D == 0 && nf1 % kTile2D == 0;
  for (int i = tid; i < E * NG; i += NT) {
    const int ty = i / NG, j = i - ty * NG;
    const int4 iv = *reinterpret_cast<const int4*>(itile + ty * P + 4 * j);
    if ((iv.x | iv.y | iv.z | iv.w) == 0) continue;
    const int tc0 = 4 * j - LEFT;
    const int gy = wrap_index(org1 - PAD + ty, nf1);
    const int gx = wrap_index(org0 - PAD + tc0, nf0);
    float4* dst = reinterpret_cast<float4*>(grid_real + int64_t(gy) * nf0 + gx);
    const float4 val = make_float4(float(iv.x) * inv_scale, float(iv.y) * inv_scale, float(iv.z) * inv_scale,
                                   float(iv.w) * inv_scale);
    if (sole && ty >= W && ty < kTile2D && tc0 >= W && tc0 + 4 <= kTile2D) *dst = val;
    else atomicAdd(dst, val);
  }
  if (bad_weight && tid == 0)
    atomicAdd(grid_real + int64_t(wrap_index(org1, nf1)) * nf0 + wrap_index(org0, nf0), __int_as_float(0x7fc00000));
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

// 3D spreading of real strengths, w <= 8: one warp per point, so that each
// shared-memory atomic instruction covers a 4-row x 7-column block of one
// plane of the footprint (two passes of rows per plane, w planes).  The tile's
// row pitch tw0p is a multiple of 8 but not of 16, which puts the 4 rows of a
// pass on disjoint bank ranges: every atomic instruction is free of bank
// conflicts.  Lane l < 3w evaluates tap l % w of axis l / w (its coefficient
// row is loaded into registers once) and the others read it by shuffle.
//
// FP32 accumulates in 32-bit fixed point: a shared-memory float atomic add is
// a compare-and-swap loop, an integer one a single instruction.  The block
// scales its contributions by s = 2^21 / 2^e with max |weight| < 2^e, so each
// is below 2^21 in magnitude (|taps| <= 1) and is rounded to an integer by one
// FMA against 1.5 * 2^23 (round to nearest: the same half-unit error as one
// float addition of a value of that size); a cell receives at most one
// contribution per point of the subproblem (at most kMaxSub = 640 < 2^10), so
// its sum stays below 2^31 and is exact.  The flush adds sum / s to the grid.
// A non-finite weight makes the block add NaN to the grid.  FP64 keeps double
// atomics.
template <int W, typename T>
__global__ void __launch_bounds__(256) spread3d_warp_kernel(const Rec<3, T>* __restrict__ recs,
                                                            const T* __restrict__ weights, T uniform,
                                                            const int* __restrict__ sub_bin,
                                                            const int* __restrict__ sub_start,
                                                            const int* __restrict__ sub_count,
                                                            const int* __restrict__ num_sub, Geom g,
                                                            const EsPoly<W, T> poly, int tw0p, T* grid_real) {
  static_assert(W <= 8, "one pass covers 4 rows of at most 8 columns");
  static_assert(kMaxSub < 1024, "fixed-point sums of at most kMaxSub contributions below 2^21 fit 31 bits");
  constexpr bool FIXED = sizeof(T) == 4;
  constexpr int Q = EsPolyDeg<W>::Q;
  constexpr int PAD = W / 2;
  constexpr float kRound = 12582912.0f;  // 1.5 * 2^23: x + kRound holds round(x) in its low mantissa bits
  constexpr int kRoundBits = 0x4B400000;  // the bits of kRound
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* tile = reinterpret_cast<T*>(smem_raw);
  int* itile = reinterpret_cast<int*>(smem_raw);
  __shared__ float s_red[8];
  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  const int tw0 = g.tw[0], tw1 = g.tw[1], tw2 = g.tw[2];
  const int plane = tw1 * tw0p;
  for (int i = threadIdx.x; i < plane * tw2; i += blockDim.x) tile[i] = T(0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int tdim = lane / W, tm = lane - (lane / W) * W;  // this lane's tap (tdim < 3 for lane < 3W)
  T cf[Q + 1];
#pragma unroll
  for (int d = 0; d <= Q; ++d) {
    T v = T(0);
#pragma unroll
    for (int m = 0; m < W; ++m)
      if (m == tm) v = poly.c[m][d];
    cf[d] = v;
  }
  // lane (r_in, c_in) covers column c_in of footprint rows r_in and r_in + 4; lanes outside the
  // footprint add zero to a cell that no other lane of the instruction touches (column c_in < 8 of
  // the padded row, or row r_in again for the second pass), so the atomics need no branch
  const int r_in = lane >> 3, c_in = lane & 7;
  const bool col_ok = c_in < W && r_in < W, row1_ok = r_in + 4 < W;
  const int r_eff = r_in < W ? r_in : 0;
  const int row1_off = row1_ok ? 4 * tw0p : 0;

  const int bin = sub_bin[sub];
  const int start = sub_start[sub], cnt = sub_count[sub];
  float scale = 1.0f, inv_scale = 1.0f;
  bool bad_weight = false;
  if constexpr (FIXED) {  // the block's largest |weight| (NaN if a weight is not finite)
    float wm = 0.0f;
    for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
      const float w = weights ? float(weights[recs[start + p].idx]) : float(uniform);
      wm = (isfinite(w) && !isnan(wm)) ? fmaxf(wm, fabsf(w)) : __int_as_float(0x7fc00000);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float t = __shfl_xor_sync(0xffffffffu, wm, o);
      wm = (isnan(wm) || isnan(t)) ? __int_as_float(0x7fc00000) : fmaxf(wm, t);
    }
    if (lane == 0) s_red[warp] = wm;
    __syncthreads();
    wm = 0.0f;
    for (int k = 0; k < nw; ++k) wm = (isnan(wm) || isnan(s_red[k])) ? __int_as_float(0x7fc00000) : fmaxf(wm, s_red[k]);
    bad_weight = isnan(wm);
    if (!bad_weight && wm > 0.0f) {
      int e = 0;
      frexpf(wm, &e);  // wm < 2^e
      e = max(-100, min(100, e));
      scale = ldexpf(1.0f, 21 - e);
      inv_scale = ldexpf(1.0f, e - 21);
    }
  } else {
    __syncthreads();  // the zeroed tile
  }

  const int bx = bin % g.nb[0];
  const int brem = bin / g.nb[0];
  const int by = brem % g.nb[1];
  const int bz = brem / g.nb[1];
  const int org0 = bx * g.tile[0], org1 = by * g.tile[1], org2 = bz * g.tile[2];
  for (int p = warp; p < cnt; p += nw) {
    const Rec<3, T> rec = recs[start + p];
    int c0, c1, c2;
    unpack_cell(3, rec.cell, c0, c1, c2);
    T sr = weights ? weights[rec.idx] : uniform;
    if constexpr (FIXED) sr *= scale;
    T u0, u1, u2;
    const int s0 = es_start<W, T>(rec.f[0], u0);
    const int s1 = es_start<W, T>(rec.f[1], u1);
    const int s2 = es_start<W, T>(rec.f[2], u2);
    const T u = tdim == 0 ? u0 : (tdim == 1 ? u1 : u2);
    T tap = cf[Q];
#pragma unroll
    for (int d = Q - 1; d >= 0; --d) tap = fma(tap, u, cf[d]);
    const T kx = __shfl_sync(0xffffffffu, tap, col_ok ? c_in : 0);
    const T ky0 = __shfl_sync(0xffffffffu, tap, W + (r_in < W ? r_in : 0));
    const T ky1 = __shfl_sync(0xffffffffu, tap, W + (row1_ok ? r_in + 4 : 0));
    const T a0 = col_ok ? sr * kx * ky0 : T(0), a1 = (col_ok && row1_ok) ? sr * kx * ky1 : T(0);
    const int l0 = c0 - org0 + s0 + PAD, l1 = c1 - org1 + s1 + PAD, l2 = c2 - org2 + s2 + PAD;
    const int base0 = (l2 * tw1 + l1 + r_eff) * tw0p + l0 + c_in;
#pragma unroll
    for (int m2 = 0; m2 < W; ++m2) {
      const T kz = __shfl_sync(0xffffffffu, tap, 2 * W + m2);
      if constexpr (FIXED) {
        atomicAdd(&itile[base0 + m2 * plane], __float_as_int(fmaf(a0, kz, kRound)) - kRoundBits);
        atomicAdd(&itile[base0 + m2 * plane + row1_off], __float_as_int(fmaf(a1, kz, kRound)) - kRoundBits);
      } else {
        atomicAdd(&tile[base0 + m2 * plane], a0 * kz);
        atomicAdd(&tile[base0 + m2 * plane + row1_off], a1 * kz);
      }
    }
  }
  __syncthreads();
  // flush (flush_tile with the padded pitch)
  const int o0 = org0 - PAD, o1 = org1 - PAD, o2 = org2 - PAD;
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  for (int i = threadIdx.x; i < tw0 * tw1 * tw2; i += blockDim.x) {
    const int i0 = i % tw0;
    const int r = i / tw0;
    const int i1 = r % tw1;
    const int i2 = r / tw1;
    T v;
    if constexpr (FIXED) v = T(itile[(i2 * tw1 + i1) * tw0p + i0]) * T(inv_scale);
    else v = tile[(i2 * tw1 + i1) * tw0p + i0];
    if (v != T(0)) {
      const int64_t gi = (int64_t(wrap_index(o2 + i2, nf2)) * nf1 + wrap_index(o1 + i1, nf1)) * nf0 +
                         wrap_index(o0 + i0, nf0);
      atomicAdd(grid_real + gi, v);
    }
  }
  if (bad_weight && threadIdx.x == 0) {
    const int64_t gi = (int64_t(wrap_index(org2, nf2)) * nf1 + wrap_index(org1, nf1)) * nf0 + wrap_index(org0, nf0);
    atomicAdd(grid_real + gi, T(__int_as_float(0x7fc00000)));
  }
}

// FP32 3D spreading of real weights, thread per point (W <= 8): the 2D
// thread-per-point scheme (spread2d_tpp_kernel) on a tw0 x tw1 x tw2 tile.
// Staging ranks the block's points by bank class (tile offset of the
// footprint mod 32) and stores them round-major in class order; each thread
// evaluates its 3W taps from the polynomial coefficients in the kernel
// parameters (the weight folded into the x taps) and adds the W^3 cells with
// 32-bit integer shared atomics (fixed point as in the 2D kernel).  Row
// pitch px = tw0 + LEFT rounded up to four cells, LEFT chosen so that the
// flush reads grid-aligned groups of four cells with one 16-byte load.
template <int W>
struct Tpp3D {
  static constexpr int PAD = W / 2;
  static constexpr int LEFT = (4 - PAD % 4) % 4;
  static constexpr int NT = 256;
  static constexpr int RMAX = (kMaxSub + NT - 1) / NT;
};

inline int spread3d_tpp_pitch(int tw0, int w) { return (tw0 + (4 - (w / 2) % 4) % 4 + 3) / 4 * 4; }

template <int W>
inline size_t spread3d_tpp_smem_bytes(const Geom& g) {
  using C = Tpp3D<W>;
  return (sizeof(float4) + sizeof(float)) * C::RMAX * C::NT +
         sizeof(int) * size_t(spread3d_tpp_pitch(g.tw[0], W)) * g.tw[1] * g.tw[2];
}

template <int W>
__global__ void __launch_bounds__(256) spread3d_tpp_kernel(const Rec<3, float>* __restrict__ recs,
                                                           const float* __restrict__ weights, float uniform,
                                                           const int* __restrict__ sub_bin,
                                                           const int* __restrict__ sub_start,
                                                           const int* __restrict__ sub_count,
                                                           const int* __restrict__ num_sub,
                                                           const int* __restrict__ bin_start, Geom g,
                                                           const EsPoly<W, float> poly, int px,
                                                           float* __restrict__ grid_real) {
  using C = Tpp3D<W>;
  static_assert(W <= 8, "kernel widths of the FP32 3D spread");
  static_assert(kMaxSub < 1024, "fixed-point sums of at most kMaxSub contributions below 2^21 fit 31 bits");
  constexpr int Q = EsPolyDeg<W>::Q;
  constexpr int PAD = C::PAD, LEFT = C::LEFT, NT = C::NT, RMAX = C::RMAX;
  constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound holds round(x) in its low mantissa bits
  constexpr int kRoundBits = 0x4B400000;  // the bits of kRound
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* srec = reinterpret_cast<float4*>(smem_raw);  // (tile offset bits, u0, u1, u2), round-major
  float* sw = reinterpret_cast<float*>(srec + RMAX * NT);
  int* itile = reinterpret_cast<int*>(sw + RMAX * NT);
  __shared__ int cls_count[32], cls_start[32];
  __shared__ float s_red[8];

  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int bin = sub_bin[sub];
  const int start = sub_start[sub], cnt = sub_count[sub];
  const int tw1 = g.tw[1], tw2 = g.tw[2];
  const int plane = tw1 * px;
  const int cells = plane * tw2;
  const int bx = bin % g.nb[0];
  const int brem = bin / g.nb[0];
  const int by = brem % g.nb[1];
  const int bz = brem / g.nb[1];
  const int org0 = bx * g.tile[0], org1 = by * g.tile[1], org2 = bz * g.tile[2];

  {
    int4* t4 = reinterpret_cast<int4*>(itile);
    for (int i = tid; i < cells / 4; i += NT) t4[i] = make_int4(0, 0, 0, 0);
  }
  if (tid < 32) cls_count[tid] = 0;
  __syncthreads();
  float4 mine[RMAX];
  float mw[RMAX];
  int key[RMAX];  // class << 16 | rank in class, or -1
  float wm = 0.0f;
#pragma unroll
  for (int k = 0; k < RMAX; ++k) {
    key[k] = -1;
    const int p = tid + k * NT;
    if (p >= cnt) continue;
    const Rec<3, float> r = recs[start + p];
    int c0, c1, c2;
    unpack_cell(3, r.cell, c0, c1, c2);
    float u0, u1, u2;
    const int s0 = es_start<W, float>(r.f[0], u0);
    const int s1 = es_start<W, float>(r.f[1], u1);
    const int s2 = es_start<W, float>(r.f[2], u2);
    const int base = ((c2 - org2 + s2 + PAD) * tw1 + (c1 - org1 + s1 + PAD)) * px + (c0 - org0 + s0 + PAD + LEFT);
    const float w = weights ? weights[r.idx] : uniform;
    wm = (isfinite(w) && !isnan(wm)) ? fmaxf(wm, fabsf(w)) : __int_as_float(0x7fc00000);
    mine[k] = make_float4(__int_as_float(base), u0, u1, u2);
    mw[k] = w;
    const int cls = base & 31;
    key[k] = (cls << 16) | atomicAdd(&cls_count[cls], 1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float t = __shfl_xor_sync(0xffffffffu, wm, o);
    wm = (isnan(wm) || isnan(t)) ? __int_as_float(0x7fc00000) : fmaxf(wm, t);
  }
  if (lane == 0) s_red[warp] = wm;
  __syncthreads();
  if (warp == 0) {  // exclusive scan of the class counts
    const int v = cls_count[lane];
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    cls_start[lane] = inc - v;
  }
  __syncthreads();
  const int R = (cnt + NT - 1) / NT;
#pragma unroll
  for (int k = 0; k < RMAX; ++k) {
    if (key[k] < 0) continue;
    const int q = cls_start[key[k] >> 16] + (key[k] & 0xffff);  // class-order position
    const int s = q / R, kk = q - s * R;                          // thread slot s = 8 lane + warp, round kk
    const int at = kk * NT + (s & 7) * 32 + (s >> 3);
    srec[at] = mine[k];
    sw[at] = mw[k];
  }
  wm = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) wm = (isnan(wm) || isnan(s_red[k])) ? __int_as_float(0x7fc00000) : fmaxf(wm, s_red[k]);
  const bool bad_weight = isnan(wm);
  float scale = 1.0f, inv_scale = 1.0f;
  if (!bad_weight && wm > 0.0f) {
    int e = 0;
    frexpf(wm, &e);  // wm < 2^e
    e = max(-100, min(100, e));
    scale = ldexpf(1.0f, 21 - e);
    inv_scale = ldexpf(1.0f, e - 21);
  }
  __syncthreads();

  const int slot = lane * 8 + warp;
  for (int kk = 0; kk < R; ++kk) {
    if (slot * R + kk >= cnt) continue;
    const int at = kk * NT + warp * 32 + lane;
    const float4 st = srec[at];
    const float ws = sw[at] * scale;
    float tx[W], ty[W], tz[W];
#pragma unroll
    for (int m = 0; m < W; ++m) {
      float a = poly.c[m][Q], b = poly.c[m][Q], c = poly.c[m][Q];
#pragma unroll
      for (int d = Q - 1; d >= 0; --d) {
        a = fmaf(a, st.y, poly.c[m][d]);
        b = fmaf(b, st.z, poly.c[m][d]);
        c = fmaf(c, st.w, poly.c[m][d]);
      }
      tx[m] = a * ws;
      ty[m] = b;
      tz[m] = c;
    }
    const int base = __float_as_int(st.x);
#pragma unroll
    for (int z = 0; z < W; ++z) {
#pragma unroll
      for (int y = 0; y < W; ++y) {
        int* row = itile + base + z * plane + y * px;
        const float yz = ty[y] * tz[z];
#pragma unroll
        for (int x = 0; x < W; ++x) atomicAdd(row + x, __float_as_int(fmaf(tx[x], yz, kRound)) - kRoundBits);
      }
    }
  }
  __syncthreads();

  // flush: grid-aligned groups of four cells along x (nf0 % 4 == 0, tile[0] % 4 == 0)
  const int o0 = org0 - PAD - LEFT, o1 = org1 - PAD, o2 = org2 - PAD;
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  const int ng = px / 4;
  const bool sole = cnt == bin_start[bin + 1] - bin_start[bin] && nf0 % g.tile[0] == 0 &&
                    nf1 % g.tile[1] == 0 && nf2 % g.tile[2] == 0;
  for (int i = tid; i < tw2 * tw1 * ng; i += NT) {
    const int j = i % ng;
    const int r = i / ng;
    const int i1 = r % tw1;
    const int i2 = r / tw1;
    const int4 iv = *reinterpret_cast<const int4*>(itile + (i2 * tw1 + i1) * px + 4 * j);
    if ((iv.x | iv.y | iv.z | iv.w) == 0) continue;
    const int tc0 = 4 * j - LEFT;
    const int64_t gi = (int64_t(wrap_index(o2 + i2, nf2)) * nf1 + wrap_index(o1 + i1, nf1)) * nf0 +
                       wrap_index(o0 + 4 * j, nf0);
    float4* dst = reinterpret_cast<float4*>(grid_real + gi);
    const float4 val = make_float4(float(iv.x) * inv_scale, float(iv.y) * inv_scale, float(iv.z) * inv_scale,
                                   float(iv.w) * inv_scale);
    if (sole && i1 >= W && i1 < g.tile[1] && i2 >= W && i2 < g.tile[2] && tc0 >= W && tc0 + 4 <= g.tile[0])
      *dst = val;
    else
      atomicAdd(dst, val);
  }
  if (bad_weight && tid == 0) {
    const int64_t gi = (int64_t(wrap_index(org2, nf2)) * nf1 + wrap_index(org1, nf1)) * nf0 + wrap_index(org0, nf0);
    atomicAdd(grid_real + gi, __int_as_float(0x7fc00000));
  }
}

// Row pitch of spread3d_warp_kernel's tile: a multiple of 8, not of 16, with
// room for the 8 - w columns past a footprint row that the lanes outside the
// footprint touch (>= tw0 + 8 - w).
inline int spread3d_pitch(int tw0, int w) {
  int p = (tw0 + std::max(0, 8 - w) + 7) / 8 * 8;
  if (p % 16 == 0) p += 8;
  return p;
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

// Tile geometry of the 2D interpolation: rows org1 - W/2 .. (64 + W rows);
// columns start at org0 - XPAD, XPAD = W/2 rounded up to even, and a row
// holds TWX (even) cells, so that with 8- or 16-byte cells a tile row is a
// whole number of 16-byte units and starts on a 16-byte boundary of the fine
// grid (what a tensor copy of the tile needs).
template <int W>
struct Interp2D {
  static constexpr int PAD = W / 2;
  static constexpr int XPAD = (PAD + 1) & ~1;
  static constexpr int TWY = kTile2D + W;
  static constexpr int TWX = (kTile2D + W + (XPAD - PAD) + 1) & ~1;
};

template <int W, typename T>
__host__ __device__ constexpr size_t interp2d_smem_bytes() {
  // + 128: the tile is placed on a 128-byte boundary for the tensor copy
  return 128 + sizeof(cplx_t<T>) * Interp2D<W>::TWX * Interp2D<W>::TWY + sizeof(uint16_t) * kMaxSub;
}

// Points per thread of a 2D tile block (256 threads, at most kMaxSub points).
constexpr int kTilePtsPerThread = (kMaxSub + 255) / 256;

// A block whose first bounded wait for its tile copy (tile_wait_polls_setting()
// mbarrier polls) runs out waits again, bounded by kTileWaitNs of the global
// timer, before it fails the evaluation.
constexpr uint64_t kTileWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Waits for phase `parity` of the barrier for at most `polls` polls (none when
// polls is 0: the wait runs out at once).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int polls) {
  for (int i = 0; i < polls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Waits for phase `parity` of the barrier for at most `ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait_timed(uint64_t* bar, unsigned parity, uint64_t ns) {
  const uint64_t t0 = global_ns();
  do {
    if (mbar_try_wait(bar, parity)) return true;
  } while (global_ns() - t0 < ns);
  return mbar_try_wait(bar, parity);
}
// 2D tensor copy global -> shared (x innermost, in elements of the map),
// completing on `bar` with its byte count.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// 2D interpolation: one block per subproblem stages the tile (+ halo) of the
// field in shared memory, then one thread per point sums its w x w taps.
// With a tensor map of the field (single pattern, power-of-64 grids), a tile
// that needs no periodic wrap is copied by one tensor copy, issued before
// the block classifies its points so the two overlap; edge tiles are read
// with plain loads.
//
// Every tap address of a point is its footprint's first cell `base` plus an
// offset that is the same for all points, so a group of lanes served by one
// shared-memory wavefront (16 lanes for 8-byte cells, 8 for 16-byte cells)
// reads without bank conflicts when the bases of its points are distinct
// modulo the group size.  The block therefore buckets its points by
// base mod G and lane c of every group takes points of class c only.
template <int W, typename T, typename Map>
__global__ void __launch_bounds__(256) interp2d_tile_kernel(const Rec<2, T>* __restrict__ recs,
                                                            const T* __restrict__ weights,
                                                            const __grid_constant__ Map map, Geom g,
                                                            const EsPoly<W, T> poly,
                                                            const cplx_t<T>* __restrict__ field, int mode, double* grad,
                                                            double2* out2, int accumulate, const GradScale gs) {
  using IP = Interp2D<W>;
  constexpr int PAD = IP::PAD, XPAD = IP::XPAD, TWX = IP::TWX, TWY = IP::TWY;
  constexpr int G = 128 / int(sizeof(cplx_t<T>));  // lanes per wavefront = bank classes
  extern __shared__ unsigned char smem_ip[];
  __shared__ __align__(8) uint64_t tile_bar;
  cplx_t<T>* tile = reinterpret_cast<cplx_t<T>*>(smem_ip + ((128u - (smem_addr(smem_ip) & 127u)) & 127u));
  uint16_t* order = reinterpret_cast<uint16_t*>(tile + TWX * TWY);  // points grouped by class
  __shared__ int cls_count[G], cls_start[G];
  TileWork<T> wk;
  if (!map.fetch(g, wk)) return;
  const int start = wk.start, cnt = wk.cnt, org0 = wk.org0, org1 = wk.org1;
  const T uniform = wk.uniform;
  const bool bad = map.nonfinite(wk);
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  field += wk.grid_off;
  const int tid = threadIdx.x;
  const CUtensorMap* tm = map.tile_tmap();
  const bool use_tma = tm != nullptr && org0 >= XPAD && org0 - XPAD + TWX <= nf0 && org1 >= PAD &&
                       org1 - PAD + TWY <= nf1;
  if (tid < G) cls_count[tid] = 0;
  if (use_tma && tid == 0) mbar_init(&tile_bar, 1);
  __syncthreads();
  if (use_tma) {
    if (tid == 0) {
      mbar_expect_tx(&tile_bar, unsigned(sizeof(cplx_t<T>) * TWX * TWY));
      tma_load_2d(tile, tm, 2 * (org0 - XPAD), org1 - PAD, &tile_bar);
    }
  } else {
    // tile read in batches of 4 loads per thread so that their latencies overlap
    constexpr int BT = 4;
    const int nthr = blockDim.x;
    for (int i0 = tid; i0 < TWX * TWY; i0 += BT * nthr) {
      cplx_t<T> v[BT];
#pragma unroll
      for (int b = 0; b < BT; ++b) {
        const int i = i0 + b * nthr;
        if (i < TWX * TWY) {
          const int x = i % TWX, y = i / TWX;
          v[b] = field[int64_t(wrap_index(org1 - PAD + y, nf1)) * nf0 + wrap_index(org0 - XPAD + x, nf0)];
        }
      }
#pragma unroll
      for (int b = 0; b < BT; ++b)
        if (i0 + b * nthr < TWX * TWY) tile[i0 + b * nthr] = v[b];
    }
  }
  // class and rank in class of this thread's points (p = tid + 256 k), kept
  // in registers until the class starts are known
  constexpr int PPT = kTilePtsPerThread;
  int code[PPT];
  {
    Rec<2, T> r[PPT];
#pragma unroll
    for (int k = 0; k < PPT; ++k)
      if (tid + 256 * k < cnt) r[k] = recs[start + tid + 256 * k];
#pragma unroll
    for (int k = 0; k < PPT; ++k) {
      code[k] = -1;
      if (tid + 256 * k >= cnt) continue;
      int c0, c1, c2;
      unpack_cell(2, r[k].cell, c0, c1, c2);
      T u;
      const int l0 = c0 - org0 + es_start<W, T>(r[k].f[0], u) + XPAD;
      const int l1 = c1 - org1 + es_start<W, T>(r[k].f[1], u) + PAD;
      const int cls = (l1 * TWX + l0) & (G - 1);
      code[k] = (cls << 12) | atomicAdd(&cls_count[cls], 1);
    }
  }
  if (use_tma) {
    // Every thread polls the copy's barrier, bounded.  If any thread's polls
    // run out, the block records STATUS_TILE_RETRY and every thread waits
    // again, bounded by time; the copy normally lands then and the block goes
    // on with a complete tile.  A copy that has still not landed fails the
    // evaluation: STATUS_TIMEOUT, a NaN energy and NaN results for the
    // block's points.  The block then returns with its copy possibly in
    // flight, so once STATUS_TIMEOUT is raised no result of the evaluation is
    // to be trusted, which the NaN energy makes visible to every caller.
    const bool ok = mbar_wait_bounded(&tile_bar, 0, map.wait_polls());
    if (__syncthreads_or(!ok)) {
      if (tid == 0)
        if (int* st = map.err_status()) raise_status(st, STATUS_TILE_RETRY);
      const bool ok2 = mbar_wait_timed(&tile_bar, 0, kTileWaitNs);
      if (__syncthreads_or(!ok2)) {
        const T nan = T(__longlong_as_double(0x7ff8000000000000ULL));
        if (tid == 0) {
          if (int* st = map.err_status()) raise_status(st, STATUS_TIMEOUT);
          if (double* e = map.fail_energy()) *e = double(nan);
        }
        for (int p = tid; p < cnt; p += blockDim.x)
          interp_store<2, T>(mode, recs[start + p].idx, T(1), nan, nan, nan, true, grad, out2, accumulate, gs);
        return;
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int c = 0; c < G; ++c) {
      cls_start[c] = acc;
      acc += cls_count[c];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PPT; ++k)
    if (code[k] >= 0) order[cls_start[code[k] >> 12] + (code[k] & 0xfff)] = uint16_t(tid + 256 * k);
  __syncthreads();
  const int cls = tid % G, grp = tid / G, ngrp = int(blockDim.x) / G;
  const int n_c = cls_count[cls];
  const uint16_t* mine = order + cls_start[cls];
  // the next record is loaded while the current point is interpolated
  Rec<2, T> nxt;
  if (grp < n_c) nxt = recs[start + mine[grp]];
  for (int j = grp; j < n_c; j += ngrp) {
    const Rec<2, T> r = nxt;
    if (j + ngrp < n_c) nxt = recs[start + mine[j + ngrp]];
    int c0, c1, c2;
    unpack_cell(2, r.cell, c0, c1, c2);
    T k0[W], k1[W];
    const int s0 = es_taps<W, T>(r.f[0], poly, k0);
    const int s1 = es_taps<W, T>(r.f[1], poly, k1);
    const int l0 = c0 - org0 + s0 + XPAD, l1 = c1 - org1 + s1 + PAD;
    T vr = 0, vi = 0;
#pragma unroll
    for (int m1 = 0; m1 < W; ++m1) {
      const cplx_t<T>* rowp = tile + (l1 + m1) * TWX + l0;
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
// directly from HBM/L2 (neighbouring threads share footprints).  With NF == 2
// the second field is real: G values of T after the G complex cells of the
// first (the 3D z field, whose type-2 transform is real).
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
    T v0r = 0, v0i = 0, v1r = 0;
    const T* __restrict__ real2 = reinterpret_cast<const T*>(fields + G);  // NF == 2: the real second field
    const int nz = (D == 3) ? W : 1;
    const int ny = (D >= 2) ? W : 1;
    for (int m2 = 0; m2 < nz; ++m2) {
      const int iz = (D == 3) ? wrap_index(c2 + s2 + m2, nf2) : 0;
      const T wz = (D == 3) ? k2[m2] : T(1);
#pragma unroll
      for (int m1 = 0; m1 < ny; ++m1) {
        const int iy = (D >= 2) ? wrap_index(c1 + s1 + m1, nf1) : 0;
        const T wy = (D >= 2) ? wz * k1[m1] : T(1);
        const int64_t row = (int64_t(iz) * nf1 + iy) * nf0;
        const cplx_t<T>* rowp = fields + row;
        T rr = 0, ri = 0, qr = 0;
#pragma unroll
        for (int m0 = 0; m0 < W; ++m0) {
          const cplx_t<T> a = __ldg(rowp + ix[m0]);
          rr += a.x * k0[m0];
          ri += a.y * k0[m0];
          if (NF == 2) qr += __ldg(real2 + row + ix[m0]) * k0[m0];
        }
        v0r += wy * rr;
        v0i += wy * ri;
        if (NF == 2) v1r += wy * qr;
      }
    }
    const T wgt = (mode == INTERP_GRAD) ? (weights ? weights[rec.idx] : uniform) : T(1);
    interp_store<D, T>(mode, rec.idx, wgt, v0r, v0i, v1r, bad, grad, out2, accumulate, gs);
  }
}

// 3D interpolation: one block per subproblem stages its bin's tile (+ halo)
// of one field at a time in shared memory and one thread per point sums its
// w^3 taps from it (instead of gathering them from L2).  As in the 2D kernel,
// every tap address of a point is its footprint's first cell plus an offset
// common to all points, so the block buckets its points by that cell modulo
// the lanes one shared-memory wavefront serves (16 for FP32 complex cells)
// and lane c of every group of 16 takes points of class c only: the reads of
// a group fall on distinct banks.  With two fields, each point's sums of the
// first are kept in shared memory for the second.
//
// Tile layout: z, y, x with x fastest; x starts XO = pad + (pad & 1) cells
// before the bin (so that the first float is a multiple of 4: the bin origin
// is even) and the row holds TXP cells (tile + w rounded up to even, plus the
// extra cell), y and z start pad cells before it.  A tile that needs no
// periodic wrap arrives by one 4D tensor copy per field (x in floats, y, z,
// field; issued for the first field before the block classifies its points,
// so copy and classification overlap); edge tiles use plain loads.
//
// With two fields (3D NUwU) the second is real (the z gradient field): its tile
// holds T per cell, x starts XR = pad rounded up to a multiple of 4 cells before
// the bin (16-byte aligned copies for FP32), rows of TXR cells (a multiple of
// 4), copied by a 3D tensor map of the real grid; its pass regroups the points
// by tile offset mod 32, so each warp's 4-byte reads fall on 32 banks.
template <int W>
struct Interp3D {
  static constexpr int PAD = W / 2;
  static constexpr int XO = PAD + (PAD & 1);
  static constexpr int XR = (PAD + 3) & ~3;
  __host__ __device__ static constexpr int txp(int tile0) { return (tile0 + W + (PAD & 1) + 1) & ~1; }
  __host__ __device__ static constexpr int txr(int tile0) { return (tile0 + W + (XR - PAD) + 3) & ~3; }
};

// Per-launch data of the 3D tile kernel's tensor copies (a __grid_constant__
// parameter, so the map's address is usable by the copy).
struct Tile3Copy {
  CUtensorMap tmap;   // the complex field as (2 nf0 floats, nf1, nf2, 1)
  CUtensorMap tmap2;  // the real second field as (nf0, nf1, nf2)
  int has_tmap = 0;
  int has_tmap2 = 0;
  int polls = 0;      // first bounded wait for a copy (mbarrier polls)
  double* energy = nullptr;  // the evaluation's energy, made NaN if a copy never lands (may be null)
};

template <int W, typename T, int NF>
__host__ __device__ constexpr size_t interp3d_extra_bytes() {
  return 128 + (NF == 2 ? sizeof(cplx_t<T>) * kMaxSub : 0) + sizeof(uint16_t) * kMaxSub * (NF == 2 ? 2 : 1);
}

// 3D tensor copy global -> shared (x innermost), completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// 4D tensor copy global -> shared (x innermost, in elements of the map),
// completing on `bar` with its byte count.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, int x, int y, int z, int f,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_addr(bar))
      : "memory");
}

template <int W, typename T, int NF>
__global__ void __launch_bounds__(256, 3) interp3d_tile_kernel(
    const Rec<3, T>* __restrict__ recs, const T* __restrict__ weights, T uniform, const int* __restrict__ sub_bin,
    const int* __restrict__ sub_start, const int* __restrict__ sub_count, const int* __restrict__ num_sub, Geom g,
    const EsPoly<W, T> poly, const cplx_t<T>* __restrict__ fields, int mode, double* grad, double2* out2,
    int accumulate, const int* __restrict__ status, const GradScale gs, const __grid_constant__ Tile3Copy cp) {
  using IP = Interp3D<W>;
  constexpr int PAD = IP::PAD, XO = IP::XO, XR = IP::XR;
  constexpr int PPT = (kMaxSub + 255) / 256;
  constexpr int G = 128 / int(sizeof(cplx_t<T>));  // lanes per wavefront = bank classes (complex cells)
  constexpr int G2 = 32;                            // bank classes of the real field's 4-byte cells
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t tile_bar;
  __shared__ int cls_count[G], cls_start[G], cls2_count[G2], cls2_start[G2];
  const int sub = blockIdx.x;
  if (sub >= *num_sub) return;
  const int bin = sub_bin[sub], start = sub_start[sub], cnt = sub_count[sub];
  const int bx = bin % g.nb[0], rb = bin / g.nb[0];
  const int by = rb % g.nb[1], bz = rb / g.nb[1];
  const int org0 = bx * g.tile[0], org1 = by * g.tile[1], org2 = bz * g.tile[2];
  const int TX = IP::txp(g.tile[0]), TXR = IP::txr(g.tile[0]), TY = g.tile[1] + W, TZ = g.tile[2] + W;
  const int ncell = TX * TY * TZ, ncell2 = TXR * TY * TZ;
  cplx_t<T>* tile = reinterpret_cast<cplx_t<T>*>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
  T* rtile = reinterpret_cast<T*>(tile);  // the real field's tile (same buffer, second pass)
  const int tile_cells = (NF == 2 && ncell2 * int(sizeof(T)) > ncell * int(sizeof(cplx_t<T>)))
                             ? (ncell2 * int(sizeof(T)) + int(sizeof(cplx_t<T>)) - 1) / int(sizeof(cplx_t<T>))
                             : ncell;
  cplx_t<T>* first = tile + tile_cells;  // NF == 2: each point's sums of the first field
  uint16_t* order = reinterpret_cast<uint16_t*>(first + (NF == 2 ? kMaxSub : 0));  // points grouped by class
  uint16_t* order2 = order + kMaxSub;  // NF == 2: points grouped by real-tile class
  const bool bad = status != nullptr && ((*status) & STATUS_NONFINITE_INPUT);
  const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
  const int tid = threadIdx.x;
  const bool yz_in = org1 >= PAD && org1 - PAD + TY <= nf1 && org2 >= PAD && org2 - PAD + TZ <= nf2;
  const bool use_tma = cp.has_tmap && org0 >= XO && org0 - XO + TX <= nf0 && yz_in;
  const bool use_tma2 = NF == 2 && cp.has_tmap2 && org0 >= XR && org0 - XR + TXR <= nf0 && yz_in;
  const unsigned tile_bytes = unsigned(sizeof(cplx_t<T>)) * unsigned(ncell);
  const unsigned tile2_bytes = unsigned(sizeof(T)) * unsigned(ncell2);
  if (tid < G) cls_count[tid] = 0;
  if (tid < G2) cls2_count[tid] = 0;
  if ((use_tma || use_tma2) && tid == 0) mbar_init(&tile_bar, 1);
  __syncthreads();
  if (use_tma && tid == 0) {
    mbar_expect_tx(&tile_bar, tile_bytes);
    tma_load_4d(tile, &cp.tmap, 2 * (org0 - XO), org1 - PAD, org2 - PAD, 0, &tile_bar);
  }
  // class and rank in class of this thread's points (p = tid + 256 k), for
  // the complex tile and (NF == 2) the real one
  int code[PPT], code2[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int p = tid + 256 * k;
    code[k] = -1;
    code2[k] = -1;
    if (p >= cnt) continue;
    const Rec<3, T> r = recs[start + p];
    int c0, c1, c2;
    unpack_cell(3, r.cell, c0, c1, c2);
    T u;
    const int b0 = c0 - org0 + es_start<W, T>(r.f[0], u);
    const int l1 = c1 - org1 + es_start<W, T>(r.f[1], u) + PAD;
    const int l2 = c2 - org2 + es_start<W, T>(r.f[2], u) + PAD;
    const int cls = ((l2 * TY + l1) * TX + b0 + XO) & (G - 1);
    code[k] = (cls << 12) | atomicAdd(&cls_count[cls], 1);
    if (NF == 2) {
      const int c2r = ((l2 * TY + l1) * TXR + b0 + XR) & (G2 - 1);
      code2[k] = (c2r << 12) | atomicAdd(&cls2_count[c2r], 1);
    }
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int c = 0; c < G; ++c) {
      cls_start[c] = acc;
      acc += cls_count[c];
    }
  } else if (NF == 2 && tid == 32) {
    int acc = 0;
    for (int c = 0; c < G2; ++c) {
      cls2_start[c] = acc;
      acc += cls2_count[c];
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    if (code[k] >= 0) order[cls_start[code[k] >> 12] + (code[k] & 0xfff)] = uint16_t(tid + 256 * k);
    if (NF == 2 && code2[k] >= 0) order2[cls2_start[code2[k] >> 12] + (code2[k] & 0xfff)] = uint16_t(tid + 256 * k);
  }
  int tma_phase = 0;  // tensor copies completed on tile_bar
  for (int f = 0; f < NF; ++f) {
    const bool real_pass = NF == 2 && f == 1;
    const bool tma_f = real_pass ? use_tma2 : use_tma;
    if (tma_f) {
      if (f > 0) {
        __syncthreads();  // every thread is done with the previous field's tile
        if (tid == 0) {
          // the tile's reads through the generic proxy come before the copy's writes
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(&tile_bar, tile2_bytes);
          tma_load_3d(rtile, &cp.tmap2, org0 - XR, org1 - PAD, org2 - PAD, &tile_bar);
        }
      }
      // bounded waits as in the 2D kernel: a retry raises STATUS_TILE_RETRY; a
      // copy that never lands fails the evaluation (STATUS_TIMEOUT, NaN energy
      // and NaN results for the block's points)
      const unsigned parity = unsigned(tma_phase & 1);
      ++tma_phase;
      const bool ok = mbar_wait_bounded(&tile_bar, parity, cp.polls);
      if (__syncthreads_or(!ok)) {
        if (tid == 0 && status != nullptr) raise_status(const_cast<int*>(status), STATUS_TILE_RETRY);
        const bool ok2 = mbar_wait_timed(&tile_bar, parity, kTileWaitNs);
        if (__syncthreads_or(!ok2)) {
          const T nan = T(__longlong_as_double(0x7ff8000000000000ULL));
          if (tid == 0) {
            if (status != nullptr) raise_status(const_cast<int*>(status), STATUS_TIMEOUT);
            if (cp.energy != nullptr) *cp.energy = double(nan);
          }
          for (int p = tid; p < cnt; p += blockDim.x)
            interp_store<3, T>(mode, recs[start + p].idx, T(1), nan, nan, nan, true, grad, out2, accumulate, gs);
          return;
        }
      }
    } else if (real_pass) {
      __syncthreads();  // every thread is done with the first field's tile
      const T* fld = reinterpret_cast<const T*>(fields + g.G());
      constexpr int BT = 4;  // loads in flight per thread
      for (int i0 = tid; i0 < ncell2; i0 += BT * 256) {
        T v[BT];
#pragma unroll
        for (int b = 0; b < BT; ++b) {
          const int i = i0 + b * 256;
          if (i < ncell2) {
            const int x = i % TXR, r = i / TXR;
            const int y = r % TY, z = r / TY;
            v[b] = fld[(int64_t(wrap_index(org2 - PAD + z, nf2)) * nf1 + wrap_index(org1 - PAD + y, nf1)) * nf0 +
                       wrap_index(org0 - XR + x, nf0)];
          }
        }
#pragma unroll
        for (int b = 0; b < BT; ++b)
          if (i0 + b * 256 < ncell2) rtile[i0 + b * 256] = v[b];
      }
    } else {
      __syncthreads();  // the order is complete
      const cplx_t<T>* fld = fields;
      constexpr int BT = 4;  // loads in flight per thread
      for (int i0 = tid; i0 < ncell; i0 += BT * 256) {
        cplx_t<T> v[BT];
#pragma unroll
        for (int b = 0; b < BT; ++b) {
          const int i = i0 + b * 256;
          if (i < ncell) {
            const int x = i % TX, r = i / TX;
            const int y = r % TY, z = r / TY;
            v[b] = fld[(int64_t(wrap_index(org2 - PAD + z, nf2)) * nf1 + wrap_index(org1 - PAD + y, nf1)) * nf0 +
                       wrap_index(org0 - XO + x, nf0)];
          }
        }
#pragma unroll
        for (int b = 0; b < BT; ++b)
          if (i0 + b * 256 < ncell) tile[i0 + b * 256] = v[b];
      }
    }
    __syncthreads();
    if (real_pass) {
      // the real field: lane c of every warp takes points of class c (mod 32)
      const int cls = tid % G2, grp = tid / G2, ngrp = int(blockDim.x) / G2;
      const int n_c = cls2_count[cls];
      const uint16_t* mine = order2 + cls2_start[cls];
      for (int j = grp; j < n_c; j += ngrp) {
        const int p = mine[j];
        const Rec<3, T> r = recs[start + p];
        int c0, c1, c2;
        unpack_cell(3, r.cell, c0, c1, c2);
        T k0[W], k1[W], k2[W];
        const int l0 = c0 - org0 + es_taps<W, T>(r.f[0], poly, k0) + XR;
        const int l1 = c1 - org1 + es_taps<W, T>(r.f[1], poly, k1) + PAD;
        const int l2 = c2 - org2 + es_taps<W, T>(r.f[2], poly, k2) + PAD;
        T vr = 0;
        for (int m2 = 0; m2 < W; ++m2) {
          T pr = 0;
#pragma unroll
          for (int m1 = 0; m1 < W; ++m1) {
            const T* rowp = rtile + (l2 + m2) * TY * TXR + (l1 + m1) * TXR + l0;
            T rr = 0;
#pragma unroll
            for (int m0 = 0; m0 < W; ++m0) rr += rowp[m0] * k0[m0];
            pr += k1[m1] * rr;
          }
          vr += k2[m2] * pr;
        }
        const T wgt = (mode == INTERP_GRAD) ? (weights ? weights[r.idx] : uniform) : T(1);
        const cplx_t<T> s0 = first[p];
        interp_store<3, T>(mode, r.idx, wgt, s0.x, s0.y, vr, bad, grad, out2, accumulate, gs);
      }
      continue;
    }
    const int cls = tid % G, grp = tid / G, ngrp = int(blockDim.x) / G;
    const int n_c = cls_count[cls];
    const uint16_t* mine = order + cls_start[cls];
    for (int j = grp; j < n_c; j += ngrp) {
      const int p = mine[j];
      const Rec<3, T> r = recs[start + p];
      int c0, c1, c2;
      unpack_cell(3, r.cell, c0, c1, c2);
      T k0[W], k1[W], k2[W];
      const int l0 = c0 - org0 + es_taps<W, T>(r.f[0], poly, k0) + XO;
      const int l1 = c1 - org1 + es_taps<W, T>(r.f[1], poly, k1) + PAD;
      const int l2 = c2 - org2 + es_taps<W, T>(r.f[2], poly, k2) + PAD;
      T vr = 0, vi = 0;
      for (int m2 = 0; m2 < W; ++m2) {
        T pr = 0, pi = 0;
#pragma unroll
        for (int m1 = 0; m1 < W; ++m1) {
          const cplx_t<T>* rowp = tile + (int64_t(l2 + m2) * TY + (l1 + m1)) * TX + l0;
          T rr = 0, ri = 0;
#pragma unroll
          for (int m0 = 0; m0 < W; ++m0) {
            const cplx_t<T> a = rowp[m0];
            rr += a.x * k0[m0];
            ri += a.y * k0[m0];
          }
          pr += k1[m1] * rr;
          pi += k1[m1] * ri;
        }
        vr += k2[m2] * pr;
        vi += k2[m2] * pi;
      }
      if (NF == 2) {
        cplx_t<T> s0;
        s0.x = vr;
        s0.y = vi;
        first[p] = s0;  // read back in the real field's pass
      } else {
        const T wgt = (mode == INTERP_GRAD) ? (weights ? weights[r.idx] : uniform) : T(1);
        interp_store<3, T>(mode, r.idx, wgt, vr, vi, T(0), bad, grad, out2, accumulate, gs);
      }
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

// Decides (once per point count) whether the one-pass sort can run: a
// cooperative launch of at most one 1024-thread block per SM whose chunk of
// points fits in shared memory next to the bin arrays (config 2's 2^20
// points over 148 SMs: 7085 points, 126 KB in FP32, 182 KB in FP64).
// The barrier's tickets assume one block count for every launch on a
// counter, so the configuration is fixed at the first sort; a later sort of
// another point count uses the two-pass sort.
template <int D, typename T>
bool onepass_setup(SortBufs& sb, int64_t N, const Geom& g) {
  if (sb.one_blocks >= 0) return sb.one_blocks > 0 && sb.one_N == N;
  sb.one_blocks = 0;
  sb.one_N = N;
  if (N < 1) return false;
  int dev = 0, coop = 0, smem_max = 0;
  FB_CUDA(cudaGetDevice(&dev));
  FB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  FB_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (!coop) return false;
  const int blocks = int(std::min<int64_t>(sm_count(), ceil_div(N, kOneThreads)));
  const int64_t chunk = ceil_div(N, blocks);
  const size_t smem = onepass_bin_bytes(int(g.nbins())) + size_t(chunk) * onepass_point_bytes<D, T>();
  if (chunk > 65535 || smem + 1024 > size_t(smem_max)) return false;
  auto kern = sort_onepass_kernel<D, T>;
  ensure_dynamic_smem(kern, smem);
  int occ = 0;
  FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kOneThreads, smem));
  if (occ < 1 || blocks > occ * sm_count()) return false;
  sb.one_blocks = blocks;
  sb.one_chunk = chunk;
  sb.one_smem = smem;
  return true;
}

template <int D, typename T>
void bin_sort_d(const double* pts, int64_t N, const MapParams& mp, const Geom& g, SortBufs& sb, void* recs, int* status,
                cudaStream_t s) {
  const int nbins = int(g.nbins());
  const size_t smem = sizeof(int) * size_t(nbins);
  auto k1 = sort_count_kernel<D, T>;
  auto k3 = sort_scatter_kernel<D, T>;
  MapParams m2 = mp;
  for (int a = 0; a < D; ++a) {
    m2.scale[a] = double(g.nf[a]) / mp.L[a];
    m2.invL[a] = 1.0 / mp.L[a];
  }
  if (onepass_setup<D, T>(sb, N, g)) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(sb.one_blocks));
    cfg.blockDim = dim3(kOneThreads);
    cfg.dynamicSmemBytes = sb.one_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FB_CUDA(cudaLaunchKernelEx(&cfg, sort_onepass_kernel<D, T>, pts, N, sb.one_chunk, m2, g, sb.bin_total.p,
                               sb.bin_start.p, sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p,
                               int(sb.max_sub), sb.done.p, sb.bar.p, static_cast<Rec<D, T>*>(recs), status));
    return;
  }
  Rec<D, T>* unsorted = reinterpret_cast<Rec<D, T>*>(sb.unsorted.p);
  if (smem > 48 * 1024) {
    ensure_dynamic_smem(k1, smem);
    ensure_dynamic_smem(k3, smem);
  }
  if (N > 0) {
    k1<<<sb.NB, kSortThreads, smem, s>>>(pts, N, sb.chunk, m2, g, sb.bin_total.p, sb.blk_off.p, unsorted, status);
    FB_LAUNCH_CHECK();
  }
  k3<<<sb.NB, kSortThreads, smem, s>>>(unsorted, N, sb.chunk, g, sb.bin_total.p, sb.blk_off.p, sb.bin_start.p,
                                       sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, int(sb.max_sub),
                                       sb.done.p, static_cast<Rec<D, T>*>(recs), status);
  FB_LAUNCH_CHECK();
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
  if constexpr (sizeof(T) == 4 && !CPLX && W >= 4 && W <= 8) {
    if (g.nf[0] % 4 == 0) {
      constexpr size_t smem_f = spread2d_tpp_smem_bytes<W>();
      auto kf = spread2d_tpp_kernel<W, TileMap1<float>>;
      if (smem_f > 48 * 1024) ensure_dynamic_smem(kf, smem_f);
      const TileMap1<float> map{sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, sb.bin_start.p, nullptr,
                                uniform};
      kf<<<unsigned(sb.max_sub), 256, smem_f, s>>>(static_cast<const Rec<2, float>*>(recs), weights, map, g,
                                                   make_es_poly<W, T>(poly), grid_real);
      FB_LAUNCH_CHECK();
      return;
    }
  }
  constexpr size_t smem = spread2d_smem_bytes<W, T, CPLX>();
  auto kern = spread2d_tile_kernel<W, T, CPLX, TileMap1<T>>;
  if (smem > 48 * 1024) ensure_dynamic_smem(kern, smem);
  const TileMap1<T> map{sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, sb.bin_start.p, nullptr, uniform};
  kern<<<unsigned(sb.max_sub), Tile2D<W>::THREADS, smem, s>>>(static_cast<const Rec<2, T>*>(recs), weights, strengths,
                                                              map, g, make_es_poly<W, T>(poly), grid_real, grid_cplx);
  FB_LAUNCH_CHECK();
}

template <int D, int W, typename T, bool CPLX>
void launch_spread_generic(const void* recs, const T* weights, T uniform, const cplx_t<T>* strengths,
                           const SortBufs& sb, const Geom& g, const std::vector<double>& poly, T* grid_real,
                           cplx_t<T>* grid_cplx, cudaStream_t s) {
  if constexpr (D == 3 && W <= 8 && !CPLX && sizeof(T) == 4) {
    const size_t smem_t = spread3d_tpp_smem_bytes<W>(g);
    if (g.nf[0] % 4 == 0 && g.tile[0] % 4 == 0 && smem_t <= 200 * 1024) {
      auto kt = spread3d_tpp_kernel<W>;
      if (smem_t > 48 * 1024) ensure_dynamic_smem(kt, smem_t);
      kt<<<unsigned(sb.max_sub), Tpp3D<W>::NT, smem_t, s>>>(
          static_cast<const Rec<3, float>*>(recs), weights, uniform, sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p,
          sb.num_sub.p, sb.bin_start.p, g, make_es_poly<W, T>(poly), spread3d_tpp_pitch(g.tw[0], W), grid_real);
      FB_LAUNCH_CHECK();
      return;
    }
  }
  if constexpr (D == 3 && W <= 8 && !CPLX) {
    const int pitch = spread3d_pitch(g.tw[0], W);
    const size_t smem3 = size_t(pitch) * g.tw[1] * g.tw[2] * sizeof(T);
    auto k3 = spread3d_warp_kernel<W, T>;
    if (smem3 <= 200 * 1024) {
      if (smem3 > 48 * 1024)
        ensure_dynamic_smem(k3, smem3);
      k3<<<unsigned(sb.max_sub), 256, smem3, s>>>(static_cast<const Rec<3, T>*>(recs), weights, uniform,
                                                 sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                 make_es_poly<W, T>(poly), pitch, grid_real);
      FB_LAUNCH_CHECK();
      return;
    }
  }
  const size_t smem = size_t(g.tile_cells()) * sizeof(T) * (CPLX ? 2 : 1);
  auto kern = spread_kernel<D, W, T, CPLX>;
  if (smem > 48 * 1024) ensure_dynamic_smem(kern, smem);
  kern<<<unsigned(sb.max_sub), 256, smem, s>>>(static_cast<const Rec<D, T>*>(recs), weights, uniform, strengths,
                                                sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                make_es_poly<W, T>(poly), grid_real, grid_cplx);
  FB_LAUNCH_CHECK();
}

// Tensor map of a complex fine grid nf0 x nf1 (cells of two T) for tile
// copies of box_x T values x box_y rows; returns 0 (plain loads are used) if
// the driver has no encoder or the grid does not meet the copy rules.
template <typename T>
int encode_tile_tmap(CUtensorMap* tm, const void* grid, int64_t nf0, int64_t nf1, int box_x, int box_y) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return Encode(nullptr);
    }
    return reinterpret_cast<Encode>(fn);
  }();
  const uint64_t row_bytes = uint64_t(nf0) * 2 * sizeof(T);
  if (!encode || grid == nullptr || (reinterpret_cast<uintptr_t>(grid) & 15) || row_bytes % 16 ||
      nf0 % kTile2D || nf1 % kTile2D || box_x > 256 || box_y > 256 || (box_x * sizeof(T)) % 16)
    return 0;
  const cuuint64_t dims[2] = {cuuint64_t(2 * nf0), cuuint64_t(nf1)};
  const cuuint64_t strides[1] = {row_bytes};
  const cuuint32_t box[2] = {cuuint32_t(box_x), cuuint32_t(box_y)};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const CUresult r = encode(tm, dt, 2, const_cast<void*>(grid), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 1 : 0;
}

template <int W, typename T>
void launch_interp2d(const void* recs, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
                     const std::vector<double>& poly, const cplx_t<T>* field, int mode, double* grad, double2* out2,
                     int acc, const int* status, cudaStream_t s, const GradScale& gs, double* fail_energy) {
  constexpr size_t smem = interp2d_smem_bytes<W, T>();
  auto kern = interp2d_tile_kernel<W, T, TileMap1<T>>;
  if (smem > 48 * 1024) ensure_dynamic_smem(kern, smem);
  TileMap1<T> map{sb.sub_bin.p, sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, sb.bin_start.p, status, uniform};
  map.polls = tile_wait_polls_setting();
  map.energy = fail_energy;
  map.has_tmap = encode_tile_tmap<T>(&map.tmap, field, g.nf[0], g.nf[1], 2 * Interp2D<W>::TWX, Interp2D<W>::TWY);
  kern<<<unsigned(sb.max_sub), 256, smem, s>>>(static_cast<const Rec<2, T>*>(recs), weights, map, g,
                                                make_es_poly<W, T>(poly), field, mode, grad, out2, acc, gs);
  FB_LAUNCH_CHECK();
}

// Tensor map of nfields complex fields of nf0 x nf1 x nf2 cells (x fastest)
// as 4D floats (2 nf0, nf1, nf2, nfields) with a box of (box_x floats,
// box_y, box_z, 1); 0 when the layout does not allow tensor copies.
template <typename T>
int encode_fields_tmap3(CUtensorMap* tm, const void* fields, int64_t nf0, int64_t nf1, int64_t nf2, int nfields,
                        int box_x, int box_y, int box_z) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return Encode(nullptr);
    }
    return reinterpret_cast<Encode>(fn);
  }();
  const uint64_t row = uint64_t(nf0) * 2 * sizeof(T), plane = row * uint64_t(nf1), field = plane * uint64_t(nf2);
  if (!encode || fields == nullptr || (reinterpret_cast<uintptr_t>(fields) & 15) || row % 16 || plane % 16 ||
      field % 16 || box_x > 256 || box_y > 256 || box_z > 256 || (box_x * sizeof(T)) % 16 ||
      box_x > 2 * nf0 || box_y > nf1 || box_z > nf2)
    return 0;
  const cuuint64_t dims[4] = {cuuint64_t(2 * nf0), cuuint64_t(nf1), cuuint64_t(nf2), cuuint64_t(nfields)};
  const cuuint64_t strides[3] = {row, plane, field};
  const cuuint32_t box[4] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(box_z), 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const CUresult r = encode(tm, dt, 4, const_cast<void*>(fields), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 1 : 0;
}

// Tensor map of a real grid of nf0 x nf1 x nf2 values of T (x fastest) with a
// box of (box_x, box_y, box_z); 0 when the layout does not allow tensor copies.
template <typename T>
int encode_real_tmap3(CUtensorMap* tm, const void* grid, int64_t nf0, int64_t nf1, int64_t nf2, int box_x, int box_y,
                      int box_z) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const Encode encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return Encode(nullptr);
    }
    return reinterpret_cast<Encode>(fn);
  }();
  const uint64_t row = uint64_t(nf0) * sizeof(T), plane = row * uint64_t(nf1);
  if (!encode || grid == nullptr || (reinterpret_cast<uintptr_t>(grid) & 15) || row % 16 || plane % 16 ||
      box_x > 256 || box_y > 256 || box_z > 256 || (box_x * sizeof(T)) % 16 || box_x > nf0 || box_y > nf1 ||
      box_z > nf2)
    return 0;
  const cuuint64_t dims[3] = {cuuint64_t(nf0), cuuint64_t(nf1), cuuint64_t(nf2)};
  const cuuint64_t strides[2] = {row, plane};
  const cuuint32_t box[3] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(box_z)};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const CUresult r = encode(tm, dt, 3, const_cast<void*>(grid), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 1 : 0;
}

// 3D FP32: the tile kernel when a bin's tile + halo fits in shared memory
// (false otherwise, and for FP64, whose w^3 loop needs 255 registers and one
// block per SM in this form: the caller uses the gathering kernel).
template <int W, typename T>
bool launch_interp3d(const void* recs, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
                     const std::vector<double>& poly, const cplx_t<T>* fields, int nfields, int mode, double* grad,
                     double2* out2, int acc, const int* status, cudaStream_t s, const GradScale& gs,
                     double* fail_energy) {
  if constexpr (sizeof(T) != 4) {
    return false;
  } else {
    using IP = Interp3D<W>;
    const int TX = IP::txp(g.tile[0]), TXR = IP::txr(g.tile[0]), TY = g.tile[1] + W, TZ = g.tile[2] + W;
    size_t tile_bytes = size_t(TX) * TY * TZ * sizeof(cplx_t<T>);
    if (nfields == 2)  // the real field's tile shares the buffer (the kernel's tile_cells)
      tile_bytes = std::max(tile_bytes, (size_t(TXR) * TY * TZ * sizeof(T) + sizeof(cplx_t<T>) - 1) /
                                            sizeof(cplx_t<T>) * sizeof(cplx_t<T>));
    if (nfields < 1 || nfields > 2) return false;
    const size_t smem = tile_bytes + (nfields == 2 ? interp3d_extra_bytes<W, T, 2>() : interp3d_extra_bytes<W, T, 1>());
    if (smem > 160 * 1024) return false;
    auto kern2 = interp3d_tile_kernel<W, T, 2>;
    auto kern1 = interp3d_tile_kernel<W, T, 1>;
    auto kern = nfields == 2 ? kern2 : kern1;
    ensure_dynamic_smem(kern, smem);
    Tile3Copy cp;
    cp.has_tmap = g.tile[0] % 2 == 0 ? encode_fields_tmap3<T>(&cp.tmap, fields, g.nf[0], g.nf[1], g.nf[2], 1,
                                                               2 * TX, TY, TZ)
                                     : 0;
    // the real field's copies start at x = org0 - XR: a multiple of 4 floats when the tile edge is
    cp.has_tmap2 = (nfields == 2 && g.tile[0] % 4 == 0)
                       ? encode_real_tmap3<T>(&cp.tmap2, fields + g.G(), g.nf[0], g.nf[1], g.nf[2], TXR, TY, TZ)
                       : 0;
    cp.polls = tile_wait_polls_setting();
    cp.energy = fail_energy;
    kern<<<unsigned(sb.max_sub), 256, smem, s>>>(static_cast<const Rec<3, T>*>(recs), weights, uniform, sb.sub_bin.p,
                                                 sb.sub_start.p, sb.sub_count.p, sb.num_sub.p, g,
                                                 make_es_poly<W, T>(poly), fields, mode, grad, out2, acc, status, gs,
                                                 cp);
    FB_LAUNCH_CHECK();
    return true;
  }
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
            double2* out2, int accumulate, const int* status, cudaStream_t s, GradScale gs, double* fail_energy) {
  if (g.D == 2 && nfields == 1) {
#define FB_I2(WW)                                                                                                  \
  launch_interp2d<FB_WCLAMP(T, WW), T>(recs, weights, uniform, sb, g, poly, fields, mode, grad, out2, accumulate, \
                                       status, s, gs, fail_energy)
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
    if (N <= 0) return;
#define FB_I3(WW)                                                                                              \
  if (!launch_interp3d<FB_WCLAMP(T, WW), T>(recs, weights, uniform, sb, g, poly, fields, nfields, mode, grad,     \
                                            out2, accumulate, status, s, gs, fail_energy))                        \
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
                          const cplx_t<T>*, int, int, double*, double2*, int, const int*, cudaStream_t, GradScale, \
                          double*);

}  // namespace fb
